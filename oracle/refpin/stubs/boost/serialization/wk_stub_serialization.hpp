// Stand-in: the serialization names and macros the reference's headers mention.  Nothing here
// serializes; the engine is run in one process and its messages are never encoded.
#pragma once
namespace boost { namespace serialization {
class access {};
enum level_type { object_serializable = 1 };
enum tracking_type { track_never = 0 };
template <class Archive, class T>
void split_free(Archive&, T&, const unsigned int) {}
template <class Archive, class T>
void split_member(Archive&, T&, const unsigned int) {}
}}  // namespace boost::serialization
#ifndef BOOST_CLASS_IMPLEMENTATION
#define BOOST_CLASS_IMPLEMENTATION(T, L)
#define BOOST_CLASS_TRACKING(T, L)
#define BOOST_SERIALIZATION_SPLIT_FREE(T)
#define BOOST_SERIALIZATION_SPLIT_MEMBER()
#endif
