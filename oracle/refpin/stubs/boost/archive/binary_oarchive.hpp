// Stand-in: the archive names the reference's serialization code mentions (never used here).
#pragma once
namespace boost { namespace archive {
class binary_iarchive {};
class binary_oarchive {};
}}  // namespace boost::archive
