// Stand-in: boost::unordered_set as std::unordered_set (see wk_stub_hash.hpp).
#pragma once
#include <unordered_set>
#include "boost/wk_stub_hash.hpp"
namespace boost {
template <class T, class H = boost::hash<T>, class E = std::equal_to<T>>
using unordered_set = std::unordered_set<T, H, E>;
}
