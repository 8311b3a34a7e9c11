// Stand-in: boost::unordered_map as std::unordered_map (see wk_stub_hash.hpp).
#pragma once
#include <unordered_map>
#include "boost/wk_stub_hash.hpp"
namespace boost {
template <class K, class V, class H = boost::hash<K>, class E = std::equal_to<K>>
using unordered_map = std::unordered_map<K, V, H, E>;
}
