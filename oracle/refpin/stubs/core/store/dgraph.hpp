// Stand-in for the reference's graph-store base class: the engine reaches the store only
// through get_triples / get_index (and get_attr, unused without attributes); the checker's
// graph serves lists it was given.  Test infrastructure only.
#pragma once
#include <cstdint>
#include "core/common/type.hpp"
#include "core/store/vertex.hpp"
namespace wukong {
class DGraph {
public:
    virtual ~DGraph() {}
    virtual edge_t* get_triples(int tid, sid_t vid, sid_t pid, dir_t d, uint64_t& sz) = 0;
    virtual edge_t* get_index(int tid, sid_t pid, dir_t d, uint64_t& sz) = 0;
    virtual attr_t get_attr(int tid, sid_t vid, sid_t pid, dir_t d, bool& has_value) {
        has_value = false;
        return attr_t();
    }
};
}  // namespace wukong
