// Stand-in for the reference's string server: ids are their own strings.  The pattern
// operators and DISTINCT / OFFSET / LIMIT never ask for strings; only ORDER BY and string
// filters would, and the checker runs neither.  Test infrastructure only.
#pragma once
#include <string>
#include <utility>
#include "core/common/type.hpp"
namespace wukong {
class StringMapping {
public:
    std::pair<bool, std::string> id2str(int tid, sid_t id) { return {true, std::to_string(id)}; }
    std::pair<bool, sid_t> str2id(int tid, const std::string& s) { return {true, (sid_t)std::stoul(s)}; }
};
}  // namespace wukong
