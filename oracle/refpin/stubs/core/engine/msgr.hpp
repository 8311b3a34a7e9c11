// Stand-in for the reference's messenger and bundle: in one process with one server and one
// engine thread the engine only ever sends its final reply, which this messenger keeps for the
// caller.  Test infrastructure only.
#pragma once
#include <vector>
#include "core/sparql/query.hpp"
#include "stringserver/string_mapping.hpp"
namespace wukong {
class Bundle {
public:
    SPARQLQuery query;
    explicit Bundle(const SPARQLQuery& r) : query(r) {}
};
class Messenger {
public:
    std::vector<SPARQLQuery> replies;
    bool send_msg(Bundle& b, int dst_sid, int dst_tid) {
        replies.push_back(b.query);
        return true;
    }
};
}  // namespace wukong
