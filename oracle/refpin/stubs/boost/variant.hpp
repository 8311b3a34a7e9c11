// Stand-in: boost::variant / static_visitor / apply_visitor / get over std::variant.
#pragma once
#include <variant>
namespace boost {
template <class... T>
class variant : public std::variant<T...> {
public:
    using std::variant<T...>::variant;
    variant() = default;
    int which() const { return (int)this->index(); }
};
template <class R = void>
struct static_visitor {
    typedef R result_type;
};
template <class Vis, class... T>
auto apply_visitor(const Vis& vis, const variant<T...>& v) {
    return std::visit(vis, static_cast<const std::variant<T...>&>(v));
}
template <class U, class... T>
U& get(variant<T...>& v) { return std::get<U>(static_cast<std::variant<T...>&>(v)); }
template <class U, class... T>
const U& get(const variant<T...>& v) { return std::get<U>(static_cast<const std::variant<T...>&>(v)); }
}  // namespace boost
