// Test-infrastructure shim (oracle build only): maps the two boost::variant
// uses in the reference's loquat_io (a typed parameter map and boost::get) onto
// std::variant, and supplies the stream operator boost provides.
#pragma once
#include <ostream>
#include <variant>

namespace boost {
template <class... Ts>
using variant = std::variant<Ts...>;
using std::get;
}  // namespace boost

template <class T0, class... Ts>
std::ostream& operator<<(std::ostream& os, const std::variant<T0, Ts...>& v) {
  std::visit([&os](const auto& x) { os << x; }, v);
  return os;
}
