// Parameter lookup stand-in: a flat "a.b.c" -> value table that the checker
// glue fills before it constructs reference objects whose constructors read
// parameters (ideal_gas_eos_t reads eos.ideal_gas_eos.gamma / kappa_id).
#pragma once
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
namespace grace {
inline std::map<std::string, double>& shim_param_table() {
  static std::map<std::string, double> t;
  return t;
}
namespace shim_detail {
inline void join(std::ostringstream&) {}
template <class A, class... R> void join(std::ostringstream& o, A const& a, R const&... r) {
  o << a;
  if (sizeof...(R)) o << '.';
  join(o, r...);
}
}  // namespace shim_detail
template <class T, class... K> T get_param(K const&... keys) {
  std::ostringstream o;
  shim_detail::join(o, keys...);
  auto it = shim_param_table().find(o.str());
  if (it == shim_param_table().end()) throw std::runtime_error("checker: missing parameter " + o.str());
  if constexpr (std::is_arithmetic_v<T>) return static_cast<T>(it->second);
  else throw std::runtime_error("checker: non-numeric parameter " + o.str());
}
}  // namespace grace
