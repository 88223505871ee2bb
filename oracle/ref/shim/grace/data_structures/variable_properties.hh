// Declares only the type names the variable-index header refers to.
#pragma once
#include <cstddef>
namespace grace {
enum bc_t { BC_NONE_SHIM = 0 };
enum var_amr_interp_t { INTERP_NONE_SHIM = 0 };
template <std::size_t N> struct variable_properties_t {};
}
