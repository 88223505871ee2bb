// Declares only the type names the variable-index and AMR helper headers
// refer to.
#pragma once
#include <cstddef>
#include <cstdint>
#include <array>
namespace grace {
enum bc_t { BC_NONE_SHIM = 0 };
// the staggering names and array types the AMR helper headers mention
enum var_staggering_t : uint8_t {
  STAG_CENTER = 0, STAG_FACEX, STAG_FACEY, STAG_EDGEXY, STAG_FACEZ, STAG_EDGEXZ, STAG_EDGEYZ, STAG_CORNER,
  N_VAR_STAGGERINGS
};
inline std::array<int, 3> get_index_staggerings(var_staggering_t stag) {
  return {stag & 1, (stag >> 1) & 1, (stag >> 2) & 1};
}
struct var_array_t {};
struct staggered_variable_arrays_t {
  var_array_t face_staggered_fields_x, face_staggered_fields_y, face_staggered_fields_z;
  var_array_t edge_staggered_fields_xy, edge_staggered_fields_xz, edge_staggered_fields_yz;
  var_array_t corner_staggered_fields;
};
enum var_amr_interp_t { INTERP_NONE_SHIM = 0 };
template <std::size_t N> struct variable_properties_t {};
}
