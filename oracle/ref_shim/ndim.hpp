// Oracle-only replacement of the CMake-generated ndim.hpp (src/utils/ndim.hpp.in):
// the dimension comes from -DHCL_REF_NDIM=1|2|3.
#pragma once
namespace hclpp {
inline constexpr int ndim = HCL_REF_NDIM;
inline constexpr int nfaces = 2 * ndim;
} // namespace hclpp
