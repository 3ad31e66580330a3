// Oracle-only stand-in: the Kokkos math wrappers map to the C++ library,
// which is what Kokkos' host backends call.
#pragma once
#include <cmath>
#include "Kokkos_Macros.hpp"
namespace Kokkos {
using std::abs;
using std::cos;
using std::fabs;
using std::fmax;
using std::fmin;
using std::isfinite;
using std::isnan;
using std::pow;
using std::sin;
using std::sqrt;
} // namespace Kokkos
