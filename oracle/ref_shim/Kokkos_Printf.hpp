// Oracle-only stand-in: Kokkos::printf maps to the C library's printf, as on
// Kokkos' host backends.
#pragma once
#include <cstdio>
#include "Kokkos_Macros.hpp"
namespace Kokkos {
using std::printf;
} // namespace Kokkos
