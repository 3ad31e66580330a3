// Oracle-only stand-in for Kokkos::numbers.
#pragma once
#include <numbers>
namespace Kokkos::numbers {
inline constexpr double pi = std::numbers::pi;
inline constexpr double ln2 = std::numbers::ln2;
} // namespace Kokkos::numbers
