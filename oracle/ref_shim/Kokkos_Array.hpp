// Oracle-only stand-in for Kokkos::Array: a fixed-size aggregate with
// operator[] (all the per-cell headers need).
#pragma once
#include <cstddef>
#include "Kokkos_Macros.hpp"
namespace Kokkos {
template <class T, std::size_t N>
struct Array
{
    T m_data[N > 0 ? N : 1];
    constexpr T& operator[](std::size_t i) noexcept { return m_data[i]; }
    constexpr T const& operator[](std::size_t i) const noexcept { return m_data[i]; }
    static constexpr std::size_t size() noexcept { return N; }
};
} // namespace Kokkos
