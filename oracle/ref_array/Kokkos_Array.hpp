// Oracle-only stand-in for Kokkos::Array in the array build (test
// infrastructure): a fixed-size aggregate with operator[], data(), begin() /
// end() (the reference feeds it to std::ranges algorithms) and the tuple
// protocol (the reference unpacks it with structured bindings).
#pragma once

#include <cstddef>
#include <tuple>
#include <type_traits>

#include "Kokkos_Macros.hpp"

namespace Kokkos {

template <class T, std::size_t N>
struct Array {
    T m_data[N > 0 ? N : 1];
    constexpr T& operator[](std::size_t i) noexcept { return m_data[i]; }
    constexpr T const& operator[](std::size_t i) const noexcept { return m_data[i]; }
    static constexpr std::size_t size() noexcept { return N; }
    constexpr T* data() noexcept { return m_data; }
    constexpr T const* data() const noexcept { return m_data; }
    constexpr T* begin() noexcept { return m_data; }
    constexpr T* end() noexcept { return m_data + N; }
    constexpr T const* begin() const noexcept { return m_data; }
    constexpr T const* end() const noexcept { return m_data + N; }
};

template <std::size_t I, class T, std::size_t N>
constexpr T& get(Array<T, N>& a) noexcept
{
    return a.m_data[I];
}
template <std::size_t I, class T, std::size_t N>
constexpr T const& get(Array<T, N> const& a) noexcept
{
    return a.m_data[I];
}
template <std::size_t I, class T, std::size_t N>
constexpr T&& get(Array<T, N>&& a) noexcept
{
    return static_cast<T&&>(a.m_data[I]);
}

} // namespace Kokkos

template <class T, std::size_t N>
struct std::tuple_size<Kokkos::Array<T, N>> : std::integral_constant<std::size_t, N> {
};
template <std::size_t I, class T, std::size_t N>
struct std::tuple_element<I, Kokkos::Array<T, N>> {
    using type = T;
};
