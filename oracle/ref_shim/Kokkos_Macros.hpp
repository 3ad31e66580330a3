// Minimal stand-in for the few Kokkos macros that the reference's per-cell
// physics headers use.  Written for the oracle build only: it lets
// hydro/euler_equations.hpp, hydro/riemann_solver.hpp, hydro/slope_limiters.hpp,
// hydro/source_terms.hpp and thermodynamics/perfect_gas.hpp compile as plain
// host C++ so the oracle can be checked against the reference's own code.
#pragma once
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
