// setups.hpp -- setup plugins (initial primitive state on the interior).
//
// Same contract as the reference (src/initialization_interface.hpp:18-40 and
// src/setups/<name>/setup.hpp): the [Initialisation] section parameterises
// the setup, which writes rho, u, P on the no_ghosts range; ghosts are filled
// later by the boundary conditions (main.cpp:305-307).
#pragma once

#include <cstdint>
#include <string>

#include "ini_reader.hpp"

namespace hcl::host {

// Uniform double in [0, 1) from (seed, i, j, k): splitmix64 chained over the
// global interior index, so every cell's perturbation is independent of the
// grid split and evaluation order.
double hash_uniform(uint64_t seed, uint64_t i, uint64_t j, uint64_t k);

struct SetupGrid {
    int ndim;
    int n[3];          // extents with ghosts
    int ng;
    const double* xc[3];
};

// Fills rho (N), u (N*ndim), P (N) in LayoutLeft on the interior cells.
// Throws std::runtime_error for an unknown setup name.
void setup_initial_prim(std::string const& name, INIReader const& reader, SetupGrid const& g, double* rho, double* u,
                        double* P);

} // namespace hcl::host
