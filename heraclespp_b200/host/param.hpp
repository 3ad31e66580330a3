// param.hpp -- runtime parameters read from the .ini file, with the keys and
// defaults of the reference's Param (src/utils/param.cpp:14-73), plus the
// factory-key lookups of the plugins on the hot path.
#pragma once

#include <array>
#include <string>

#include "heracles_b200.h"
#include "ini_reader.hpp"

namespace hcl::host {

class Param
{
public:
    std::string problem;
    bool restart;
    std::string restart_file;
    double rmax_shift;
    std::array<int, 3> Nx_glob_ng;
    std::string grid_type;
    int Ng;
    double x0min, x0max, x1min, x1max, x2min, x2max;
    std::string shift_grid;
    bool mpi_device_aware;
    std::array<int, 3> mpi_dims_cart;
    double t_ini, t_end, cfl;
    int max_iter;
    int iter_output_frequency;
    double time_output_frequency;
    double time_first_output;
    std::string directory, prefix;
    int time_job;
    std::string reconstruction_type;
    std::string riemann_solver;
    double gx0, gx1, gx2, M;
    double gamma, mu;
    std::string bc_choice, bc_priority;
    int nfx;
    std::string user_step;
    std::string pressure_fix;
    double eps_pf;

    explicit Param(INIReader const& reader);
};

// factory_face_reconstruction (hydro/face_reconstruction.cpp:31-50); throws
// std::runtime_error("Unknown face reconstruction algorithm: X.")
int limiter_id(std::string const& name);
// factory_godunov_scheme (hydro/godunov_scheme.hpp:305-321); throws
// std::runtime_error("Invalid riemann solver: X.")
int riemann_id(std::string const& name);
// factory_boundary_construction (boundary_factory.hpp:31-47); throws
// std::runtime_error("Unknown boundary condition : X.")
int bc_id(std::string const& name);

// Per-face boundary names as main.cpp:174-185 resolves them: BC_X{d}_{left,
// right} falls back to BC_X{d}, which falls back to BC; throws
// std::runtime_error when a face stays undefined.
std::array<std::string, 6> resolve_boundaries(INIReader const& reader, Param const& param, int ndim);

// Builds the C-ABI configuration of one domain from the parameters.  ndim,
// geometry and gravity are compile-time choices in the reference (CMake
// options Heraclespp_NDIM/_GEOM/_GRAVITY) and are passed explicitly here.
hcl_config make_config(INIReader const& reader, Param const& param, int ndim, int geometry, int gravity,
                       int precision, int device);

} // namespace hcl::host
