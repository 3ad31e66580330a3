// param.cpp -- see param.hpp.  Keys and defaults follow utils/param.cpp:14-73.
#include "param.hpp"

#include <stdexcept>
#include <string>

namespace hcl::host {

Param::Param(INIReader const& reader)
{
    problem = reader.Get("Problem", "type", "ShockTube");
    restart = reader.GetBoolean("Problem", "restart", false);
    restart_file = reader.Get("Problem", "restart_file", "None");
    rmax_shift = reader.GetReal("Problem", "rmax_shift", 1E20);

    Nx_glob_ng[0] = (int)reader.GetInteger("Grid", "Nx0_glob", 0);
    Nx_glob_ng[1] = (int)reader.GetInteger("Grid", "Nx1_glob", 0);
    Nx_glob_ng[2] = (int)reader.GetInteger("Grid", "Nx2_glob", 0);
    grid_type = reader.Get("Grid", "type", "Regular");
    Ng = (int)reader.GetInteger("Grid", "Nghost", 2);
    x0min = reader.GetReal("Grid", "x0min", 0.0);
    x0max = reader.GetReal("Grid", "x0max", 1.0);
    x1min = reader.GetReal("Grid", "x1min", 0.0);
    x1max = reader.GetReal("Grid", "x1max", 1.0);
    x2min = reader.GetReal("Grid", "x2min", 0.0);
    x2max = reader.GetReal("Grid", "x2max", 1.0);
    shift_grid = reader.Get("Grid", "shift_grid", "Off");

    mpi_device_aware = reader.GetBoolean("Parallelization", "mpi_device_aware", false);
    mpi_dims_cart[0] = (int)reader.GetInteger("Parallelization", "mpi_dims_cart_x0", 0);
    mpi_dims_cart[1] = (int)reader.GetInteger("Parallelization", "mpi_dims_cart_x1", 0);
    mpi_dims_cart[2] = (int)reader.GetInteger("Parallelization", "mpi_dims_cart_x2", 0);

    t_ini = reader.GetReal("Run", "t_ini", 0.);
    t_end = reader.GetReal("Run", "t_end", 0.2);
    cfl = reader.GetReal("Run", "cfl", 0.4);

    max_iter = (int)reader.GetInteger("Output", "max_iter", 10000);
    iter_output_frequency = (int)reader.GetInteger("Output", "iter_frequency", 0);
    time_output_frequency = reader.GetReal("Output", "time_frequency", 0.0);
    time_first_output = reader.GetReal("Output", "time_first_output", t_ini + time_output_frequency);
    directory = reader.Get("Output", "directory", ".");
    prefix = reader.Get("Output", "prefix", "result");
    time_job = (int)reader.GetInteger("Output", "time_job", 20);

    reconstruction_type = reader.Get("Hydro", "reconstruction", "VanLeer");
    riemann_solver = reader.Get("Hydro", "riemann_solver", "HLL");

    gx0 = reader.GetReal("Gravity", "gx0", 0.0);
    gx1 = reader.GetReal("Gravity", "gx1", 0.0);
    gx2 = reader.GetReal("Gravity", "gx2", 0.0);
    M = reader.GetReal("Gravity", "M", 1.0);

    gamma = reader.GetReal("Perfect Gas", "gamma", 5. / 3);
    mu = reader.GetReal("Perfect Gas", "mu", 1.);

    bc_choice = reader.Get("Boundary Condition", "BC", "");
    bc_priority = reader.Get("Boundary Condition", "priority", "");

    nfx = (int)reader.GetInteger("Passive Scalar", "nfx", 0);
    user_step = reader.Get("User step", "user_step", "Off");
    pressure_fix = reader.Get("Pressure fix", "pressure_fix", "Off");
    eps_pf = reader.GetReal("Pressure fix", "eps_pf", 0.000001);
}

int limiter_id(std::string const& name)
{
    if (name == "Constant") {
        return HCL_LIMITER_CONSTANT;
    }
    if (name == "VanLeer") {
        return HCL_LIMITER_VANLEER;
    }
    if (name == "Minmod") {
        return HCL_LIMITER_MINMOD;
    }
    if (name == "VanAlbada") {
        return HCL_LIMITER_VANALBADA;
    }
    throw std::runtime_error("Unknown face reconstruction algorithm: " + name + ".");
}

int riemann_id(std::string const& name)
{
    if (name == "HLL") {
        return HCL_RIEMANN_HLL;
    }
    if (name == "HLLC") {
        return HCL_RIEMANN_HLLC;
    }
    if (name == "Low Mach") {
        return HCL_RIEMANN_LOW_MACH;
    }
    throw std::runtime_error("Invalid riemann solver: " + name + ".");
}

int bc_id(std::string const& name)
{
    if (name == "NullGradient") {
        return HCL_BC_NULLGRADIENT;
    }
    if (name == "Periodic") {
        return HCL_BC_PERIODIC;
    }
    if (name == "Reflexive") {
        return HCL_BC_REFLEXIVE;
    }
    throw std::runtime_error("Unknown boundary condition : " + name + ".");
}

std::array<std::string, 6> resolve_boundaries(INIReader const& reader, Param const& param, int ndim)
{
    static const char* dirs[3] = {"_X0", "_X1", "_X2"};
    static const char* faces[2] = {"_left", "_right"};
    std::array<std::string, 6> out;
    for (int idim = 0; idim < 3; ++idim) {
        for (int iface = 0; iface < 2; ++iface) {
            out[2 * idim + iface] = "Periodic";
        }
    }
    for (int idim = 0; idim < ndim; ++idim) {
        const std::string dir = reader.Get("Boundary Condition", std::string("BC") + dirs[idim], param.bc_choice);
        for (int iface = 0; iface < 2; ++iface) {
            out[2 * idim + iface] =
                    reader.Get("Boundary Condition", std::string("BC") + dirs[idim] + faces[iface], dir);
            if (out[2 * idim + iface].empty()) {
                throw std::runtime_error(std::string("boundary condition not fully defined for dimension ") + dirs[idim]);
            }
        }
    }
    return out;
}

hcl_config make_config(INIReader const& reader, Param const& param, int ndim, int geometry, int gravity,
                       int precision, int device)
{
    hcl_config c;
    hcl_config_default(&c);
    c.ndim = ndim;
    for (int d = 0; d < 3; ++d) {
        c.nx[d] = d < ndim ? param.Nx_glob_ng[d] : 1;
    }
    c.nghost = param.Ng;
    c.nfx = param.nfx;
    c.geometry = geometry;
    c.gamma = param.gamma;
    c.mmw = param.mu;
    c.limiter = limiter_id(param.reconstruction_type);
    c.riemann = riemann_id(param.riemann_solver);
    const auto bcs = resolve_boundaries(reader, param, ndim);
    for (int f = 0; f < 6; ++f) {
        c.bc[f] = bc_id(bcs[f]);
    }
    c.gravity = gravity;
    c.g[0] = param.gx0;
    c.g[1] = param.gx1;
    c.g[2] = param.gx2;
    c.central_mass = param.M;
    c.xmin[0] = param.x0min;
    c.xmax[0] = param.x0max;
    c.xmin[1] = param.x1min;
    c.xmax[1] = param.x1max;
    c.xmin[2] = param.x2min;
    c.xmax[2] = param.x2max;
    c.precision = precision;
    c.device = device;
    c.pressure_fix = param.pressure_fix == "On" ? 1 : 0; // main.cpp:459
    c.eps_pf = param.eps_pf;
    if (param.grid_type != "Regular") {
        throw std::runtime_error("Unknown grid type: " + param.grid_type + " (UserDefined grids go through hcl_config::nodes).");
    }
    return c;
}

} // namespace hcl::host
