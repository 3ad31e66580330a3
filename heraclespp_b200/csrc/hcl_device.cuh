// hcl_device.cuh -- parameter blocks shared by every kernel of the library.
//
// The grid is one domain with Nghost ghost layers on active dimensions; every
// array follows the reference's Kokkos::LayoutLeft views (i fastest, trailing
// component indices slowest).  See include/heracles_b200.h for the maps.
#pragma once

#include <cstdint>

namespace hcl {

// SI constants of units/units.hpp:176-179 (Joule, Kelvin, kg are 1.0 there).
constexpr double kKb = 1.380649E-23;
constexpr double kMp = 1.672649E-27;
constexpr double kG = 6.6743015E-11;
constexpr double kPi = 3.141592653589793238462643383279502884;
// radiation constant, units.hpp:69-74 (Joule, m, K are 1 there)
constexpr double kAr = (8 * (kPi * kPi * kPi * kPi * kPi) * (kKb * kKb * kKb * kKb)) /
                       (15 * (6.62607015E-34 * 6.62607015E-34 * 6.62607015E-34) *
                        ((2.99792458E8 * 2.99792458E8) * 2.99792458E8));

enum : int { LIM_CONSTANT = 0, LIM_VANLEER = 1, LIM_MINMOD = 2, LIM_VANALBADA = 3 };
enum : int { RS_HLL = 0, RS_HLLC = 1, RS_SPLITTING = 2 };
enum : int { BC_NULLGRADIENT = 0, BC_PERIODIC = 1, BC_REFLEXIVE = 2 };
enum : int { GEOM_CARTESIAN = 0, GEOM_SPHERICAL = 1 };
enum : int { GRAV_UNIFORM = 0, GRAV_POINT_MASS = 1, GRAV_INTERNAL_MASS = 2 };
// EOS_PERFECT_GAS_FAST: the perfect gas in the fast-FP64 kernels (P = (gamma-1) e
// without the temperature round trip, one reciprocal per state); a compile-time
// kind of the fused kernels only, never a configured EOS.
enum : int { EOS_PERFECT_GAS = 0, EOS_RAD_GAS = 1, EOS_PERFECT_GAS_FAST = 2 };

// Everything a kernel needs to know about the grid and the physics plugins.
// Passed by value (it lives in the kernel parameter space).
struct GridDev {
    int ndim;
    int ng;
    int nfx;
    int n[3];       // cells with ghosts (Nx_local_wg)
    int nx[3];      // interior cells (Nx_glob_ng)
    int64_t N;      // n0*n1*n2
    int geom;
    int limiter;
    int riemann;
    int bc[6];
    int gravity;
    double g[3];
    double gamma, gamma_m1, mmw;
    int eos;              // EOS_PERFECT_GAS or EOS_RAD_GAS
    int pressure_fix;     // [Pressure fix] On (the FP64 fused step applies it)
    double eps_pf;
    // grid arrays (device)
    const double* x[3];   // nodes (n+1)
    const double* dx[3];  // n
    const double* xc[3];  // n
    const double* ds;     // N*3
    const double* dv;     // N
    const double* g_r;    // point-mass / internal-mass g(i), n[0]
    // geometry helpers precomputed on the host for spherical runs (per index):
    const double* cot_mid1;   // cos((x1_j+x1_{j+1})/2)/sin(...) per j, source_terms.hpp:38
    const double* sin1;       // sin(x1_j) per node j, source_terms.hpp:58-59
    const double* sin_xc1;    // sin(x1c_j) per j, time_step.hpp:67
    int uniform_cart;         // 1 when Cartesian with uniform dx per dim (to 1e-12)
    int uniform_dx;           // 1 when dx is uniform per dim (to 1e-12), any geometry
    double inv_dx[3];         // 1/dx per dim when uniform_dx
    float inv_dx_f[3];        // the same rounded to FP32 (CFL of the mixed march kernels)
    float cfl_kc2;            // gamma (gamma - 1) / 2 in FP32 (same use)
};

__host__ __device__ inline int64_t lidx(const GridDev& g, int i, int j, int k)
{
    return (int64_t)i + (int64_t)g.n[0] * ((int64_t)j + (int64_t)g.n[1] * (int64_t)k);
}

// Gravity functor value g(i,j,k,dir) (gravity/gravity.hpp:36-40, :63-70).
__device__ inline double gravity_at(const GridDev& g, int i, int dir)
{
    if (g.gravity != GRAV_UNIFORM) { // point mass, internal mass: the radial table
        return dir == 0 ? g.g_r[i] : 0.0;
    }
    return g.g[dir];
}

// Range::with_ghosts(ng_eff) bounds (mesh/range.cpp:388-403).
__host__ __device__ inline void cell_range(const GridDev& g, int ng_eff, int b[3], int e[3])
{
    for (int d = 0; d < 3; ++d) {
        if (d < g.ndim) {
            b[d] = g.ng - ng_eff;
            e[d] = g.ng + g.nx[d] + ng_eff;
        } else {
            b[d] = 0;
            e[d] = 1;
        }
    }
}

// Source index of a cell along one dimension after the boundary fill of
// boundary_distribute.hpp:42-76 on one rank (periodic self-exchange of
// ghost_sync, then NullGradient / Reflexive overwrites, boundary.cpp:221-296).
// Composing the per-dimension maps gives exactly the reference's result for
// every ghost cell, corners included, independently of the face order.
// Returns the source index; *flip is set when the momentum component of this
// dimension changes sign (Reflexive).
__host__ __device__ inline int bc_source(int l, int n, int ng, int bc_left, int bc_right, int* flip)
{
    *flip = 0;
    if (l >= ng && l < n - ng) {
        return l;
    }
    const int nxi = n - 2 * ng;
    if (l < ng) {
        if (bc_left == BC_PERIODIC) {
            return l + nxi;
        }
        if (bc_left == BC_NULLGRADIENT) {
            return ng;
        }
        *flip = 1;
        return 2 * ng - 1 - l;
    }
    if (bc_right == BC_PERIODIC) {
        return l - nxi;
    }
    if (bc_right == BC_NULLGRADIENT) {
        return n - ng - 1;
    }
    *flip = 1;
    return 2 * (n - ng) - 1 - l;
}

// Control block of the device-resident time loop (main.cpp:354-531).  Slots
// are indexed by the step's position in a graph chunk so that no block of a
// step reads a value another block of the same step writes.
struct StepCtl {
    unsigned long long inv_dt_bits[3]; // atomicMax slots of 1/dt (non-negative doubles)
    double t[2];                       // time before step s: t[s % 2]
    int iter[2];                       // iterations done before step s
    int time_output_id[2];             // main.cpp:208
    int iter_output_id[2];             // main.cpp:209
    int stop[2];                       // set once the loop must exit (main.cpp:380,384)
    int errflag[2];                    // set by any CTA that meets an invalid state
    int final_buf;                     // state buffer holding the last state when stopped
    int err;                           // HCL_ERR_INVALID_STATE / HCL_ERR_NEGATIVE_DT
    unsigned long long bad_cell;       // first bad cell (atomicMin), ~0 when none
    double last_dt;
    int pad;
};

struct RunParamsDev {
    double cfl, t_end;
    int max_iter;
    int iter_frequency;
    double time_frequency, time_first_output;
    int fixed_dt;      // 0: CFL dt, 1: dts[iter], 2: dt_value
    double dt_value;
    const double* dts; // device, indexed by absolute iteration
    double* dt_log;    // optional device log of dt per absolute iteration
    int dt_log_cap;
};

// Ordered-key encoding so that atomicMax on unsigned 64-bit integers orders
// non-negative doubles correctly.
__device__ inline unsigned long long dbl_bits(double v)
{
    return (unsigned long long)__double_as_longlong(v);
}

} // namespace hcl
