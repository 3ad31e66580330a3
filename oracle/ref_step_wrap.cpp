// TEST INFRASTRUCTURE (oracle): a C-ABI wrapper around the reference's own
// array code for the MUSCL-Hancock step, compiled from the reference sources
// where they lie (oracle/Makefile, target ref-step) against the host Kokkos
// and single-rank MPI stand-ins of oracle/ref_array.  The product never links
// it.  It serves two purposes:
//  * the stage functions below run the reference's classes on caller arrays
//    (LayoutLeft, the reference's View extents), so that tests can check
//    oracle/hcl_oracle.c's array-level restatement against them;
//  * rs_run drives those classes in the order of the reference's time loop
//    (src/main.cpp:354-531, without the outputs), on the host cores through
//    the stand-in's OpenMP loops: the reference's FP64 CPU path, timed as the
//    benchmark's CPU baseline.
//
// NDIM and the geometry are compile-time choices of the reference
// (Heraclespp_NDIM, Heraclespp_GEOM); one shared object is built per pair.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>
#include <unistd.h>

#include <Kokkos_Core.hpp>

#include "array_conversion.hpp"
#include "boundary.hpp"
#include "boundary_distribute.hpp"
#include "boundary_factory.hpp"
#include "extrapolation_reconstruction.hpp"
#include "face_reconstruction.hpp"
#include "godunov_scheme.hpp"
#include "gravity.hpp"
#include "grid.hpp"
#include "grid_type.hpp"
#include "hydro_reconstruction.hpp"
#include "internal_energy.hpp"
#include "param.hpp"
#include "perfect_gas.hpp"
#include "pressure_fix.hpp"
#include "time_step.hpp"

using namespace hclpp;

extern "C" {
// configuration of one wrapped domain (strings are the reference's factory keys)
struct rs_config {
    int nx[3];
    int ng;
    int nfx;
    double xmin[3], xmax[3];
    double gamma, mmw;
    const char* limiter;
    const char* riemann;
    const char* bc[6];
    const char* bc_priority; // "" for the default order
    int gravity;             // 0 uniform, 1 point mass
    double g[3];
    double central_mass;
};
}

namespace {

using EOS = thermodynamics::PerfectGas;

template <class Gravity>
struct Ops {
    Gravity g;
    std::array<std::unique_ptr<IBoundaryCondition<Gravity>>, nfaces> bcs_array;
    std::unique_ptr<DistributedBoundaryCondition> bcs;
    std::unique_ptr<IHydroReconstruction<Gravity>> reconstruction;
    std::unique_ptr<IGodunovScheme<Gravity>> godunov;
    KV_double_6d u_rec;
    KV_double_5d P_rec;
};

struct RefStep {
    std::unique_ptr<Param> param;
    std::unique_ptr<Grid> grid;
    EOS eos{1.4, 1.0};
    int gravity = 0;
    std::unique_ptr<Ops<UniformGravity>> uni;
    std::unique_ptr<Ops<PointMassGravity>> pm;
    int n[3] = {1, 1, 1};
    int nfx = 0;
};

std::string ini_text(const rs_config& c)
{
    char buf[4096];
    std::snprintf(buf, sizeof(buf),
                  "[Grid]\nNx0_glob = %d\nNx1_glob = %d\nNx2_glob = %d\nNghost = %d\ntype = Regular\n"
                  "x0min = %.17g\nx0max = %.17g\nx1min = %.17g\nx1max = %.17g\nx2min = %.17g\nx2max = %.17g\n"
                  "[Hydro]\nreconstruction = %s\nriemann_solver = %s\n"
                  "[Perfect Gas]\ngamma = %.17g\nmu = %.17g\n"
                  "[Gravity]\ngx0 = %.17g\ngx1 = %.17g\ngx2 = %.17g\nM = %.17g\n"
                  "[Passive Scalar]\nnfx = %d\n"
                  "[Boundary Condition]\npriority = %s\n",
                  c.nx[0], c.nx[1], c.nx[2], c.ng, c.xmin[0], c.xmax[0], c.xmin[1], c.xmax[1], c.xmin[2], c.xmax[2],
                  c.limiter, c.riemann, c.gamma, c.mmw, c.g[0], c.g[1], c.g[2], c.central_mass, c.nfx,
                  c.bc_priority ? c.bc_priority : "");
    return buf;
}

template <class Gravity>
std::unique_ptr<Ops<Gravity>> make_ops(RefStep& s, const rs_config& c, Gravity g)
{
    auto ops = std::make_unique<Ops<Gravity>>(Ops<Gravity>{std::move(g), {}, nullptr, nullptr, nullptr, {}, {}});
    for (int idim = 0; idim < ndim; ++idim) {
        for (int iface = 0; iface < 2; ++iface) {
            ops->bcs_array[(idim * 2) + iface] = factory_boundary_construction<Gravity>(c.bc[(idim * 2) + iface], idim,
                                                                                       iface);
        }
    }
    ops->bcs = std::make_unique<DistributedBoundaryCondition>(*s.grid, *s.param);
    const auto& w = s.grid->Nx_local_wg;
    ops->u_rec = KV_double_6d("u_rec", w[0], w[1], w[2], 2, ndim, ndim);
    ops->P_rec = KV_double_5d("P_rec", w[0], w[1], w[2], 2, ndim);
    ops->reconstruction = std::make_unique<MUSCLHancockHydroReconstruction<EOS, Gravity>>(
        factory_face_reconstruction(c.limiter), std::make_unique<HancockExtrapolationReconstruction<EOS, Gravity>>(s.eos),
        s.eos, ops->P_rec, ops->u_rec);
    ops->godunov = factory_godunov_scheme<EOS, Gravity>(c.riemann, s.eos);
    return ops;
}

// unmanaged views of the caller's LayoutLeft arrays
struct Arrays {
    KV_double_3d rho, E, P, rho_new, E_new;
    KV_double_4d rhou, u, fx, rhou_new, fx_new;
    KV_double_5d rho_rec, E_rec;
    KV_double_6d rhou_rec, fx_rec;
};

KV_double_3d v3(const RefStep& s, const double* p)
{
    return KV_double_3d(const_cast<double*>(p), s.n[0], s.n[1], s.n[2]);
}
KV_double_4d v4(const RefStep& s, const double* p, int c)
{
    return KV_double_4d(const_cast<double*>(p), s.n[0], s.n[1], s.n[2], c);
}
KV_double_5d v5(const RefStep& s, const double* p)
{
    return KV_double_5d(const_cast<double*>(p), s.n[0], s.n[1], s.n[2], 2, ndim);
}
KV_double_6d v6(const RefStep& s, const double* p, int c)
{
    return KV_double_6d(const_cast<double*>(p), s.n[0], s.n[1], s.n[2], 2, ndim, c);
}

// calls f(ops) with the gravity the domain was created with
template <class F>
auto with_ops(RefStep& s, F&& f)
{
    if (s.gravity == 1) {
        return f(*s.pm);
    }
    return f(*s.uni);
}

} // namespace

extern "C" {

void* rs_create(const rs_config* c)
{
    try {
        auto s = std::make_unique<RefStep>();
        char path[] = "/tmp/hcl_ref_stepXXXXXX";
        const int fd = mkstemp(path);
        if (fd < 0) {
            return nullptr;
        }
        const std::string text = ini_text(*c);
        if (write(fd, text.data(), text.size()) != (ssize_t)text.size()) {
            close(fd);
            unlink(path);
            return nullptr;
        }
        close(fd);
        INIReader reader(path);
        unlink(path);
        s->param = std::make_unique<Param>(reader);
        s->eos = EOS(s->param->gamma, s->param->mu);
        s->grid = std::make_unique<Grid>(s->param->Nx_glob_ng, s->param->mpi_dims_cart, s->param->Ng);
        for (int d = 0; d < 3; ++d) {
            s->n[d] = s->grid->Nx_local_wg[d];
        }
        s->nfx = c->nfx;
        // Grid::set_grid from the Regular grid type (main.cpp:263-266)
        KV_double_1d x0("x0_glob", s->grid->Nx_glob_ng[0] + (2 * s->grid->Nghost[0]) + 1);
        KV_double_1d x1("x1_glob", s->grid->Nx_glob_ng[1] + (2 * s->grid->Nghost[1]) + 1);
        KV_double_1d x2("x2_glob", s->grid->Nx_glob_ng[2] + (2 * s->grid->Nghost[2]) + 1);
        Regular(*s->param).execute(s->grid->Nghost, s->grid->Nx_glob_ng, x0, x1, x2);
        s->grid->set_grid(x0, x1, x2);
        s->gravity = c->gravity;
        if (c->gravity == 1) {
            s->pm = make_ops(*s, *c, make_point_mass_gravity(s->param->M, *s->grid));
        } else {
            s->uni = make_ops(*s, *c, make_uniform_gravity(s->param->gx0, s->param->gx1, s->param->gx2));
        }
        return s.release();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "rs_create: %s\n", e.what());
        return nullptr;
    }
}

void rs_destroy(void* h)
{
    delete static_cast<RefStep*>(h);
}

void rs_set_threads(int n)
{
    if (n > 0) {
        omp_set_num_threads(n);
    }
}

int rs_get_threads(void)
{
    return omp_get_max_threads();
}

// grid arrays: cell sizes and centres per dimension (n_d each), ds (N x 3), dv (N)
void rs_grid(void* h, double* dx, double* xc, double* ds, double* dv)
{
    auto& s = *static_cast<RefStep*>(h);
    const Grid& g = *s.grid;
    const KV_double_1d dxs[3] = {g.dx0, g.dx1, g.dx2};
    const KV_double_1d xcs[3] = {g.x0_center, g.x1_center, g.x2_center};
    int off = 0;
    for (int d = 0; d < 3; ++d) {
        for (int i = 0; i < s.n[d]; ++i) {
            dx[off + i] = dxs[d](i);
            xc[off + i] = xcs[d](i);
        }
        off += s.n[d];
    }
    Kokkos::deep_copy(KV_double_4d(ds, s.n[0], s.n[1], s.n[2], 3), g.ds);
    Kokkos::deep_copy(KV_double_3d(dv, s.n[0], s.n[1], s.n[2]), g.dv);
}

// conv_prim_to_cons (array_conversion.hpp:32-104)
void rs_conv_prim_to_cons(void* h, int ng_eff, const double* rho, const double* u, const double* P, double* rhou,
                          double* E)
{
    auto& s = *static_cast<RefStep*>(h);
    conv_prim_to_cons(s.grid->range.with_ghosts(ng_eff), s.eos, v3(s, rho), v4(s, u, ndim), v3(s, P), v4(s, rhou, ndim),
                      v3(s, E));
}

// conv_cons_to_prim (array_conversion.hpp:106-172)
void rs_conv_cons_to_prim(void* h, int ng_eff, const double* rho, const double* rhou, const double* E, double* u,
                          double* P)
{
    auto& s = *static_cast<RefStep*>(h);
    conv_cons_to_prim(s.grid->range.with_ghosts(ng_eff), s.eos, v3(s, rho), v4(s, rhou, ndim), v3(s, E),
                      v4(s, u, ndim), v3(s, P));
}

// MUSCLHancockHydroReconstruction::execute (hydro_reconstruction.hpp:85-129)
void rs_hydro_reconstruction(void* h, int ng_eff, double dt, const double* rho, const double* u, const double* P,
                             const double* fx, double* rho_rec, double* rhou_rec, double* E_rec, double* fx_rec)
{
    auto& s = *static_cast<RefStep*>(h);
    with_ops(s, [&](auto& ops) {
        ops.reconstruction->execute(s.grid->range.with_ghosts(ng_eff), *s.grid, ops.g, dt, v3(s, rho), v4(s, u, ndim),
                                    v3(s, P), v4(s, fx, s.nfx), v5(s, rho_rec), v6(s, rhou_rec, ndim), v5(s, E_rec),
                                    v6(s, fx_rec, s.nfx));
        return 0;
    });
}

// IGodunovScheme::execute (godunov_scheme.hpp:77-302)
void rs_godunov(void* h, int ng_eff, double dt, const double* rho, const double* rhou, const double* E, const double* fx,
                const double* rho_rec, const double* rhou_rec, const double* E_rec, const double* fx_rec,
                double* rho_new, double* rhou_new, double* E_new, double* fx_new)
{
    auto& s = *static_cast<RefStep*>(h);
    with_ops(s, [&](auto& ops) {
        ops.godunov->execute(s.grid->range.with_ghosts(ng_eff), *s.grid, ops.g, dt, v3(s, rho), v4(s, rhou, ndim),
                             v3(s, E), v4(s, fx, s.nfx), v5(s, rho_rec), v6(s, rhou_rec, ndim), v5(s, E_rec),
                             v6(s, fx_rec, s.nfx), v3(s, rho_new), v4(s, rhou_new, ndim), v3(s, E_new),
                             v4(s, fx_new, s.nfx));
        return 0;
    });
}

// DistributedBoundaryCondition::operator() on one rank (boundary_distribute.hpp:42-76)
void rs_boundaries(void* h, double* rho, double* rhou, double* E, double* fx)
{
    auto& s = *static_cast<RefStep*>(h);
    with_ops(s, [&](auto& ops) {
        (*ops.bcs)(ops.bcs_array, *s.grid, ops.g, v3(s, rho), v4(s, rhou, ndim), v3(s, E), v4(s, fx, s.nfx));
        return 0;
    });
}

// time_step (time_step.hpp:35-82): the largest admissible dt at CFL 1
double rs_time_step(void* h, int ng_eff, const double* rho, const double* u, const double* P)
{
    auto& s = *static_cast<RefStep*>(h);
    return time_step(s.grid->range.with_ghosts(ng_eff), s.eos, *s.grid, v3(s, rho), v4(s, u, ndim), v3(s, P));
}

// minimum_internal_energy (internal_energy.cpp:20-45) over no_ghosts
double rs_min_internal_energy(void* h, const double* rho, const double* rhou, const double* E)
{
    auto& s = *static_cast<RefStep*>(h);
    return minimum_internal_energy(s.grid->range.no_ghosts(), *s.grid, v3(s, rho), v4(s, rhou, ndim), v3(s, E));
}

// The time loop of main.cpp:354-531 from the conservative state (ghosts
// filled), without outputs or grid shifts: dt from the CFL condition (clamped
// to t_end), the internal-energy check, reconstruction at dt/2, the Godunov
// update, the boundaries, the copy into the state and cons -> prim.  Steps
// until t_end or max_iter.  Returns 0, or 4 when the internal-energy check
// fails (the state is left as it was before that step).  dts (optional)
// receives each step's dt.
int rs_run(void* h, double* rho, double* rhou, double* E, double* fx, double cfl, double t_end, int max_iter,
           double* t_out, int* iter_out, double* dts)
{
    auto& s = *static_cast<RefStep*>(h);
    const int n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
    KV_double_3d rho_v = v3(s, rho), E_v = v3(s, E);
    KV_double_4d rhou_v = v4(s, rhou, ndim), fx_v = v4(s, fx, s.nfx);
    KV_double_4d u("u", n0, n1, n2, ndim);
    KV_double_3d P("P", n0, n1, n2);
    KV_double_5d rho_rec("rho_rec", n0, n1, n2, 2, ndim);
    KV_double_6d rhou_rec("rhou_rec", n0, n1, n2, 2, ndim, ndim);
    KV_double_5d E_rec("E_rec", n0, n1, n2, 2, ndim);
    KV_double_6d fx_rec("fx_rec", n0, n1, n2, 2, ndim, s.nfx);
    KV_double_3d rho_new("rho_new", n0, n1, n2);
    KV_double_4d rhou_new("rhou_new", n0, n1, n2, ndim);
    KV_double_3d E_new("E_new", n0, n1, n2);
    KV_double_4d fx_new("fx_new", n0, n1, n2, s.nfx);
    const Grid& grid = *s.grid;
    conv_cons_to_prim(grid.range.all_ghosts(), s.eos, rho_v, rhou_v, E_v, u, P);
    double t = 0;
    int iter = 0;
    int status = 0;
    with_ops(s, [&](auto& ops) {
        bool should_exit = false;
        while (!should_exit) {
            double dt = cfl * time_step(grid.range.all_ghosts(), s.eos, grid, rho_v, u, P);
            if ((t + dt) >= t_end) {
                dt = t_end - t;
                should_exit = true;
            }
            if ((iter + 1) >= max_iter) {
                should_exit = true;
            }
            const double min_evol = minimum_internal_energy(grid.range.no_ghosts(), grid, rho_v, rhou_v, E_v);
            if (std::isnan(min_evol) || min_evol < 0) {
                status = 4;
                return 0;
            }
            ops.reconstruction->execute(grid.range.with_ghosts(1), grid, ops.g, dt / 2, rho_v, u, P, fx_v, rho_rec,
                                        rhou_rec, E_rec, fx_rec);
            ops.godunov->execute(grid.range.no_ghosts(), grid, ops.g, dt, rho_v, rhou_v, E_v, fx_v, rho_rec, rhou_rec,
                                 E_rec, fx_rec, rho_new, rhou_new, E_new, fx_new);
            (*ops.bcs)(ops.bcs_array, grid, ops.g, rho_new, rhou_new, E_new, fx_new);
            Kokkos::deep_copy(rho_v, rho_new);
            Kokkos::deep_copy(rhou_v, rhou_new);
            Kokkos::deep_copy(E_v, E_new);
            Kokkos::deep_copy(fx_v, fx_new);
            conv_cons_to_prim(grid.range.all_ghosts(), s.eos, rho_new, rhou_new, E_new, u, P);
            if (dts) {
                dts[iter] = dt;
            }
            t += dt;
            ++iter;
        }
        return 0;
    });
    *t_out = t;
    *iter_out = iter;
    return status;
}

} // extern "C"
