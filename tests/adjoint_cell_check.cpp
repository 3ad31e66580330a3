// Test helper: extern "C" wrappers over heraclespp_b200/csrc/adjoint_cell.cuh
// compiled as plain host C++ (tests/test_adjoint_cpu.py builds it with g++ and
// checks each reverse-mode function against central finite differences).
#include "adjoint_cell.cuh"

using namespace hcl::adj;

namespace {
Eos<double> eos_of(double gamma)
{
    return Eos<double>{gamma, gamma - 1, 1.0 / (gamma - 1)};
}

template <int ND>
void riemann_fwd_nd(int solver, double gamma, const double* UL, const double* UR, int l, double* F)
{
    riemann<ND>(eos_of(gamma), solver, UL, UR, l, F);
}

template <int ND>
void riemann_rev_nd(int solver, double gamma, const double* UL, const double* UR, int l, const double* Fb, double* ULb,
                    double* URb)
{
    riemann_rev<ND>(eos_of(gamma), solver, UL, UR, l, Fb, ULb, URb);
}
SphGeo<double> geo_of(const double* g)
{
    return SphGeo<double>{g[0], g[1], g[2], g[3], g[4], g[5]};
}
} // namespace

extern "C" {

// geo = {k, dS, dS_p, rf, cot, sf}
void t_sph_src(int nd, int d, const double* geo, const double* WL, const double* WR, double* S)
{
    if (nd == 1) {
        sph_source<1>(geo_of(geo), d, WL, WR, S);
    } else if (nd == 2) {
        sph_source<2>(geo_of(geo), d, WL, WR, S);
    } else {
        sph_source<3>(geo_of(geo), d, WL, WR, S);
    }
}

void t_sph_src_rev(int nd, int d, const double* geo, const double* WL, const double* WR, const double* Sb, double* WLb,
                   double* WRb)
{
    if (nd == 1) {
        sph_source_rev<1>(geo_of(geo), d, WL, WR, Sb, WLb, WRb);
    } else if (nd == 2) {
        sph_source_rev<2>(geo_of(geo), d, WL, WR, Sb, WLb, WRb);
    } else {
        sph_source_rev<3>(geo_of(geo), d, WL, WR, Sb, WLb, WRb);
    }
}

void t_riemann_fwd(int nd, int solver, double gamma, const double* UL, const double* UR, int l, double* F)
{
    if (nd == 1) {
        riemann_fwd_nd<1>(solver, gamma, UL, UR, l, F);
    } else if (nd == 2) {
        riemann_fwd_nd<2>(solver, gamma, UL, UR, l, F);
    } else {
        riemann_fwd_nd<3>(solver, gamma, UL, UR, l, F);
    }
}

void t_riemann_rev(int nd, int solver, double gamma, const double* UL, const double* UR, int l, const double* Fb,
                   double* ULb, double* URb)
{
    if (nd == 1) {
        riemann_rev_nd<1>(solver, gamma, UL, UR, l, Fb, ULb, URb);
    } else if (nd == 2) {
        riemann_rev_nd<2>(solver, gamma, UL, UR, l, Fb, ULb, URb);
    } else {
        riemann_rev_nd<3>(solver, gamma, UL, UR, l, Fb, ULb, URb);
    }
}

void t_flux_fwd(double gamma, const double* W, int l, double* F)
{
    flux_prim<2>(eos_of(gamma), W, l, F);
}

void t_flux_rev(double gamma, const double* W, int l, const double* Fb, double* Wb)
{
    flux_prim_rev<2>(eos_of(gamma), W, l, Fb, Wb);
}

void t_p2c_fwd(double gamma, const double* W, double* U)
{
    cons_from_prim<2>(eos_of(gamma), W, U);
}

void t_p2c_rev(double gamma, const double* W, const double* Ub, double* Wb)
{
    cons_from_prim_rev<2>(eos_of(gamma), W, Ub, Wb);
}

void t_c2p_fwd(double gamma, const double* U, double* W)
{
    prim_from_cons<2>(eos_of(gamma), U, W);
}

void t_c2p_rev(double gamma, const double* U, const double* Wb, double* Ub)
{
    prim_from_cons_rev<2>(eos_of(gamma), U, Wb, Ub);
}

double t_limiter(int lim, double R, double L, double* gR, double* gL)
{
    return limiter<double>(lim, R, L, gR, gL);
}

double t_limiter_on(int lim, int active, double R, double L, double* gR, double* gL)
{
    return limiter_on<double>(lim, active != 0, R, L, gR, gL);
}

} // extern "C"
