// ref_cell_wrap.cpp -- extern "C" entry points over the reference's OWN
// per-cell physics headers, compiled from where they lie in the reference
// tree (hydro/euler_equations.hpp, hydro/riemann_solver.hpp,
// hydro/slope_limiters.hpp, hydro/source_terms.hpp,
// thermodynamics/perfect_gas.hpp + perfect_gas.cpp,
// thermodynamics/rad_gas.hpp + rad_gas.cpp).
//
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/Makefile and
// used by tests to check the C restatement in hcl_oracle.c bit for bit.
// State vectors are [rho, v_0..v_{ndim-1}, E or P].
#include <stdexcept>

#include <euler_equations.hpp>
#include <perfect_gas.hpp>
#include <rad_gas.hpp>
#include <riemann_solver.hpp>
#include <slope_limiters.hpp>
#include <source_terms.hpp>

namespace {

using hclpp::EulerCons;
using hclpp::EulerFlux;
using hclpp::EulerPrim;
using hclpp::ndim;
using hclpp::thermodynamics::PerfectGas;
using hclpp::thermodynamics::RadGas;

EulerCons load_cons(double const* v)
{
    EulerCons c;
    c.rho = v[0];
    for (int d = 0; d < ndim; ++d) {
        c.rhou[d] = v[1 + d];
    }
    c.E = v[1 + ndim];
    return c;
}

EulerPrim load_prim(double const* v)
{
    EulerPrim p;
    p.rho = v[0];
    for (int d = 0; d < ndim; ++d) {
        p.u[d] = v[1 + d];
    }
    p.P = v[1 + ndim];
    return p;
}

template <class S>
void store(S const& s, double* v)
{
    v[0] = s.rho;
    for (int d = 0; d < ndim; ++d) {
        if constexpr (requires { s.rhou; }) {
            v[1 + d] = s.rhou[d];
        } else {
            v[1 + d] = s.u[d];
        }
    }
    if constexpr (requires { s.E; }) {
        v[1 + ndim] = s.E;
    } else {
        v[1 + ndim] = s.P;
    }
}

} // namespace

namespace {

template <class Eos>
void riemann_with(int solver, Eos const& eos, double const* consL, double const* consR, int locdim, double* flux)
{
    EulerCons const L = load_cons(consL);
    EulerCons const R = load_cons(consR);
    EulerFlux f;
    if (solver == 0) {
        f = hclpp::HLL()(L, R, locdim, eos);
    } else if (solver == 1) {
        f = hclpp::HLLC()(L, R, locdim, eos);
    } else {
        f = hclpp::Splitting()(L, R, locdim, eos);
    }
    flux[0] = f.rho;
    for (int d = 0; d < ndim; ++d) {
        flux[1 + d] = f.rhou[d];
    }
    flux[1 + ndim] = f.E;
}

} // namespace

extern "C" {

int ref_ndim()
{
    return ndim;
}

// 0 = valid, 1 = std::domain_error from the PerfectGas constructor
int ref_perfect_gas_check(double gamma, double mmw)
{
    try {
        PerfectGas const eos(gamma, mmw);
        (void)eos;
    } catch (std::domain_error const&) {
        return 1;
    }
    return 0;
}

int ref_eos_valid(double rho, double P)
{
    return PerfectGas::is_valid(rho, P) ? 1 : 0;
}

double ref_evol_from_pres(double gamma, double mmw, double rho, double P)
{
    return PerfectGas(gamma, mmw).compute_evol_from_pres(rho, P);
}

double ref_pres_from_evol(double gamma, double mmw, double rho, double evol)
{
    return PerfectGas(gamma, mmw).compute_pres_from_evol(rho, evol);
}

double ref_speed_of_sound(double gamma, double mmw, double rho, double P)
{
    return PerfectGas(gamma, mmw).compute_speed_of_sound(rho, P);
}

void ref_to_prim(double gamma, double mmw, double const* cons, double* prim)
{
    store(hclpp::to_prim(load_cons(cons), PerfectGas(gamma, mmw)), prim);
}

void ref_to_cons(double gamma, double mmw, double const* prim, double* cons)
{
    store(hclpp::to_cons(load_prim(prim), PerfectGas(gamma, mmw)), cons);
}

void ref_flux_from_prim(double gamma, double mmw, double const* prim, int locdim, double* flux)
{
    EulerFlux const f = hclpp::compute_flux(load_prim(prim), locdim, PerfectGas(gamma, mmw));
    flux[0] = f.rho;
    for (int d = 0; d < ndim; ++d) {
        flux[1 + d] = f.rhou[d];
    }
    flux[1 + ndim] = f.E;
}

void ref_flux_from_cons(double gamma, double mmw, double const* cons, int locdim, double* flux)
{
    EulerFlux const f = hclpp::compute_flux(load_cons(cons), locdim, PerfectGas(gamma, mmw));
    flux[0] = f.rho;
    for (int d = 0; d < ndim; ++d) {
        flux[1 + d] = f.rhou[d];
    }
    flux[1 + ndim] = f.E;
}

double ref_ek_prim(double const* prim)
{
    return hclpp::compute_ek(load_prim(prim));
}

double ref_ek_cons(double const* cons)
{
    return hclpp::compute_ek(load_cons(cons));
}

// 0 = valid, 1 = std::domain_error from the RadGas constructor
int ref_rad_gas_check(double gamma, double mmw)
{
    try {
        RadGas const eos(gamma, mmw);
        (void)eos;
    } catch (std::domain_error const&) {
        return 1;
    }
    return 0;
}

double ref_rad_evol_from_pres(double gamma, double mmw, double rho, double P)
{
    return RadGas(gamma, mmw).compute_evol_from_pres(rho, P);
}

double ref_rad_pres_from_evol(double gamma, double mmw, double rho, double evol)
{
    return RadGas(gamma, mmw).compute_pres_from_evol(rho, evol);
}

double ref_rad_speed_of_sound(double gamma, double mmw, double rho, double P)
{
    return RadGas(gamma, mmw).compute_speed_of_sound(rho, P);
}

double ref_rad_temp_from_pres(double gamma, double mmw, double rho, double P)
{
    return RadGas(gamma, mmw).compute_temp_from_pres(rho, P);
}

// the Riemann solvers with the RadGas EOS
void ref_rad_riemann(int solver, double gamma, double mmw, double const* consL, double const* consR, int locdim,
                     double* flux)
{
    riemann_with(solver, RadGas(gamma, mmw), consL, consR, locdim, flux);
}

// solver: 0 HLL, 1 HLLC, 2 Splitting ("Low Mach")
void ref_riemann(int solver, double gamma, double mmw, double const* consL, double const* consR, int locdim, double* flux)
{
    PerfectGas const eos(gamma, mmw);
    EulerCons const L = load_cons(consL);
    EulerCons const R = load_cons(consR);
    EulerFlux f;
    if (solver == 0) {
        f = hclpp::HLL()(L, R, locdim, eos);
    } else if (solver == 1) {
        f = hclpp::HLLC()(L, R, locdim, eos);
    } else {
        f = hclpp::Splitting()(L, R, locdim, eos);
    }
    flux[0] = f.rho;
    for (int d = 0; d < ndim; ++d) {
        flux[1 + d] = f.rhou[d];
    }
    flux[1 + ndim] = f.E;
}

// limiter: 0 Constant, 1 VanLeer, 2 Minmod, 3 VanAlbada
double ref_slope(int limiter, double diffR, double diffL)
{
    switch (limiter) {
    case 0:
        return hclpp::Constant()(diffR, diffL);
    case 1:
        return hclpp::VanLeer()(diffR, diffL);
    case 2:
        return hclpp::Minmod()(diffR, diffL);
    default:
        return hclpp::VanAlbada()(diffR, diffL);
    }
}

double ref_source_grad_pres(double dtodv, double PL, double PR, double dS, double dS_p)
{
    return hclpp::source_grad_pres(dtodv, PL, PR, dS, dS_p);
}

double ref_source_grad_u_r(double dtodv, double rhoL, double rhoR, double uL, double uR, double dS, double dS_p)
{
    return hclpp::source_grad_u_r(dtodv, rhoL, rhoR, uL, uR, dS, dS_p);
}

double ref_source_grad_u_idir_r(double dtodv, double x0, double x0_p, double rhoL, double rhoR, double uL_r, double uR_r,
                                double uL_o, double uR_o, double dS, double dS_p)
{
    return hclpp::source_grad_u_idir_r(dtodv, x0, x0_p, rhoL, rhoR, uL_r, uR_r, uL_o, uR_o, dS, dS_p);
}

double ref_source_grad_u_th(double dtodv, double x1, double x1_p, double rhoL, double rhoR, double uL, double uR, double dS,
                            double dS_p)
{
    return hclpp::source_grad_u_th(dtodv, x1, x1_p, rhoL, rhoR, uL, uR, dS, dS_p);
}

double ref_source_grad_u_phi(double dtodv, double x1, double x1_p, double rhoL, double rhoR, double uL_th, double uR_th,
                             double uL_phi, double uR_phi, double dS, double dS_p)
{
    return hclpp::source_grad_u_phi(dtodv, x1, x1_p, rhoL, rhoR, uL_th, uR_th, uL_phi, uR_phi, dS, dS_p);
}

} // extern "C"
