// adjoint_step.cuh -- discrete adjoint of one fused MUSCL-Hancock step.
//
// Forward step (Cartesian, uniform spacing; uniform gravity, or the point-mass
// field g(i) along x0, which does not depend on the state):
//   U'_c = U_c + sum_d c_d (F_{c-1/2,d} - F_{c+1/2,d}) + dt g-terms(U_c),
//   F_{f,d} = Riemann(H_{L,d}, H_{R,d}),  H = Hancock face states built from the
//   limited slopes of the primitive stencil of each cell, and ghosts of U' are
//   images of interior cells.  dt is held fixed (recorded by the forward run).
//
// One CTA owns a tile.  It recomputes the forward face states of the tile on
// chip, then runs the reverse sweep: the adjoint of each face it owns (its
// cells' left faces) through the Riemann solver, of the Hancock predictor and
// the limited slopes of every cell it touched, and of the primitive recovery,
// and adds the result for every cell of its halo-extended tile into lam_in
// with atomics (neighbouring tiles overlap by the stencil width).  The
// transpose of the boundary fill is applied as the contributions are made: a
// contribution to a ghost cell goes to the interior cell the ghost is filled
// from.  The gather kernel k_fold_ghosts folds the ghosts of the final
// adjoint the caller supplies.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "adjoint_cell.cuh"
#include "fused_step.cuh"
#include "hcl_device.cuh"
#include "stages.hpp"

namespace hcl::adjoint {

using fused::Shape;
using fused::sidx;
using fused::StateDev;

template <int ND, class R, int TX, int TY, int TZ>
struct AdjShape {
    using S = Shape<ND, TX, TY, TZ>;
    // per passive scalar: its face values on the A arrays ([2][A_d] per d)
    static constexpr int XA = S::A_TOTAL / S::NV;
    __host__ __device__ static constexpr int XAoff(int d) { return S::Aoff(d) / S::NV; }
    // one value per face of the tile (the F_d arrays)
    static constexpr int FS = S::F_TOTAL / S::NV;
    __host__ __device__ static constexpr int FSoff(int d) { return S::Foff(d) / S::NV; }
    static constexpr size_t smem()
    {
        // W, Wb, lam: [NV][NP]; A, Ab: A_TOTAL each
        return sizeof(R) * (2 * (size_t)S::NV * S::NP + 2 * (size_t)S::A_TOTAL) + sizeof(double) * (size_t)S::NV * S::NP;
    }
    // with nfx passive scalars: the density and scalar adjoints of the new
    // state's division ([1 + nfx][TVOL], FP64), the scalar primitives and
    // their adjoints ([nfx][NP] each), the predicted face values and their
    // adjoints ([nfx][XA] each) and the Riemann mass flux of every face [FS]
    static constexpr size_t smem(int nfx)
    {
        return smem() + (nfx > 0 ? sizeof(double) * (size_t)(1 + nfx) * S::TVOL +
                                       sizeof(R) * ((size_t)nfx * (2 * S::NP + 2 * XA) + FS)
                                 : 0);
    }
};

// Primitives of a conservative FP64 state rounded exactly as the forward
// FP64 step rounds them (physics_exact.cuh to_prim for the perfect gas:
// hydro/euler_equations.hpp:41-65, :111-122 with the temperature round trip of
// thermodynamics/perfect_gas.hpp:58-78), written with round-to-nearest
// intrinsics so that no contraction changes them.  The FP64 sweep takes the
// limiters' branches from the differences of these values (phase 4), so that
// at rounding-level ties, which flat and solid-body regions produce, they are
// the branches the forward step took; the Riemann selections it takes on the
// face states it builds from them.  The derivatives are those of
// P = (gamma - 1) e, which equal the round trip's.
template <int ND>
__device__ __forceinline__ void prim_forward_rounding(const GridDev& g, const double* q, double* w)
{
    double norm = __dmul_rn(q[1], q[1]);
#pragma unroll
    for (int d = 1; d < ND; ++d) {
        norm = __dadd_rn(norm, __dmul_rn(q[1 + d], q[1 + d]));
    }
    // halving is exact: x * 0.5 rounds as x / 2 does
    const double ek = __dmul_rn(__ddiv_rn(norm, q[0]), 0.5);
    const double evol = __dsub_rn(q[1 + ND], ek);
    w[0] = q[0];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        w[1 + d] = __ddiv_rn(q[1 + d], q[0]);
    }
    const double T = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(evol, g.mmw), kMp), g.gamma_m1), __dmul_rn(q[0], kKb));
    w[1 + ND] = __ddiv_rn(__dmul_rn(__dmul_rn(q[0], kKb), T), __dmul_rn(g.mmw, kMp));
}

// Round-to-nearest FP64 operations that no contraction changes, for the
// values the FP64 sweep must round exactly as the forward step does.
namespace fwd {
__device__ __forceinline__ double mul(double a, double b)
{
    return __dmul_rn(a, b);
}
__device__ __forceinline__ double add(double a, double b)
{
    return __dadd_rn(a, b);
}
__device__ __forceinline__ double sub(double a, double b)
{
    return __dsub_rn(a, b);
}
__device__ __forceinline__ double div(double a, double b)
{
    return __ddiv_rn(a, b);
}
} // namespace fwd

// The reverse sweep of one tile (index `tile` in x-fastest tile order) by the
// whole CTA; smem_raw holds AdjShape::smem() bytes.  It starts with a CTA
// barrier, so a CTA may run several tiles back to back.
// redirect: a contribution to a ghost cell goes straight to the interior cell
// the ghost is filled from (bc_source in each dimension, the normal momentum
// negated for a Reflexive face), so that lam_in needs no fold afterwards.
// lam_zero (optional): a third adjoint buffer, which the CTA clears on its own
// interior tile for the next step to add into.
// SPH: spherical geometry (uniform spacing per coordinate): the flux
// differences carry each face's area over the cell's volume
// (extrapolation_reconstruction.hpp:130-142, godunov_scheme.hpp:157-163) and
// the geometric source terms enter the predictor and the update
// (adj::sph_source).
// gbar (optional, internal-mass gravity): gbar[i] += dJ/dg_r[i], the
// derivative with respect to the radial gravity table the step read, over
// the cells the tile's face states and output cells touch.
// EXACTB (FP64 sweep): take the primitives as the bit-exact FP64 forward
// step rounds them and its limiter branch test (phases 1 and 4); for a
// forward in other arithmetic (FP32-mixed, fast FP64) the plain forms.
// FX: the g.nfx passive scalars (state planes NV .. NV + nfx - 1, mass
// fractions) ride along; smem_raw then holds AdjShape::smem(g.nfx) bytes.
// Their forward (extrapolation_reconstruction.hpp:87-88, :315-339,
// godunov_scheme.hpp:262-301): face values x_f = x -/+ phi/2 from the limited
// slopes, times the face density, plus the predictor's increment
// sum_d c_d (x_{L,d} m_{L,d} - x_{R,d} m_{R,d}) (m: the mass fluxes of the
// reconstructed face states), over the predicted face density; the update
// rho'x' = rho x + sum_d c_d (x_up m - x_up m) with the upwind face value of
// each face's Riemann mass flux m, and x' = clamp(rho'x' / rho', 0, 1).  Phases
// 2b and 2c recompute the mass fluxes and each output cell's division; the
// reverse of the division adds -lam_v v / rho' to the new density's adjoint
// and the upwind fluxes add x_up lam to the mass flux, both on the faces of
// the tile's own cells (phase 3, which also runs the Riemann reverse for the
// scalar part of a face the next tile owns); phase 4 takes the predicted face
// values back to the face densities, the mass fluxes of the reconstructed
// states and the scalars' slopes.  Branches (limiters, the upwind choice, the
// clamp) are those of the sweep's own recomputation.
// NU: a grid of user-defined nodes (g.uniform_dx false); the regular-grid
// instantiation keeps the homogeneous limiter forms and one coefficient per
// direction, and carries none of the per-cell spacing code.
template <int ND, class R, int TX, int TY, int TZ, int NT, bool SPH = false, bool EXACTB = true, bool FX = false,
          bool NU = false>
__device__ __forceinline__ void adjoint_tile(const GridDev& g, const StateDev& U, const StateDev& lam_out,
                                             const StateDev& lam_in, double dt, int tile, unsigned char* smem_raw,
                                             const StateDev* lam_zero = nullptr, bool redirect = false,
                                             double* gbar = nullptr)
{
    using S = Shape<ND, TX, TY, TZ>;
    using AS = AdjShape<ND, R, TX, TY, TZ>;
    constexpr int NV = S::NV;
    const int nfx = FX ? g.nfx : 0;
    __syncthreads(); // the previous tile of this CTA is done with the shared arrays
    double* sl = reinterpret_cast<double*>(smem_raw);       // lambda' [NV][NP] (FP64)
    double* sgr = sl + NV * S::NP;                          // FX: new-density adjoint of the division [TVOL]
    double* sgx = sgr + (FX ? S::TVOL : 0);                 // FX: adjoint of rho'x' [nfx][TVOL]
    R* sw = reinterpret_cast<R*>(sgx + nfx * S::TVOL);      // primitives [NV][NP]
    R* swb = sw + NV * S::NP;                               // primitive adjoints [NV][NP]
    R* sa = swb + NV * S::NP;                               // face states per d [2][NV][A_d]
    R* sab = sa + S::A_TOTAL;                               // face-state adjoints
    R* swx = sab + S::A_TOTAL;                              // FX: scalar primitives [nfx][NP]
    R* swxb = swx + nfx * S::NP;                            // FX: their adjoints
    R* sxa = swxb + nfx * S::NP;                            // FX: predicted face values [nfx][XA]
    R* sxab = sxa + nfx * AS::XA;                           // FX: their adjoints
    R* sfm = sxab + nfx * AS::XA;                           // FX: Riemann mass flux per face [FS]

    const int tid = threadIdx.x;
    const adj::Eos<R> eos{(R)g.gamma, (R)g.gamma_m1, (R)(1.0 / g.gamma_m1)};
    const double dth = dt / 2;
    R cth[3], cfull[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        cth[d] = (R)(dth * g.inv_dx[d]);
        cfull[d] = (R)(dt * g.inv_dx[d]);
    }

    int ntile[2];
    ntile[0] = (g.nx[0] + S::T0 - 1) / S::T0;
    ntile[1] = (g.nx[1] + S::T1 - 1) / S::T1;
    int tc[3];
    {
        int b = tile;
        tc[0] = b % ntile[0];
        b /= ntile[0];
        tc[1] = b % ntile[1];
        tc[2] = b / ntile[1];
    }
    const int t0[3] = {tc[0] * S::T0, tc[1] * S::T1, tc[2] * S::T2};
    const int gorg[3] = {g.ng + t0[0], ND >= 2 ? g.ng + t0[1] : 0, ND >= 3 ? g.ng + t0[2] : 0};
    const int lstride[3] = {1, S::L0, S::L0 * S::L1};
    auto ntile_d = [&](int d) { return (g.nx[d] + S::T(d) - 1) / S::T(d); };
    // spherical geometry of the cell at global index (i, j, k), clamped into
    // the arrays (cells beyond them carry no adjoint)
    auto geo_cell = [&](int i, int j, int k) {
        return lidx(g, min(max(i, 0), g.n[0] - 1), min(max(j, 0), g.n[1] - 1), min(max(k, 0), g.n[2] - 1));
    };
    // source-term factors along d of that cell; kfac is dt (update) or dt/2
    // (predictor) and is divided by the cell's volume
    auto sph_geo = [&](int i, int j, int k, int d, double kfac) {
        adj::SphGeo<R> sg;
        const int64_t c = geo_cell(i, j, k);
        const int64_t cp = geo_cell(i + (d == 0), j + (d == 1), k + (d == 2));
        sg.k = (R)(kfac / g.dv[c]);
        sg.dS = (R)g.ds[c + g.N * d];
        sg.dSp = (R)g.ds[cp + g.N * d];
        const int ic = min(max(i, 0), g.n[0] - 1);
        const double x0 = g.x[0][ic], x0p = g.x[0][ic + 1];
        sg.rf = (R)((x0p - x0) / (x0p + x0));
        sg.cot = R(0);
        sg.sf = R(0);
        if (ND == 3) { // the polar-angle factors enter the 3-D terms only
            const int jc = min(max(j, 0), g.n[1] - 1);
            const double sm = g.sin1[jc], sp = g.sin1[jc + 1];
            sg.cot = (R)g.cot_mid1[jc];
            sg.sf = (R)((sp - sm) / (sp + sm));
        }
        return sg;
    };

    // Grids of non-uniform spacing (limited_linear_reconstruction.hpp:46-64):
    // the face values are w -/+ (dl/2) lim(dR / hR, dL / hL) with the half
    // spacings hR = (dl + dl_p)/2, hL = (dl_m + dl)/2, so phi = dl lim(...)
    // and its partials carry dl/hR and dl/hL; on uniform grids (g.uniform_dx)
    // the limiters' degree-1 homogeneity gives lim(dR, dL).  `gd` is the
    // cell's global index along d; `exact`: the FP64 sweep's forward-rounded
    // branch test.
    auto limited_phi = [&](int d, int gd, R dR, R dL, R* gR, R* gL, bool exact) -> R {
        if constexpr (!NU) {
            return adj::limiter(g.limiter, dR, dL, gR, gL);
        }
        const int c = min(max(gd, 1), g.n[d] - 2);
        const double dl = g.dx[d][c];
        const double hR = fwd::div(fwd::add(dl, g.dx[d][c + 1]), 2.0);
        const double hL = fwd::div(fwd::add(g.dx[d][c - 1], dl), 2.0);
        R a, b, sl;
        if (exact) {
            const bool active = fwd::mul(fwd::div((double)dL, hL), fwd::div((double)dR, hR)) > 0;
            sl = adj::limiter_on(g.limiter, active, (R)(dR / hR), (R)(dL / hL), &a, &b);
        } else {
            sl = adj::limiter(g.limiter, (R)(dR / hR), (R)(dL / hL), &a, &b);
        }
        *gR = (R)(dl / hR) * a;
        *gL = (R)(dl / hL) * b;
        return (R)dl * sl;
    };
    // Cartesian predictor (dt/2) and update (dt) coefficients of the cell at
    // global index gd along d: dt dS / dV = dt / dx_gd
    auto cth_at = [&](int d, int gd) -> R {
        if constexpr (!NU) {
            return cth[d];
        }
        return (R)(dth / g.dx[d][min(max(gd, 0), g.n[d] - 1)]);
    };
    auto cfull_at = [&](int d, int gd) -> double {
        if constexpr (!NU) {
            return dt * g.inv_dx[d];
        }
        return dt / g.dx[d][min(max(gd, 0), g.n[d] - 1)];
    };

    if (lam_zero) {
        // this tile's interior cells of the buffer the next step adds into
        for (int c = tid; c < S::TVOL; c += NT) {
            const int x0 = c % S::T0, x1 = (c / S::T0) % S::T1, x2 = c / (S::T0 * S::T1);
            if (t0[0] + x0 < g.nx[0] && (ND < 2 || t0[1] + x1 < g.nx[1]) && (ND < 3 || t0[2] + x2 < g.nx[2])) {
                const int64_t o = sidx(*lam_zero, g.n[1], gorg[0] + x0, gorg[1] + x1, gorg[2] + x2);
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    lam_zero->q[o + lam_zero->plane * v] = 0.0;
                }
                for (int k = 0; k < nfx; ++k) {
                    lam_zero->q[o + lam_zero->plane * (NV + k)] = 0.0;
                }
            }
        }
    }

    // ---- phase 1: primitives, lambda', zero adjoint buffers --------------
    for (int p = tid; p < S::NP; p += NT) {
        const int lx = p % S::L0;
        const int ly = (p / S::L0) % S::L1;
        const int lz = p / (S::L0 * S::L1);
        const int ri = gorg[0] - 2 + lx;
        const int rj = ND >= 2 ? gorg[1] - 2 + ly : 0;
        const int rk = ND >= 3 ? gorg[2] - 2 + lz : 0;
        const int gi = min(max(ri, 0), g.n[0] - 1);
        const int gj = min(max(rj, 0), g.n[1] - 1);
        const int gk = min(max(rk, 0), g.n[2] - 1);
        const int64_t o = sidx(U, g.n[1], gi, gj, gk);
        R q[NV], w[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            q[v] = (R)U.q[o + U.plane * v];
        }
        if constexpr (std::is_same<R, double>::value && EXACTB) {
            prim_forward_rounding<ND>(g, q, w);
        } else {
            adj::prim_from_cons<ND>(eos, q, w);
        }
        // lambda' lives on output (interior) cells only
        bool out_cell = ri >= g.ng && ri < g.n[0] - g.ng;
        if (ND >= 2) {
            out_cell = out_cell && rj >= g.ng && rj < g.n[1] - g.ng;
        }
        if (ND >= 3) {
            out_cell = out_cell && rk >= g.ng && rk < g.n[2] - g.ng;
        }
        const int64_t ol = sidx(lam_out, g.n[1], gi, gj, gk);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            sw[v * S::NP + p] = w[v];
            swb[v * S::NP + p] = R(0);
            sl[v * S::NP + p] = out_cell ? lam_out.q[ol + lam_out.plane * v] : 0.0;
        }
        for (int k = 0; k < nfx; ++k) {
            swx[k * S::NP + p] = (R)U.q[o + U.plane * (NV + k)];
            swxb[k * S::NP + p] = R(0);
        }
    }
    for (int a = tid; a < S::A_TOTAL; a += NT) {
        sab[a] = R(0);
    }
    for (int a = tid; a < nfx * AS::XA; a += NT) {
        sxab[a] = R(0);
    }
    __syncthreads();

    // helper: decode the a-th cell of the union H (interior + one slab per side and dim)
    auto decode_h = [&](int h, int x[3], int& own) {
        x[0] = x[1] = x[2] = 0;
        own = -1;
        int r = h;
        if (r < S::TVOL) {
            x[0] = r % S::T0;
            x[1] = (r / S::T0) % S::T1;
            x[2] = r / (S::T0 * S::T1);
            return;
        }
        r -= S::TVOL;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const int slab = S::TVOL / S::T(d);
            if (own < 0) {
                if (r < 2 * slab) {
                    own = d;
                    const int side = r / slab;
                    int rr = r % slab;
#pragma unroll
                    for (int e = 0; e < 3; ++e) {
                        if (e == d) {
                            continue;
                        }
                        x[e] = rr % S::T(e);
                        rr /= S::T(e);
                    }
                    x[d] = side == 0 ? -1 : S::T(d);
                } else {
                    r -= 2 * slab;
                }
            }
        }
    };
    auto lcell = [&](const int x[3]) {
        return (x[0] + 2) + S::L0 * ((ND >= 2 ? x[1] + 2 : 0) + S::L1 * (ND >= 3 ? x[2] + 2 : 0));
    };

    // ---- phase 2: forward Hancock face states (recomputed) -----------------
    for (int h = tid; h < S::HCOUNT; h += NT) {
        int x[3], own;
        decode_h(h, x, own);
        const int lc = lcell(x);
        const int gi = gorg[0] + x[0]; // x0 index of the cell (gravity table)
        const int gj = gorg[1] + x[1], gk = gorg[2] + x[2];
        R fp[2][ND][NV];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const R wc = sw[v * S::NP + lc];
                R gR, gL;
                // the value only: a branch taken differently at a raw product
                // that underflows changes it by less than 1e-270
                const R phi = limited_phi(d, gorg[d] + x[d], sw[v * S::NP + lc + lstride[d]] - wc,
                                          wc - sw[v * S::NP + lc - lstride[d]], &gR, &gL, false);
                fp[0][d][v] = wc - R(0.5) * phi;
                fp[1][d][v] = wc + R(0.5) * phi;
            }
        }
        R fc[2][ND][NV];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                adj::cons_from_prim<ND>(eos, fp[s][d], fc[s][d]);
            }
        }
        R inc[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            inc[v] = R(0);
        }
        // FX: mass fluxes of the reconstructed face states and the predictor's
        // coefficients of the left and right face along d
        R mfl[ND], mfr[ND], ccl[ND], ccr[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            R fL[NV], fR[NV];
            adj::flux_prim<ND>(eos, fp[0][d], d, fL);
            adj::flux_prim<ND>(eos, fp[1][d], d, fR);
            mfl[d] = fL[0];
            mfr[d] = fR[0];
            if constexpr (SPH) {
                const adj::SphGeo<R> sg = sph_geo(gi, gj, gk, d, dth);
                const R cl = sg.k * sg.dS, cr = sg.k * sg.dSp;
                ccl[d] = cl;
                ccr[d] = cr;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    inc[v] += cl * fL[v] - cr * fR[v];
                }
                adj::sph_source<ND>(sg, d, fp[0][d], fp[1][d], inc);
            } else {
                const R ct = cth_at(d, gorg[d] + x[d]);
                ccl[d] = ccr[d] = ct;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    inc[v] += ct * (fL[v] - fR[v]);
                }
            }
        }
        if constexpr (FX) {
            // predicted face values of each scalar (written in the forms of the
            // density's predictor, so that a scalar equal to 1 over the stencil
            // gives face values of exactly 1, as in the forward step)
            for (int k = 0; k < nfx; ++k) {
                const R* xk = swx + k * S::NP;
                R xf[2][ND];
                R xinc = R(0);
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    const R xc = xk[lc];
                    R gR, gL;
                    const R phi =
                        limited_phi(d, gorg[d] + x[d], xk[lc + lstride[d]] - xc, xc - xk[lc - lstride[d]], &gR, &gL, false);
                    xf[0][d] = xc - R(0.5) * phi;
                    xf[1][d] = xc + R(0.5) * phi;
                }
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    if constexpr (SPH) {
                        xinc += ccl[d] * (xf[0][d] * mfl[d]) - ccr[d] * (xf[1][d] * mfr[d]);
                    } else {
                        xinc += ccl[d] * (xf[0][d] * mfl[d] - xf[1][d] * mfr[d]);
                    }
                }
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    if (own >= 0 && own != d) {
                        continue;
                    }
                    const int ax = x[0] + (d == 0), ay = x[1] + (d == 1), az = x[2] + (d == 2);
                    const int a = ax + S::Adim(d, 0) * (ay + S::Adim(d, 1) * az);
                    R* xb = sxa + k * AS::XA + AS::XAoff(d);
#pragma unroll
                    for (int s2 = 0; s2 < 2; ++s2) {
                        const R rho_pred = fc[s2][d][0] + inc[0];
                        xb[s2 * S::Asize(d) + a] = (xf[s2][d] * fc[s2][d][0] + xinc) / rho_pred;
                    }
                }
            }
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            if (own >= 0 && own != d) {
                continue;
            }
            const int ax = x[0] + (d == 0), ay = x[1] + (d == 1), az = x[2] + (d == 2);
            const int a = ax + S::Adim(d, 0) * (ay + S::Adim(d, 1) * az);
            R* base = sa + S::Aoff(d);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                R hs[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    hs[v] = fc[s][d][v] + inc[v];
                }
#pragma unroll
                for (int e = 0; e < ND; ++e) {
                    const R gg = (R)(dth * gravity_at(g, gi, e));
                    hs[1 + e] += gg * fc[s][d][0];
                    hs[1 + ND] += gg * fc[s][d][1 + e];
                }
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    base[(s * NV + v) * S::Asize(d) + a] = hs[v];
                }
            }
        }
    }
    __syncthreads();

    // tile-interior index of an own output cell, -1 for a cell outside the
    // tile or beyond the domain
    auto own_index = [&](const int x[3]) {
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            if (x[d] < 0 || x[d] >= S::T(d) || t0[d] + x[d] >= g.nx[d]) {
                return -1;
            }
        }
        return x[0] + S::T0 * (x[1] + S::T1 * x[2]);
    };
    // update coefficient of the left (side 0) or right (side 1) face along d
    // of tile cell x: dt dS / dV of that cell (dt/dx on Cartesian grids)
    auto upd_coef = [&](const int x[3], int d, int side) -> double {
        if constexpr (SPH) {
            const int i1 = gorg[0] + x[0], j1 = gorg[1] + x[1], k1 = gorg[2] + x[2];
            const int64_t c = geo_cell(i1, j1, k1);
            const int64_t cf = side ? geo_cell(i1 + (d == 0), j1 + (d == 1), k1 + (d == 2)) : c;
            return dt / g.dv[c] * g.ds[cf + g.N * d];
        } else {
            return cfull_at(d, gorg[d] + x[d]);
        }
    };
    // A index along d of tile cell x (the H cells -1 .. T_d along d)
    auto a_index = [&](const int x[3], int d) {
        return (x[0] + (d == 0)) + S::Adim(d, 0) * ((x[1] + (d == 1)) + S::Adim(d, 1) * (x[2] + (d == 2)));
    };
    auto a_step = [&](int d) { return d == 0 ? 1 : (d == 1 ? S::Adim(d, 0) : S::Adim(d, 0) * S::Adim(d, 1)); };
    if constexpr (FX) {
        // ---- phase 2b: Riemann mass flux of every face of the tile -------------
        if (nfx > 0) {
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                const R* base = sa + S::Aoff(d);
                for (int f = tid; f < S::Fsize(d); f += NT) {
                    int x[3];
                    x[0] = f % S::Fdim(d, 0);
                    x[1] = (f / S::Fdim(d, 0)) % S::Fdim(d, 1);
                    x[2] = f / (S::Fdim(d, 0) * S::Fdim(d, 1));
                    const int aRd = a_index(x, d);
                    const int aLd = aRd - a_step(d);
                    R UL[NV], UR[NV], F[NV];
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        UL[v] = base[(NV + v) * S::Asize(d) + aLd];
                        UR[v] = base[v * S::Asize(d) + aRd];
                    }
                    adj::riemann<ND>(eos, g.riemann, UL, UR, d, F);
                    sfm[AS::FSoff(d) + f] = F[0];
                }
            }
            __syncthreads();
            // ---- phase 2c: each own output cell's division rho'x' / rho' ---------
            // (godunov_scheme.hpp:294-301): the clamp's branch, the adjoint of
            // rho'x' and the division's part of the new density's adjoint
            for (int c = tid; c < S::TVOL; c += NT) {
                int x[3] = {c % S::T0, (c / S::T0) % S::T1, c / (S::T0 * S::T1)};
                if (own_index(x) < 0) {
                    sgr[c] = 0.0;
                    for (int k = 0; k < nfx; ++k) {
                        sgx[k * S::TVOL + c] = 0.0;
                    }
                    continue;
                }
                const int lc = lcell(x);
                double cl[ND], cr[ND];
                R ml[ND], mr[ND];
                int fl_[ND], fr_[ND];
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    cl[d] = upd_coef(x, d, 0);
                    cr[d] = upd_coef(x, d, 1);
                    fl_[d] = x[0] + S::Fdim(d, 0) * (x[1] + S::Fdim(d, 1) * x[2]);
                    const int st = d == 0 ? 1 : (d == 1 ? S::Fdim(d, 0) : S::Fdim(d, 0) * S::Fdim(d, 1));
                    fr_[d] = fl_[d] + st;
                    ml[d] = sfm[AS::FSoff(d) + fl_[d]];
                    mr[d] = sfm[AS::FSoff(d) + fr_[d]];
                }
                const R rc = sw[lc];
                R rn = rc;
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    rn += (R)cl[d] * ml[d] - (R)cr[d] * mr[d];
                }
                const int64_t ol = sidx(lam_out, g.n[1], gorg[0] + x[0], gorg[1] + x[1], gorg[2] + x[2]);
                double extra = 0.0;
                for (int k = 0; k < nfx; ++k) {
                    const R* xa = sxa + k * AS::XA;
                    R rx = swx[k * S::NP + lc] * rc;
#pragma unroll
                    for (int d = 0; d < ND; ++d) {
                        const R* xd = xa + AS::XAoff(d);
                        const int a = a_index(x, d);
                        // left face: this cell's left value when the mass flows
                        // left, else the left cell's right value; right face alike
                        const R xl = ml[d] < R(0) ? xd[a] : xd[S::Asize(d) + a - a_step(d)];
                        const R xr = mr[d] < R(0) ? xd[a + a_step(d)] : xd[S::Asize(d) + a];
                        rx += (R)cl[d] * (xl * ml[d]) - (R)cr[d] * (xr * mr[d]);
                    }
                    const R v = rx / rn;
                    const bool free_ = !(v < R(0)) && !(v > R(1));
                    const double lv = free_ ? lam_out.q[ol + lam_out.plane * (NV + k)] : 0.0;
                    const double lrx = lv / (double)rn;
                    sgx[k * S::TVOL + c] = lrx;
                    extra -= lrx * (double)v;
                }
                sgr[c] = extra;
            }
            __syncthreads();
        }
    }

    // ---- phase 3: adjoint of each owned face through the Riemann solver ---------
    // A tile owns the left face of each of its interior cells; the last tile
    // along d also owns the domain's last face (the right face of the last
    // interior cell), so every face an interior update uses has one owner.
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const R* base = sa + S::Aoff(d);
        R* bb = sab + S::Aoff(d);
        const bool last_d = tc[d] == ntile_d(d) - 1;
        for (int f = tid; f < S::Fsize(d); f += NT) {
            int x[3];
            x[0] = f % S::Fdim(d, 0);
            x[1] = (f / S::Fdim(d, 0)) % S::Fdim(d, 1);
            x[2] = f / (S::Fdim(d, 0) * S::Fdim(d, 1));
            // the next tile along d owns the face x_d = T_d; with passive
            // scalars this tile still runs the Riemann reverse for the part of
            // that face's mass-flux adjoint its own cell contributes
            const bool owned = !(x[d] == S::T(d) && !last_d);
            if (!owned && (!FX || nfx == 0)) {
                continue;
            }
            // cells R = x and L = x - e_d (R may be the slab cell x_d = T_d)
            const int lcR = lcell(x);
            const int lcL = lcR - lstride[d];
            R Fb[NV];
            bool nz = false;
            if (!owned) {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    Fb[v] = R(0);
                }
            } else if constexpr (SPH) {
                // the face enters U'_R with +dt dS / dv_R and U'_L with -dt dS / dv_L
                const int i1 = gorg[0] + x[0], j1 = gorg[1] + x[1], k1 = gorg[2] + x[2];
                const int64_t cR = geo_cell(i1, j1, k1);
                const int64_t cL = geo_cell(i1 - (d == 0), j1 - (d == 1), k1 - (d == 2));
                const double area = g.ds[cR + g.N * d];
                const double kR = dt / g.dv[cR] * area, kL = dt / g.dv[cL] * area;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    Fb[v] = (R)(kR * sl[v * S::NP + lcR] - kL * sl[v * S::NP + lcL]);
                    nz |= Fb[v] != R(0);
                }
            } else {
                if constexpr (!NU) {
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        Fb[v] = (R)(cfull[d] * (sl[v * S::NP + lcR] - sl[v * S::NP + lcL]));
                        nz |= Fb[v] != R(0);
                    }
                } else {
                    // the face enters U'_R with +dt/dx_R and U'_L with -dt/dx_L
                    const double cR = cfull_at(d, gorg[d] + x[d]), cL = cfull_at(d, gorg[d] + x[d] - 1);
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        Fb[v] = (R)(cR * sl[v * S::NP + lcR] - cL * sl[v * S::NP + lcL]);
                        nz |= Fb[v] != R(0);
                    }
                }
            }
            if constexpr (FX) {
                // scalar part from the tile's own cells on either side: the
                // division's density adjoint and the upwind fluxes x_up m
                int xl[3] = {x[0], x[1], x[2]};
                xl[d] -= 1;
                const int tR = own_index(x), tL = own_index(xl);
                if (nfx > 0 && (tR >= 0 || tL >= 0)) {
                    const R m = sfm[AS::FSoff(d) + f];
                    const int aR = a_index(x, d), aL = aR - a_step(d);
                    const double cR = tR >= 0 ? upd_coef(x, d, 0) : 0.0;  // R's left face
                    const double cL = tL >= 0 ? upd_coef(xl, d, 1) : 0.0; // L's right face
                    double gm = (tR >= 0 ? cR * sgr[tR] : 0.0) - (tL >= 0 ? cL * sgr[tL] : 0.0);
                    // upwind value: the right cell's left value when the mass flows left
                    const int slot = m < R(0) ? aR : S::Asize(d) + aL;
                    for (int k = 0; k < nfx; ++k) {
                        const double lf = (tR >= 0 ? cR * sgx[k * S::TVOL + tR] : 0.0) -
                                          (tL >= 0 ? cL * sgx[k * S::TVOL + tL] : 0.0);
                        if (lf != 0.0) {
                            const int xo = k * AS::XA + AS::XAoff(d) + slot;
                            gm += lf * (double)sxa[xo];
                            sxab[xo] = (R)(lf * (double)m);
                        }
                    }
                    if (gm != 0.0) {
                        Fb[0] += (R)gm;
                        nz = true;
                    }
                }
            }
            if (!nz) {
                continue;
            }
            // A coordinates: the left cell x_d - 1 has A index x_d along d, the right cell x_d + 1
            const int aLd = x[0] + S::Adim(d, 0) * (x[1] + S::Adim(d, 1) * x[2]);
            const int stepd = d == 0 ? 1 : (d == 1 ? S::Adim(d, 0) : S::Adim(d, 0) * S::Adim(d, 1));
            const int aRd = aLd + stepd;
            R UL[NV], UR[NV], ULb[NV], URb[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                UL[v] = base[(NV + v) * S::Asize(d) + aLd];
                UR[v] = base[v * S::Asize(d) + aRd];
                ULb[v] = URb[v] = R(0);
            }
            adj::riemann_rev<ND>(eos, g.riemann, UL, UR, d, Fb, ULb, URb);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                bb[(NV + v) * S::Asize(d) + aLd] = ULb[v];
                bb[v * S::Asize(d) + aRd] = URb[v];
            }
        }
    }
    __syncthreads();

    // ---- phase 4: reverse Hancock + slopes of every cell with face adjoints ------
    for (int h = tid; h < S::HCOUNT; h += NT) {
        int x[3], own;
        decode_h(h, x, own);
        const int lc = lcell(x);
        const int gi = gorg[0] + x[0]; // x0 index of the cell (gravity table)
        const int gj = gorg[1] + x[1], gk = gorg[2] + x[2];
        // gather this cell's face-state adjoints
        R Hb[2][ND][NV];
        bool any = false;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const bool has = own < 0 || own == d;
            const int ax = x[0] + (d == 0), ay = x[1] + (d == 1), az = x[2] + (d == 2);
            const int a = ax + S::Adim(d, 0) * (ay + S::Adim(d, 1) * az);
            const R* bb = sab + S::Aoff(d);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    Hb[s][d][v] = has ? bb[(s * NV + v) * S::Asize(d) + a] : R(0);
                    any |= Hb[s][d][v] != R(0);
                }
                if constexpr (FX) {
                    for (int k = 0; k < nfx; ++k) {
                        any |= has && sxab[k * AS::XA + AS::XAoff(d) + s * S::Asize(d) + a] != R(0);
                    }
                }
            }
        }
        if constexpr (SPH) {
            // the update's source terms on this cell's predicted states
            // (godunov_scheme.hpp:165-256), for the tile's own cells
            if (own < 0) {
                R lamc[NV];
                bool lz = false;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    lamc[v] = (R)sl[v * S::NP + lc];
                    lz |= lamc[v] != R(0);
                }
                if (lz) {
                    any = true;
#pragma unroll
                    for (int d = 0; d < (ND < 2 ? ND : 2); ++d) {
                        const int ax = x[0] + (d == 0), ay = x[1] + (d == 1), az = x[2] + (d == 2);
                        const int a = ax + S::Adim(d, 0) * (ay + S::Adim(d, 1) * az);
                        const R* base = sa + S::Aoff(d);
                        R H[2][NV], pH[2][NV], pHb[2][NV];
#pragma unroll
                        for (int s = 0; s < 2; ++s) {
#pragma unroll
                            for (int v = 0; v < NV; ++v) {
                                H[s][v] = base[(s * NV + v) * S::Asize(d) + a];
                                pHb[s][v] = R(0);
                            }
                            adj::prim_from_cons<ND>(eos, H[s], pH[s]);
                        }
                        adj::sph_source_rev<ND>(sph_geo(gi, gj, gk, d, dt), d, pH[0], pH[1], lamc, pHb[0], pHb[1]);
#pragma unroll
                        for (int s = 0; s < 2; ++s) {
                            adj::prim_from_cons_rev<ND>(eos, H[s], pHb[s], Hb[s][d]);
                        }
                    }
                }
            }
        }
        if (!any) {
            continue;
        }
        // recompute slopes and face primitives.  The FP64 sweep takes each
        // limiter's branch from the forward's R*L > 0, which the forward forms
        // from the differences divided by the half-spacings (dl + dl_p)/2 and
        // (dl_m + dl)/2.  Where the raw product is too small for those
        // quotients' product to stay above the subnormal range (1.0e-33 x
        // 3.1e-292 underflows to 0, (64 x 1.0e-33) x (64 x 3.1e-292) does
        // not), the test is evaluated as the forward rounds it; elsewhere both
        // products have the same sign.  The FP32 sweep decides on its own
        // differences.
        R fp[2][ND][NV], gRs[ND][NV], gLs[ND][NV];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const R wc = sw[v * S::NP + lc];
                const R dR = sw[v * S::NP + lc + lstride[d]] - wc;
                const R dL = wc - sw[v * S::NP + lc - lstride[d]];
                R phi;
                if constexpr (NU) {
                    phi = limited_phi(d, gorg[d] + x[d], dR, dL, &gRs[d][v], &gLs[d][v],
                                      std::is_same<R, double>::value && EXACTB);
                } else if constexpr (std::is_same<R, double>::value && EXACTB) {
                    const double prod = dR * dL;
                    bool active = prod > 0;
                    if (fabs(prod) * (g.inv_dx[d] * g.inv_dx[d]) <= 1e-270) {
                        const int gd = min(max(gorg[d] + x[d], 1), g.n[d] - 2);
                        const double dl = g.dx[d][gd];
                        const double hR = fwd::div(fwd::add(dl, g.dx[d][gd + 1]), 2.0);
                        const double hL = fwd::div(fwd::add(g.dx[d][gd - 1], dl), 2.0);
                        active = fwd::mul(fwd::div(dL, hL), fwd::div(dR, hR)) > 0;
                    }
                    phi = adj::limiter_on(g.limiter, active, dR, dL, &gRs[d][v], &gLs[d][v]);
                } else {
                    phi = adj::limiter(g.limiter, dR, dL, &gRs[d][v], &gLs[d][v]);
                }
                fp[0][d][v] = wc - R(0.5) * phi;
                fp[1][d][v] = wc + R(0.5) * phi;
            }
        }
        R fpb[2][ND][NV];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    fpb[s][d][v] = R(0);
                }
            }
        }
        // FX: reverse of the scalars' predicted face values
        // x_p[s][ip] = (x_f[s][ip] rho_f[s][ip] + xinc) / rho_p[s][ip],
        // xinc = sum_d (c_l x_f[0][d] m[0][d] - c_r x_f[1][d] m[1][d]): adjoints of the
        // predicted face densities (Hb[.][.][0]), of the face densities (fpb[.][.][0]),
        // of the face mass fluxes m (mfb, taken back through the flux's first
        // component below) and of the scalars' slopes
        R mfb[2][ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            mfb[0][d] = mfb[1][d] = R(0);
        }
        if constexpr (FX) {
            R mf[2][ND], ccl[ND], ccr[ND];
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                mf[0][d] = fp[0][d][0] * fp[0][d][1 + d];
                mf[1][d] = fp[1][d][0] * fp[1][d][1 + d];
                if constexpr (SPH) {
                    const adj::SphGeo<R> sg = sph_geo(gi, gj, gk, d, dth);
                    ccl[d] = sg.k * sg.dS;
                    ccr[d] = sg.k * sg.dSp;
                } else {
                    ccl[d] = ccr[d] = cth_at(d, gorg[d] + x[d]);
                }
            }
            for (int k = 0; k < nfx; ++k) {
                R* xk = swx + k * S::NP;
                R xf[2][ND], xgR[ND], xgL[ND];
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    const R xc = xk[lc];
                    const R phi = limited_phi(d, gorg[d] + x[d], xk[lc + lstride[d]] - xc, xc - xk[lc - lstride[d]],
                                              &xgR[d], &xgL[d], false);
                    xf[0][d] = xc - R(0.5) * phi;
                    xf[1][d] = xc + R(0.5) * phi;
                }
                R xinc = R(0);
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    xinc += ccl[d] * (xf[0][d] * mf[0][d]) - ccr[d] * (xf[1][d] * mf[1][d]);
                }
                R xfb[2][ND];
                R xincb = R(0);
#pragma unroll
                for (int ip = 0; ip < ND; ++ip) {
                    xfb[0][ip] = xfb[1][ip] = R(0);
                    if (own >= 0 && own != ip) {
                        continue;
                    }
                    const int a = a_index(x, ip);
                    const R* base = sa + S::Aoff(ip);
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const R xpb = sxab[k * AS::XA + AS::XAoff(ip) + s * S::Asize(ip) + a];
                        if (xpb == R(0)) {
                            continue;
                        }
                        const R rp = base[s * NV * S::Asize(ip) + a]; // predicted face density
                        const R inv = R(1) / rp;
                        const R xp = (xf[s][ip] * fp[s][ip][0] + xinc) * inv;
                        const R xrb = xpb * inv;
                        Hb[s][ip][0] -= xrb * xp;
                        xfb[s][ip] += xrb * fp[s][ip][0];
                        fpb[s][ip][0] += xrb * xf[s][ip];
                        xincb += xrb;
                    }
                }
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    xfb[0][d] += ccl[d] * xincb * mf[0][d];
                    xfb[1][d] -= ccr[d] * xincb * mf[1][d];
                    mfb[0][d] += ccl[d] * xincb * xf[0][d];
                    mfb[1][d] -= ccr[d] * xincb * xf[1][d];
                }
                // slopes: x_f[0/1][d] = x_c -/+ phi/2
                R* xkb = swxb + k * S::NP;
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    const R phib = R(0.5) * (xfb[1][d] - xfb[0][d]);
                    const R dRb = phib * xgR[d];
                    const R dLb = phib * xgL[d];
                    const R own_b = xfb[0][d] + xfb[1][d] - dRb + dLb;
                    if (own_b != R(0)) {
                        atomicAdd(&xkb[lc], own_b);
                    }
                    if (dRb != R(0)) {
                        atomicAdd(&xkb[lc + lstride[d]], dRb);
                    }
                    if (dLb != R(0)) {
                        atomicAdd(&xkb[lc - lstride[d]], -dLb);
                    }
                }
            }
        }
        // H[s][ipos] = cons(fp[s][ipos]) + sum_d cth_d (F(fp[0][d]) - F(fp[1][d])) + gravity(cons(fp[s][ipos]))
        R Sb[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            Sb[v] = R(0);
        }
        if (gbar) {
            // H[s][ip]: m_0 += (dt/2) g_r rho_f, E += (dt/2) g_r m_0,f of the
            // face state's conserved form (extrapolation_reconstruction.hpp:306-312)
            double gs = 0.0;
#pragma unroll
            for (int ip = 0; ip < ND; ++ip) {
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    R fc[NV];
                    adj::cons_from_prim<ND>(eos, fp[s][ip], fc);
                    gs += (double)Hb[s][ip][1] * (double)fc[0] + (double)Hb[s][ip][1 + ND] * (double)fc[1];
                }
            }
            if (gs != 0.0 && gi >= 0 && gi < g.n[0]) {
                atomicAdd(&gbar[gi], dth * gs);
            }
        }
#pragma unroll
        for (int ip = 0; ip < ND; ++ip) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                R cb[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    cb[v] = Hb[s][ip][v];
                    Sb[v] += Hb[s][ip][v];
                }
#pragma unroll
                for (int e = 0; e < ND; ++e) {
                    const R gg = (R)(dth * gravity_at(g, gi, e));
                    cb[0] += gg * Hb[s][ip][1 + e];
                    cb[1 + e] += gg * Hb[s][ip][1 + ND];
                }
                adj::cons_from_prim_rev<ND>(eos, fp[s][ip], cb, fpb[s][ip]);
            }
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            R Fb0[NV], Fb1[NV];
            if constexpr (SPH) {
                const adj::SphGeo<R> sg = sph_geo(gi, gj, gk, d, dth);
                const R cl = sg.k * sg.dS, cr = sg.k * sg.dSp;
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    Fb0[v] = cl * Sb[v];
                    Fb1[v] = -cr * Sb[v];
                }
                adj::sph_source_rev<ND>(sg, d, fp[0][d], fp[1][d], Sb, fpb[0][d], fpb[1][d]);
            } else {
                const R ct = cth_at(d, gorg[d] + x[d]);
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    Fb0[v] = ct * Sb[v];
                    Fb1[v] = -ct * Sb[v];
                }
            }
            if constexpr (FX) {
                Fb0[0] += mfb[0][d];
                Fb1[0] += mfb[1][d];
            }
            adj::flux_prim_rev<ND>(eos, fp[0][d], d, Fb0, fpb[0][d]);
            adj::flux_prim_rev<ND>(eos, fp[1][d], d, Fb1, fpb[1][d]);
        }
        // slopes: fp[0/1][d][v] = w_c -/+ phi/2, phi = limiter(w_{c+1} - w_c, w_c - w_{c-1})
#pragma unroll
        for (int d = 0; d < ND; ++d) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const R phib = R(0.5) * (fpb[1][d][v] - fpb[0][d][v]);
                const R dRb = phib * gRs[d][v];
                const R dLb = phib * gLs[d][v];
                atomicAdd(&swb[v * S::NP + lc], fpb[0][d][v] + fpb[1][d][v] - dRb + dLb);
                if (dRb != R(0)) {
                    atomicAdd(&swb[v * S::NP + lc + lstride[d]], dRb);
                }
                if (dLb != R(0)) {
                    atomicAdd(&swb[v * S::NP + lc - lstride[d]], -dLb);
                }
            }
        }
    }
    __syncthreads();

    // ---- phase 5: primitive recovery reverse, identity and gravity terms ---------
    for (int p = tid; p < S::NP; p += NT) {
        const int lx = p % S::L0;
        const int ly = (p / S::L0) % S::L1;
        const int lz = p / (S::L0 * S::L1);
        const int ri = gorg[0] - 2 + lx;
        const int rj = ND >= 2 ? gorg[1] - 2 + ly : 0;
        const int rk = ND >= 3 ? gorg[2] - 2 + lz : 0;
        if (ri < 0 || ri >= g.n[0] || rj < 0 || rj >= g.n[1] || rk < 0 || rk >= g.n[2]) {
            continue;
        }
        // owned output cell of this tile (identity + Godunov gravity terms)
        const int x0 = lx - 2, x1 = ly - 2, x2 = lz - 2;
        bool own_cell = x0 >= 0 && x0 < S::T0 && ri < g.n[0] - g.ng;
        if (ND >= 2) {
            own_cell = own_cell && x1 >= 0 && x1 < S::T1 && rj < g.n[1] - g.ng;
        }
        if (ND >= 3) {
            own_cell = own_cell && x2 >= 0 && x2 < S::T2 && rk < g.n[2] - g.ng;
        }
        R wb[NV];
        bool nz = own_cell;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            wb[v] = swb[v * S::NP + p];
            nz |= wb[v] != R(0);
        }
        for (int k = 0; k < nfx; ++k) {
            nz |= swxb[k * S::NP + p] != R(0);
        }
        if (!nz) {
            continue;
        }
        const int64_t o = sidx(U, g.n[1], ri, rj, rk);
        R q[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            q[v] = (R)U.q[o + U.plane * v];
        }
        R ub[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ub[v] = R(0);
        }
        adj::prim_from_cons_rev<ND>(eos, q, wb, ub);
        double outv[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            outv[v] = (double)ub[v];
        }
        if (own_cell) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                outv[v] += sl[v * S::NP + p];
            }
#pragma unroll
            for (int e = 0; e < ND; ++e) {
                // U'_m_e += dt g_e rho ; U'_E += dt g_e m_e   (godunov_scheme.hpp:258-260)
                const double ge = gravity_at(g, ri, e);
                outv[0] += dt * ge * sl[(1 + e) * S::NP + p];
                outv[1 + e] += dt * ge * sl[(1 + ND) * S::NP + p];
            }
            if (gbar) {
                const double gs = sl[1 * S::NP + p] * U.q[o] + sl[(1 + ND) * S::NP + p] * U.q[o + U.plane];
                if (gs != 0.0) {
                    atomicAdd(&gbar[ri], dt * gs);
                }
            }
        }
        int si = ri, sj = rj, sk = rk;
        int fl[3] = {0, 0, 0};
        if (redirect) {
            si = bc_source(ri, g.n[0], g.ng, g.bc[0], g.bc[1], &fl[0]);
            if (ND >= 2) {
                sj = bc_source(rj, g.n[1], g.ng, g.bc[2], g.bc[3], &fl[1]);
            }
            if (ND >= 3) {
                sk = bc_source(rk, g.n[2], g.ng, g.bc[4], g.bc[5], &fl[2]);
            }
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                if (fl[d]) {
                    outv[1 + d] = -outv[1 + d];
                }
            }
        }
        const int64_t oo = sidx(lam_in, g.n[1], si, sj, sk);
        if constexpr (FX) {
            // scalars: slopes and predictor; for an own cell also the identity
            // part rho'x' = rho x + ... (its density part goes to outv[0], with the
            // division's new-density adjoint, since rho' = rho + ...)
            // (x1, x2 are -2 along the inactive dimensions)
            const int tcell = own_cell ? x0 + S::T0 * ((ND >= 2 ? x1 : 0) + S::T1 * (ND >= 3 ? x2 : 0)) : -1;
            if (own_cell) {
                outv[0] += sgr[tcell]; // the density plane's atomic follows below
            }
            for (int k = 0; k < nfx; ++k) {
                double xb = (double)swxb[k * S::NP + p];
                if (own_cell) {
                    const double lrx = sgx[k * S::TVOL + tcell];
                    xb += lrx * U.q[o];
                    outv[0] += lrx * U.q[o + U.plane * (NV + k)];
                }
                if (xb != 0.0) {
                    atomicAdd(&lam_in.q[oo + lam_in.plane * (NV + k)], xb);
                }
            }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            if (outv[v] != 0.0) {
                atomicAdd(&lam_in.q[oo + lam_in.plane * v], outv[v]);
            }
        }
    }
}

// NT threads per CTA (any count: every phase strides over its items by NT).
// The FP32 sweep runs three CTAs per SM (56 registers, a few spilled): the
// tile's phases wait at barriers and the third CTA fills those waits
// (Gresho 512^2 backward pass 25.4 -> 23.8 ms).
template <class R, int NT>
constexpr int adj_min_blocks()
{
    return sizeof(R) == 8 ? (NT <= 256 ? 2 : 1) : (NT <= 256 ? 3 : (NT <= 384 ? 3 : 1));
}

// FX (passive scalars): one CTA per SM (the scalars' shared arrays)
template <int ND, class R, int TX, int TY, int TZ, int NT, bool SPH, bool EXACTB, bool FX = false, bool NU = false>
__global__ void __launch_bounds__(NT, FX ? 1 : adj_min_blocks<R, NT>())
k_adjoint_step(GridDev g, StateDev U, StateDev lam_out, StateDev lam_in, double dt, StateDev lam_zero, double* gbar)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    adjoint_tile<ND, R, TX, TY, TZ, NT, SPH, EXACTB, FX, NU>(g, U, lam_out, lam_in, dt, blockIdx.x, smem_raw,
                                                             &lam_zero, true, gbar);
}

// Transpose of the boundary fill: every interior cell gathers the adjoints of
// its ghost images (sign-flipped momentum for Reflexive faces).  Cells
// first, first + stride, ... of the interior.
template <int ND>
__device__ __forceinline__ void fold_cells(const GridDev& g, const StateDev& lam, int64_t first, int64_t stride)
{
    const int64_t count = (int64_t)g.nx[0] * g.nx[1] * g.nx[2];
    for (int64_t idx = first; idx < count; idx += stride) {
        const int ii = (int)(idx % g.nx[0]);
        const int64_t r = idx / g.nx[0];
        const int jj = (int)(r % g.nx[1]);
        const int kk = (int)(r / g.nx[1]);
        const int gidx[3] = {g.ng + ii, ND >= 2 ? g.ng + jj : 0, ND >= 3 ? g.ng + kk : 0};
        int pos[3][9], flp[3][9], cnt[3] = {1, 1, 1};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            pos[d][0] = gidx[d];
            flp[d][0] = 0;
            if (d < ND) {
                cnt[d] += fused::ghost_images(gidx[d], g.n[d], g.ng, g.bc[2 * d], g.bc[2 * d + 1], &pos[d][1], &flp[d][1]);
            }
        }
        if (cnt[0] * cnt[1] * cnt[2] == 1) {
            continue;
        }
        double acc[ND + 2];
        const int64_t oc = sidx(lam, g.n[1], gidx[0], gidx[1], gidx[2]);
#pragma unroll
        for (int v = 0; v < ND + 2; ++v) {
            acc[v] = lam.q[oc + lam.plane * v];
        }
        for (int a2 = 0; a2 < cnt[2]; ++a2) {
            for (int a1 = 0; a1 < cnt[1]; ++a1) {
                for (int a0 = 0; a0 < cnt[0]; ++a0) {
                    if (a0 == 0 && a1 == 0 && a2 == 0) {
                        continue;
                    }
                    const int64_t og = sidx(lam, g.n[1], pos[0][a0], pos[1][a1], pos[2][a2]);
                    const int fl[3] = {flp[0][a0], flp[1][a1], flp[2][a2]};
                    acc[0] += lam.q[og];
#pragma unroll
                    for (int d = 0; d < ND; ++d) {
                        const double v = lam.q[og + lam.plane * (1 + d)];
                        acc[1 + d] += fl[d] ? -v : v;
                    }
                    acc[1 + ND] += lam.q[og + lam.plane * (1 + ND)];
                    for (int k = 0; k < g.nfx; ++k) {
                        lam.q[oc + lam.plane * (ND + 2 + k)] += lam.q[og + lam.plane * (ND + 2 + k)];
                    }
                }
            }
        }
#pragma unroll
        for (int v = 0; v < ND + 2; ++v) {
            lam.q[oc + lam.plane * v] = acc[v];
        }
    }
}

template <int ND>
__global__ void k_fold_ghosts(GridDev g, StateDev lam)
{
    fold_cells<ND>(g, lam, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

} // namespace hcl::adjoint
