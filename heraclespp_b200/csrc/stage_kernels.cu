// stage_kernels.cu -- one CUDA kernel per Kokkos kernel of the reference's
// time loop, with the reference's FP64 arithmetic (this file is compiled with
// --fmad=false).  These back the stage entry points of the C ABI, which a
// maintainer wires in place of the reference's plugins; they are also the
// stage-by-stage parity path.  Iteration spaces are the reference's Ranges.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "hcl_device.cuh"
#include "physics_exact.cuh"
#include "stages.hpp"

namespace hcl {

std::atomic<int64_t> g_launches{0};

namespace {

constexpr int kThreads = 256;
// The two heaviest stage kernels (Hancock predictor, Godunov update: long FP64
// dependency chains in the reference's order, 130-140 registers unbounded)
// ask for three CTAs per SM; the extra warps hide the chains' latency (KH
// 2048^2 FP64 stage-composed step with one passive scalar 3.81 -> 2.61 ms,
// two CTAs per SM 2.68 ms; the same bits).
constexpr int kHeavyMinBlocks = 3;

struct Box {
    int b[3];
    int w[3];
    int64_t count;
};

Box make_box(const GridDev& g, int ng_eff)
{
    Box bx;
    int e[3];
    cell_range(g, ng_eff, bx.b, e);
    bx.count = 1;
    for (int d = 0; d < 3; ++d) {
        bx.w[d] = e[d] - bx.b[d];
        bx.count *= bx.w[d];
    }
    return bx;
}

__device__ __forceinline__ void box_ijk(const Box& bx, int64_t idx, int& i, int& j, int& k)
{
    i = bx.b[0] + (int)(idx % bx.w[0]);
    const int64_t r = idx / bx.w[0];
    j = bx.b[1] + (int)(r % bx.w[1]);
    k = bx.b[2] + (int)(r / bx.w[1]);
}

int grid_for(int64_t count)
{
    int64_t blocks = (count + kThreads - 1) / kThreads;
    if (blocks > 148 * 16) {
        blocks = 148 * 16;
    }
    if (blocks < 1) {
        blocks = 1;
    }
    return (int)blocks;
}


// ---------------------------------------------------------------------------
// array_conversion.hpp:32-104 "conv_prim_to_cons_array"
template <int ND>
__global__ void k_prim_to_cons(GridDev g, Box bx, const double* __restrict__ rho, const double* __restrict__ u,
                               const double* __restrict__ P, double* __restrict__ rhou, double* __restrict__ E)
{
    const exact::Eos eos = exact::eos_of(g);
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        double p[ND + 2], q[ND + 2];
        p[0] = rho[c];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            p[1 + d] = u[c + g.N * d];
        }
        p[1 + ND] = P[c];
        exact::to_cons<ND>(eos, p, q);
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            rhou[c + g.N * d] = q[1 + d];
        }
        E[c] = q[1 + ND];
    }
}

// array_conversion.hpp:106-172 "conv_cons_to_prim_array"
template <int ND>
__global__ void k_cons_to_prim(GridDev g, Box bx, const double* __restrict__ rho, const double* __restrict__ rhou,
                               const double* __restrict__ E, double* __restrict__ u, double* __restrict__ P)
{
    const exact::Eos eos = exact::eos_of(g);
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        double q[ND + 2], p[ND + 2];
        q[0] = rho[c];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            q[1 + d] = rhou[c + g.N * d];
        }
        q[1 + ND] = E[c];
        exact::to_prim<ND>(eos, q, p);
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            u[c + g.N * d] = p[1 + d];
        }
        P[c] = p[1 + ND];
    }
}

// analysis/temperature.hpp:18-25 "fill_temperature_array"
__global__ void k_temperature(GridDev g, Box bx, const double* __restrict__ rho, const double* __restrict__ P,
                              double* __restrict__ T)
{
    const exact::Eos eos = exact::eos_of(g);
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        T[c] = exact::temperature(eos, rho[c], P[c]);
    }
}

// limited_linear_reconstruction.hpp:46-64 "face_reconstruction":
// var_rec(c, s, idim) = rec[c + N*s + 2N*idim]
template <int ND>
__global__ void k_face_recon(GridDev g, Box bx, const double* __restrict__ var, double* __restrict__ rec)
{
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        const double v = var[c];
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
            const int ki = idim == 0, kj = idim == 1, kk = idim == 2;
            const double dl = (ki * g.dx[0][i]) + (kj * g.dx[1][j]) + (kk * g.dx[2][k]);
            const double dl_m = (ki * g.dx[0][i - ki]) + (kj * g.dx[1][j - kj]) + (kk * g.dx[2][k - kk]);
            const double dl_p = (ki * g.dx[0][i + ki]) + (kj * g.dx[1][j + kj]) + (kk * g.dx[2][k + kk]);
            const double vp = var[lidx(g, i + ki, j + kj, k + kk)];
            const double vm = var[lidx(g, i - ki, j - kj, k - kk)];
            const double slope = exact::slope(g.limiter, (vp - v) / ((dl + dl_p) / 2), (v - vm) / ((dl_m + dl) / 2));
            rec[c + 2 * g.N * idim] = v - ((dl / 2) * slope);
            rec[c + g.N + 2 * g.N * idim] = v + ((dl / 2) * slope);
        }
    }
}

// hydro_reconstruction.hpp:111-126: face primitives -> face conservatives
template <int ND>
__global__ void k_faces_prim_to_cons(GridDev g, Box bx, const double* __restrict__ rho_rec,
                                     const double* __restrict__ u_rec, const double* __restrict__ P_rec,
                                     double* __restrict__ rhou_rec, double* __restrict__ E_rec)
{
    const exact::Eos eos = exact::eos_of(g);
    const int64_t S5 = 2 * g.N;
    const int64_t S6 = 2 * g.N * ND;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int64_t o = c + g.N * s + S5 * idim;
                double p[ND + 2], q[ND + 2];
                p[0] = rho_rec[o];
#pragma unroll
                for (int r = 0; r < ND; ++r) {
                    p[1 + r] = u_rec[o + S6 * r];
                }
                p[1 + ND] = P_rec[o];
                exact::to_cons<ND>(eos, p, q);
#pragma unroll
                for (int r = 0; r < ND; ++r) {
                    rhou_rec[o + S6 * r] = q[1 + r];
                }
                E_rec[o] = q[1 + ND];
            }
        }
    }
}

// extrapolation_reconstruction.hpp:90-325 "Hancock_extrapolation"
template <int ND>
__global__ void __launch_bounds__(kThreads, kHeavyMinBlocks) k_hancock(GridDev g, Box bx, double dt, const double* __restrict__ u_rec,
                          const double* __restrict__ P_rec, double* __restrict__ rho_rec, double* __restrict__ rhou_rec,
                          double* __restrict__ E_rec, double* __restrict__ fx_rec, const double* __restrict__ fx_rec_old)
{
    const exact::Eos eos = exact::eos_of(g);
    const int64_t N = g.N;
    const int64_t S5 = 2 * N;
    const int64_t S6 = 2 * N * ND;
    const int nfx = g.nfx;
    const bool sph = g.geom == GEOM_SPHERICAL;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        double rho_old[2][ND];
        double rhou_old[2][ND][ND];
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
            rho_old[0][idim] = rho_rec[c + S5 * idim];
            rho_old[1][idim] = rho_rec[c + N + S5 * idim];
#pragma unroll
            for (int r = 0; r < ND; ++r) {
                rhou_old[0][idim][r] = rhou_rec[c + S5 * idim + S6 * r];
                rhou_old[1][idim][r] = rhou_rec[c + N + S5 * idim + S6 * r];
            }
            for (int f = 0; f < nfx; ++f) {
                const int64_t of = c + S5 * idim + S6 * f;
                fx_rec[of] *= rho_rec[c + S5 * idim];
                fx_rec[of + N] *= rho_rec[c + N + S5 * idim];
            }
        }
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
            const int64_t cp = lidx(g, i + (idim == 0), j + (idim == 1), k + (idim == 2));
            double pL[ND + 2], pR[ND + 2], fL[ND + 2], fR[ND + 2];
            pL[0] = rho_old[0][idim];
            pR[0] = rho_old[1][idim];
#pragma unroll
            for (int r = 0; r < ND; ++r) {
                pL[1 + r] = u_rec[c + S5 * idim + S6 * r];
                pR[1 + r] = u_rec[c + N + S5 * idim + S6 * r];
            }
            pL[1 + ND] = P_rec[c + S5 * idim];
            pR[1 + ND] = P_rec[c + N + S5 * idim];
            exact::flux_prim<ND>(eos, pL, idim, fL);
            exact::flux_prim<ND>(eos, pR, idim, fR);
            const double dtodv = dt / g.dv[c];
            const double dsc = g.ds[c + N * idim];
            const double dsp = g.ds[cp + N * idim];
#pragma unroll
            for (int ipos = 0; ipos < ND; ++ipos) {
                const int64_t o0 = c + S5 * ipos;
                const int64_t o1 = o0 + N;
                rho_rec[o0] += dtodv * ((fL[0] * dsc) - (fR[0] * dsp));
                rho_rec[o1] += dtodv * ((fL[0] * dsc) - (fR[0] * dsp));
#pragma unroll
                for (int r = 0; r < ND; ++r) {
                    rhou_rec[o0 + S6 * r] += dtodv * ((fL[1 + r] * dsc) - (fR[1 + r] * dsp));
                    rhou_rec[o1 + S6 * r] += dtodv * ((fL[1 + r] * dsc) - (fR[1 + r] * dsp));
                }
                E_rec[o0] += dtodv * ((fL[1 + ND] * dsc) - (fR[1 + ND] * dsp));
                E_rec[o1] += dtodv * ((fL[1 + ND] * dsc) - (fR[1 + ND] * dsp));
            }
            if (sph) {
                // :145-303
                const double PL = pL[1 + ND], PR = pR[1 + ND];
#pragma unroll
                for (int ipos = 0; ipos < ND; ++ipos) {
                    const int64_t o0 = c + S5 * ipos;
                    const int64_t o1 = o0 + N;
                    if (idim == 0) {
                        const double sp = exact::src_grad_pres(dtodv, PL, PR, dsc, dsp);
                        rhou_rec[o0 + S6 * idim] += sp;
                        rhou_rec[o1 + S6 * idim] += sp;
                        if constexpr (ND >= 2) {
                            const double sr = exact::src_grad_u_r(dtodv, pL[0], pR[0], pL[2], pR[2], dsc, dsp);
                            rhou_rec[o0 + S6 * idim] += sr;
                            rhou_rec[o1 + S6 * idim] += sr;
                            const double st = exact::src_grad_u_idir_r(dtodv, g.x[0][i], g.x[0][i + 1], pL[0], pR[0],
                                                                       pL[1], pR[1], pL[2], pR[2], dsc, dsp);
                            rhou_rec[o0 + S6 * 1] -= st;
                            rhou_rec[o1 + S6 * 1] -= st;
                        }
                        if constexpr (ND == 3) {
                            const double sr = exact::src_grad_u_r(dtodv, pL[0], pR[0], pL[3], pR[3], dsc, dsp);
                            rhou_rec[o0 + S6 * idim] += sr;
                            rhou_rec[o1 + S6 * idim] += sr;
                            const double sf = exact::src_grad_u_idir_r(dtodv, g.x[0][i], g.x[0][i + 1], pL[0], pR[0],
                                                                       pL[1], pR[1], pL[3], pR[3], dsc, dsp);
                            rhou_rec[o0 + S6 * 2] -= sf;
                            rhou_rec[o1 + S6 * 2] -= sf;
                        }
                    }
                    if (idim == 1) {
                        const double sp = exact::src_grad_pres(dtodv, PL, PR, dsc, dsp);
                        rhou_rec[o0 + S6 * idim] += sp;
                        rhou_rec[o1 + S6 * idim] += sp;
                        if constexpr (ND == 3) {
                            const double sth = exact::src_grad_u_th(dtodv, g.cot_mid1[j], pL[0], pR[0], pL[3], pR[3], dsc, dsp);
                            rhou_rec[o0 + S6 * idim] += sth;
                            rhou_rec[o1 + S6 * idim] += sth;
                            const double sph2 = exact::src_grad_u_phi(dtodv, g.sin1[j], g.sin1[j + 1], pL[0], pR[0],
                                                                      pL[2], pR[2], pL[3], pR[3], dsc, dsp);
                            rhou_rec[o0 + S6 * 2] -= sph2;
                            rhou_rec[o1 + S6 * 2] -= sph2;
                        }
                    }
                }
            }
            // gravity :306-312
            const double gd = gravity_at(g, i, idim);
#pragma unroll
            for (int ipos = 0; ipos < ND; ++ipos) {
                const int64_t o0 = c + S5 * ipos;
                const int64_t o1 = o0 + N;
                rhou_rec[o0 + S6 * idim] += dt * gd * rho_old[0][ipos];
                rhou_rec[o1 + S6 * idim] += dt * gd * rho_old[1][ipos];
                E_rec[o0] += dt * gd * rhou_old[0][ipos][idim];
                E_rec[o1] += dt * gd * rhou_old[1][ipos][idim];
            }
            // passive scalars :315-337
            for (int f = 0; f < nfx; ++f) {
                const int64_t off = S6 * f;
                const double ffL = fx_rec_old[c + S5 * idim + off] * fL[0];
                const double ffR = fx_rec_old[c + N + S5 * idim + off] * fR[0];
#pragma unroll
                for (int ipos = 0; ipos < ND; ++ipos) {
                    const int64_t o0 = c + S5 * ipos + off;
                    fx_rec[o0] += dtodv * ((ffL * dsc) - (ffR * dsp));
                    fx_rec[o0 + N] += dtodv * ((ffL * dsc) - (ffR * dsp));
                }
            }
        }
    }
}

// extrapolation_reconstruction.hpp:329-339 "passive_scalar_extrapolation"
template <int ND>
__global__ void k_passive_extrap(GridDev g, Box bx, const double* __restrict__ rho_rec, double* __restrict__ fx_rec)
{
    const int64_t N = g.N;
    const int64_t S5 = 2 * N;
    const int64_t S6 = 2 * N * ND;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        for (int idim = 0; idim < ND; ++idim) {
            for (int f = 0; f < g.nfx; ++f) {
                const int64_t o = c + S5 * idim + S6 * f;
                fx_rec[o] /= rho_rec[c + S5 * idim];
                fx_rec[o + N] /= rho_rec[c + N + S5 * idim];
            }
        }
    }
}

// godunov_scheme.hpp:110-292 "Riemann_based_Godunov_scheme"
template <int ND>
__global__ void __launch_bounds__(kThreads, kHeavyMinBlocks) k_godunov(GridDev g, Box bx, double dt, const double* __restrict__ rho, const double* __restrict__ rhou,
                          const double* __restrict__ E, const double* __restrict__ fx,
                          const double* __restrict__ rho_rec, const double* __restrict__ rhou_rec,
                          const double* __restrict__ E_rec, const double* __restrict__ fx_rec,
                          double* __restrict__ rho_new, double* __restrict__ rhou_new, double* __restrict__ E_new,
                          double* __restrict__ fx_new)
{
    const exact::Eos eos = exact::eos_of(g);
    const int64_t N = g.N;
    const int64_t S5 = 2 * N;
    const int64_t S6 = 2 * N * ND;
    const bool sph = g.geom == GEOM_SPHERICAL;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        double rn = rho[c];
        double En = E[c];
        double mn[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            mn[d] = rhou[c + N * d];
        }
        for (int f = 0; f < g.nfx; ++f) {
            fx_new[c + N * f] = fx[c + N * f] * rho[c];
        }
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
            const int64_t cm = lidx(g, i - (idim == 0), j - (idim == 1), k - (idim == 2));
            const int64_t cp = lidx(g, i + (idim == 0), j + (idim == 1), k + (idim == 2));
            double mR[ND + 2], vL[ND + 2], vR[ND + 2], pLn[ND + 2], FL[ND + 2], FR[ND + 2];
            mR[0] = rho_rec[cm + N + S5 * idim];
            vL[0] = rho_rec[c + S5 * idim];
            vR[0] = rho_rec[c + N + S5 * idim];
            pLn[0] = rho_rec[cp + S5 * idim];
#pragma unroll
            for (int r = 0; r < ND; ++r) {
                mR[1 + r] = rhou_rec[cm + N + S5 * idim + S6 * r];
                vL[1 + r] = rhou_rec[c + S5 * idim + S6 * r];
                vR[1 + r] = rhou_rec[c + N + S5 * idim + S6 * r];
                pLn[1 + r] = rhou_rec[cp + S5 * idim + S6 * r];
            }
            mR[1 + ND] = E_rec[cm + N + S5 * idim];
            vL[1 + ND] = E_rec[c + S5 * idim];
            vR[1 + ND] = E_rec[c + N + S5 * idim];
            pLn[1 + ND] = E_rec[cp + S5 * idim];
            exact::riemann<ND>(eos, g.riemann, mR, vL, idim, FL);
            exact::riemann<ND>(eos, g.riemann, vR, pLn, idim, FR);
            const double dtodv = dt / g.dv[c];
            const double dsc = g.ds[c + N * idim];
            const double dsp = g.ds[cp + N * idim];
            rn += dtodv * ((FL[0] * dsc) - (FR[0] * dsp));
#pragma unroll
            for (int r = 0; r < ND; ++r) {
                mn[r] += dtodv * ((FL[1 + r] * dsc) - (FR[1 + r] * dsp));
            }
            En += dtodv * ((FL[1 + ND] * dsc) - (FR[1 + ND] * dsp));
            if (sph) {
                // :165-256
                double pl[ND + 2], pr[ND + 2];
                exact::to_prim<ND>(eos, vL, pl);
                exact::to_prim<ND>(eos, vR, pr);
                if (idim == 0) {
                    mn[0] += exact::src_grad_pres(dtodv, pl[1 + ND], pr[1 + ND], dsc, dsp);
                    if constexpr (ND >= 2) {
                        mn[0] += exact::src_grad_u_r(dtodv, pl[0], pr[0], pl[2], pr[2], dsc, dsp);
                        mn[1] -= exact::src_grad_u_idir_r(dtodv, g.x[0][i], g.x[0][i + 1], pl[0], pr[0], pl[1], pr[1],
                                                          pl[2], pr[2], dsc, dsp);
                    }
                    if constexpr (ND == 3) {
                        mn[0] += exact::src_grad_u_r(dtodv, pl[0], pr[0], pl[3], pr[3], dsc, dsp);
                        mn[2] -= exact::src_grad_u_idir_r(dtodv, g.x[0][i], g.x[0][i + 1], pl[0], pr[0], pl[1], pr[1],
                                                          pl[3], pr[3], dsc, dsp);
                    }
                }
                if constexpr (ND >= 2) {
                    if (idim == 1) {
                        mn[1] += exact::src_grad_pres(dtodv, pl[1 + ND], pr[1 + ND], dsc, dsp);
                        if constexpr (ND == 3) {
                            mn[1] += exact::src_grad_u_th(dtodv, g.cot_mid1[j], pl[0], pr[0], pl[3], pr[3], dsc, dsp);
                            mn[2] -= exact::src_grad_u_phi(dtodv, g.sin1[j], g.sin1[j + 1], pl[0], pr[0], pl[2], pr[2],
                                                           pl[3], pr[3], dsc, dsp);
                        }
                    }
                }
            }
            // gravity :258-260
            const double gd = gravity_at(g, i, idim);
            mn[idim] += dt * gd * rho[c];
            En += dt * gd * rhou[c + N * idim];
            // passive scalars :262-290
            for (int f = 0; f < g.nfx; ++f) {
                const int64_t off = S6 * f;
                int64_t iL = cm, iR = c;
                int64_t sL = 1, sR = 1;
                if (FL[0] < 0) {
                    iL = c;
                    sL = 0;
                }
                if (FR[0] < 0) {
                    iR = cp;
                    sR = 0;
                }
                const double ffL = fx_rec[iL + N * sL + S5 * idim + off] * FL[0];
                const double ffR = fx_rec[iR + N * sR + S5 * idim + off] * FR[0];
                fx_new[c + N * f] += dtodv * ((ffL * dsc) - (ffR * dsp));
            }
        }
        rho_new[c] = rn;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            rhou_new[c + N * d] = mn[d];
        }
        E_new[c] = En;
    }
}

// pressure_fix.hpp:19-172: where the old internal energy is below eps times
// the kinetic energy, E_new is rebuilt from a blend of the Godunov increment
// and a pressure-work estimate from the face velocities (the reference's loop
// order, including the overwrite of E_new inside the inner loop)
template <int ND>
__global__ void k_pressure_fix(GridDev g, Box bx, double dt, double eps, const double* __restrict__ rho,
                               const double* __restrict__ rhou, const double* __restrict__ E,
                               const double* __restrict__ rho_rec, const double* __restrict__ rhou_rec,
                               const double* __restrict__ E_rec, const double* __restrict__ rho_new,
                               const double* __restrict__ rhou_new, double* __restrict__ E_new)
{
    const exact::Eos eos = exact::eos_of(g);
    const int64_t N = g.N;
    const int64_t S5 = 2 * N;
    const int64_t S6 = 2 * N * ND;
    const double eps2 = eps / 10;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        double cons[ND + 2], cons_new[ND + 2], prim[ND + 2];
        cons[0] = rho[c];
        cons_new[0] = rho_new[c];
#pragma unroll
        for (int r = 0; r < ND; ++r) {
            cons[1 + r] = rhou[c + N * r];
            cons_new[1 + r] = rhou_new[c + N * r];
        }
        cons[1 + ND] = E[c];
        cons_new[1 + ND] = E_new[c];
        exact::to_prim<ND>(eos, cons, prim);
        const double ekin = exact::ek_cons<ND>(cons);
        const double evol = E[c] - ekin;
        const double evol_new = E_new[c] - exact::ek_cons<ND>(cons_new);
        const double de_god = evol_new - evol;
        if (!(evol < eps * ekin)) {
            continue;
        }
        double En = E[c];
        double divU = 0;
        double divUE = 0;
        double einL = 0;
        double einR = 0;
        double alpha = (evol * evol) / (ekin * ekin * eps * eps);
        if (evol < eps2 * ekin) {
            alpha = 0;
        }
        for (int idim = 0; idim < ND; ++idim) {
            const int64_t cm = lidx(g, i - (idim == 0), j - (idim == 1), k - (idim == 2));
            const int64_t cp = lidx(g, i + (idim == 0), j + (idim == 1), k + (idim == 2));
            for (int ipos = 0; ipos < ND; ++ipos) {
                double vL[ND + 2], vR[ND + 2], mR[ND + 2], pL[ND + 2], cons_p[ND + 2], cons_m[ND + 2];
                double primL[ND + 2], primR[ND + 2], prim_mR[ND + 2], prim_pL[ND + 2];
                vL[0] = rho_rec[c + S5 * idim];
                vR[0] = rho_rec[c + N + S5 * idim];
                mR[0] = rho_rec[cm + N + S5 * idim];
                pL[0] = rho_rec[cp + S5 * idim];
                cons_p[0] = rho[cp];
                cons_m[0] = rho[cm];
#pragma unroll
                for (int r = 0; r < ND; ++r) {
                    vL[1 + r] = rhou_rec[c + S5 * idim + S6 * r];
                    vR[1 + r] = rhou_rec[c + N + S5 * idim + S6 * r];
                    mR[1 + r] = rhou_rec[cm + N + S5 * idim + S6 * r];
                    pL[1 + r] = rhou_rec[cp + S5 * idim + S6 * r];
                    cons_p[1 + r] = rhou[cp + N * r];
                    cons_m[1 + r] = rhou[cm + N * r];
                }
                vL[1 + ND] = E_rec[c + S5 * idim];
                vR[1 + ND] = E_rec[c + N + S5 * idim];
                mR[1 + ND] = E_rec[cm + N + S5 * idim];
                pL[1 + ND] = E_rec[cp + S5 * idim];
                cons_p[1 + ND] = E[cp];
                cons_m[1 + ND] = E[cm];
                exact::to_prim<ND>(eos, vL, primL);
                exact::to_prim<ND>(eos, vR, primR);
                exact::to_prim<ND>(eos, mR, prim_mR);
                exact::to_prim<ND>(eos, pL, prim_pL);
                const double us = (prim_mR[1 + ipos] + primL[1 + ipos]) / 2;
                const double us_p = (primR[1 + ipos] + prim_pL[1 + ipos]) / 2;
                divU += ((us_p * g.ds[cp + N * ipos]) - (us * g.ds[c + N * ipos])) / g.dv[c];
                if (us_p > 0) {
                    einR = E[c] - exact::ek_cons<ND>(cons);
                } else {
                    einR = E[cp] - exact::ek_cons<ND>(cons_p);
                }
                if (us < 0) {
                    einL = E[c] - exact::ek_cons<ND>(cons);
                } else {
                    einL = E[cm] - exact::ek_cons<ND>(cons_m);
                }
                divUE += ((us_p * einR * g.ds[cp + N * ipos]) - (us * einL * g.ds[c + N * ipos])) / g.dv[c];
                const double de_pf = dt * ((-prim[1 + ND] * divU) - divUE);
                double sum = 0;
#pragma unroll
                for (int idr = 0; idr < ND; ++idr) {
                    sum += cons[1 + idr] * cons[1 + idr] / cons[0];
                }
                const double de_tot = (alpha * de_god) + ((1 - alpha) * de_pf);
                En = evol + de_tot + (1. / 2 * sum);
            }
        }
        E_new[c] = En;
    }
}

// godunov_scheme.hpp:294-301 "passive_scalar_Godunov"
__global__ void k_passive_godunov(GridDev g, Box bx, const double* __restrict__ rho_new, double* __restrict__ fx_new)
{
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        for (int f = 0; f < g.nfx; ++f) {
            const double v = fx_new[c + g.N * f] / rho_new[c];
            fx_new[c + g.N * f] = v < 0. ? 0. : (v > 1. ? 1. : v);
        }
    }
}

// boundary_distribute.hpp:42-76 on one rank, as a gather (see bc_source)
template <int ND>
__global__ void k_fill_ghosts(GridDev g, double* __restrict__ rho, double* __restrict__ rhou, double* __restrict__ E,
                              double* __restrict__ fx)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g.N; c += (int64_t)gridDim.x * blockDim.x) {
        int idx[3];
        idx[0] = (int)(c % g.n[0]);
        const int64_t r = c / g.n[0];
        idx[1] = (int)(r % g.n[1]);
        idx[2] = (int)(r / g.n[1]);
        int src[3] = {idx[0], idx[1], idx[2]};
        int flip[3] = {0, 0, 0};
        bool ghost = false;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            src[d] = bc_source(idx[d], g.n[d], g.ng, g.bc[2 * d], g.bc[2 * d + 1], &flip[d]);
            ghost |= src[d] != idx[d];
        }
        if (!ghost) {
            continue;
        }
        const int64_t s = lidx(g, src[0], src[1], src[2]);
        rho[c] = rho[s];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const double v = rhou[s + g.N * d];
            rhou[c + g.N * d] = flip[d] ? -v : v;
        }
        E[c] = E[s];
        for (int f = 0; f < g.nfx; ++f) {
            fx[c + g.N * f] = fx[s + g.N * f];
        }
    }
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// time_step.hpp:55-77 "time_step" (Max reducer): per-cell sum_d (|u_d|+c)/dx_geom_d
template <int ND>
__global__ void k_time_step(GridDev g, Box bx, const double* __restrict__ rho, const double* __restrict__ u,
                            const double* __restrict__ P, unsigned long long* inv_bits)
{
    const exact::Eos eos = exact::eos_of(g);
    double local = 0;
    bool has_nan = false;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        const double sound = exact::sound(eos, rho[c], P[c]);
        double dxg[3] = {g.dx[0][i], g.dx[1][j], g.dx[2][k]};
        if (g.geom == GEOM_SPHERICAL) {
            if (ND == 2) {
                dxg[1] *= g.xc[0][i];
            }
            if (ND == 3) {
                dxg[1] *= g.xc[0][i];
                dxg[2] *= g.xc[0][i] * g.sin_xc1[j];
            }
        }
        double cell = 0;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            cell += (fabs(u[c + g.N * d]) + sound) / dxg[d];
        }
        has_nan |= isnan(cell);
        local = local > cell ? local : cell;
    }
    local = warp_max(local);
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[w] = local;
    }
    __syncthreads();
    if (w == 0) {
        local = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        local = warp_max(local);
        if (lane == 0) {
            atomicMax(inv_bits, dbl_bits(local));
        }
    }
    if (has_nan) {
        atomicMax(inv_bits, 0x7ff8000000000000ull);
    }
}

// ordered key for doubles of any sign: monotone under unsigned compare
__device__ __forceinline__ unsigned long long min_key(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// internal_energy.cpp:25-42 "min_internal_energy" over no_ghosts
template <int ND>
__global__ void k_min_evol(GridDev g, Box bx, const double* __restrict__ rho, const double* __restrict__ rhou,
                           const double* __restrict__ E, unsigned long long* key, int* nan_flag)
{
    unsigned long long local = ~0ull;
    bool has_nan = false;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        double q[ND + 2];
        q[0] = rho[c];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            q[1 + d] = rhou[c + g.N * d];
        }
        q[1 + ND] = E[c];
        const double ev = q[1 + ND] - exact::ek_cons<ND>(q);
        if (isnan(ev)) {
            has_nan = true;
        } else {
            const unsigned long long kk = min_key(ev);
            local = kk < local ? kk : local;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, local, o);
        local = other < local ? other : local;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(key, local);
    }
    if (has_nan) {
        atomicOr(nan_flag, 1);
    }
}

// Compensated (TwoSum) partial sums of var*dv, one pair per block.
__device__ __forceinline__ void two_sum_acc(double& s, double& e, double v)
{
    const double t = s + v;
    const double bp = t - s;
    e += (s - (t - bp)) + (v - bp);
    s = t;
}

constexpr int kRedBlocks = 296;

__global__ void k_integrate_partial(GridDev g, Box bx, const double* __restrict__ var, double* partials)
{
    double s = 0, e = 0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < bx.count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        box_ijk(bx, idx, i, j, k);
        const int64_t c = lidx(g, i, j, k);
        two_sum_acc(s, e, var[c] * g.dv[c]);
    }
    __shared__ double ss[kThreads], se[kThreads];
    ss[threadIdx.x] = s;
    se[threadIdx.x] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0, Ecomp = 0;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            two_sum_acc(S, Ecomp, ss[t]);
            Ecomp += se[t];
        }
        partials[2 * blockIdx.x] = S;
        partials[2 * blockIdx.x + 1] = Ecomp;
    }
}

__global__ void k_integrate_final(const double* partials, int nblocks, double* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double S = 0, Ecomp = 0;
        for (int b = 0; b < nblocks; ++b) {
            two_sum_acc(S, Ecomp, partials[2 * b]);
            Ecomp += partials[2 * b + 1];
        }
        out[0] = S + Ecomp;
        out[1] = Ecomp;
    }
}

template <class F>
void dispatch_nd(int nd, F&& f)
{
    if (nd == 1) {
        f(std::integral_constant<int, 1>{});
    } else if (nd == 2) {
        f(std::integral_constant<int, 2>{});
    } else {
        f(std::integral_constant<int, 3>{});
    }
}

// InternalMassGravity (gravity.cpp:59-128), one CTA: each thread sums the
// density of one radial shell over the interior (j, k) (j outer, k inner),
// thread 0 runs the enclosed-mass sum outwards from the central mass, then
// every thread turns its cells' enclosed mass into g = -G M / xc^2.  rho has
// rows of `pitch` doubles (n0 for the reference layout); shell: nx0 + ng
// doubles of scratch; g_r: n0 doubles (the handle's radial table).
__global__ void k_internal_mass_gravity(GridDev g, const double* __restrict__ rho, int pitch, double central_mass,
                                        double* __restrict__ shell, double* __restrict__ g_r)
{
    const int ng = g.ng;
    const int nsh = g.nx[0] + ng;
    const int g1 = g.ndim >= 2 ? ng : 0;
    const int g2 = g.ndim >= 3 ? ng : 0;
    for (int i = threadIdx.x; i < nsh; i += blockDim.x) {
        double sm = 0;
        double sd = 0;
        for (int j = 0; j < g.nx[1]; ++j) {
            for (int k = 0; k < g.nx[2]; ++k) {
                const int64_t id = lidx(g, i + ng, j + g1, k + g2);
                const int64_t ir = ((int64_t)(k + g2) * g.n[1] + (j + g1)) * pitch + (i + ng);
                sm += rho[ir] * g.dv[id];
                sd += g.dv[id];
            }
        }
        shell[i] = sm / sd;
    }
    __syncthreads();
    const double* x0 = g.x[0];
    const double* xc = g.xc[0];
    if (threadIdx.x == 0) {
        const double vol_s3 = 4 * kPi / 3;
        for (int i = 0; i < ng; ++i) {
            g_r[i] = central_mass;
        }
        double partial = 0;
        for (int i = ng; i < g.nx[0] + 2 * ng; ++i) {
            const int off = i - ng;
            const double x3 = x0[i] * x0[i] * x0[i];
            if (i == ng) {
                partial += central_mass + (vol_s3 * ((xc[i] * xc[i] * xc[i]) - x3) * shell[off]);
            } else {
                partial += (vol_s3 * (x3 - (xc[i - 1] * xc[i - 1] * xc[i - 1])) * shell[off - 1]) +
                           (vol_s3 * ((xc[i] * xc[i] * xc[i]) - x3) * shell[off]);
            }
            g_r[i] = partial;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < g.n[0]; i += blockDim.x) {
        g_r[i] = -kG * g_r[i] / (xc[i] * xc[i]);
    }
}

} // namespace

namespace stage {

void conv_prim_to_cons(const GridDev& g, int ng_eff, const double* rho, const double* u, const double* P,
                       double* rhou, double* E, cudaStream_t s)
{
    const Box bx = make_box(g, ng_eff);
    dispatch_nd(g.ndim, [&](auto nd) {
        k_prim_to_cons<decltype(nd)::value><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho, u, P, rhou, E);
    });
    ++g_launches;
}

void conv_cons_to_prim(const GridDev& g, int ng_eff, const double* rho, const double* rhou, const double* E,
                       double* u, double* P, cudaStream_t s)
{
    const Box bx = make_box(g, ng_eff);
    dispatch_nd(g.ndim, [&](auto nd) {
        k_cons_to_prim<decltype(nd)::value><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho, rhou, E, u, P);
    });
    ++g_launches;
}

void temperature(const GridDev& g, int ng_eff, const double* rho, const double* P, double* T, cudaStream_t s)
{
    const Box bx = make_box(g, ng_eff);
    k_temperature<<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho, P, T);
    ++g_launches;
}

void face_reconstruction(const GridDev& g, int ng_eff, const double* var, double* var_rec, cudaStream_t s)
{
    const Box bx = make_box(g, ng_eff);
    dispatch_nd(g.ndim, [&](auto nd) {
        k_face_recon<decltype(nd)::value><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, var, var_rec);
    });
    ++g_launches;
}

void hydro_reconstruction(const GridDev& g, int ng_eff, double dt, const double* rho, const double* u,
                          const double* P, const double* fx, double* rho_rec, double* rhou_rec, double* E_rec,
                          double* fx_rec, double* u_rec, double* P_rec, double* fx_rec_old, cudaStream_t s)
{
    const int nd = g.ndim;
    const int64_t N = g.N;
    // hydro_reconstruction.hpp:99-109
    face_reconstruction(g, ng_eff, rho, rho_rec, s);
    for (int d = 0; d < nd; ++d) {
        face_reconstruction(g, ng_eff, u + N * d, u_rec + 2 * N * nd * d, s);
    }
    face_reconstruction(g, ng_eff, P, P_rec, s);
    for (int f = 0; f < g.nfx; ++f) {
        face_reconstruction(g, ng_eff, fx + N * f, fx_rec + 2 * N * nd * f, s);
    }
    const Box bx = make_box(g, ng_eff);
    dispatch_nd(nd, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        k_faces_prim_to_cons<ND><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho_rec, u_rec, P_rec, rhou_rec, E_rec);
    });
    ++g_launches;
    // extrapolation_reconstruction.hpp:87-88
    if (g.nfx > 0) {
        cudaMemcpyAsync(fx_rec_old, fx_rec, sizeof(double) * (size_t)(2 * N * nd * g.nfx), cudaMemcpyDeviceToDevice, s);
    }
    dispatch_nd(nd, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        k_hancock<ND><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, dt, u_rec, P_rec, rho_rec, rhou_rec, E_rec, fx_rec,
                                                              fx_rec_old);
        if (g.nfx > 0) {
            k_passive_extrap<ND><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho_rec, fx_rec);
        }
    });
    g_launches += g.nfx > 0 ? 2 : 1;
}

void godunov(const GridDev& g, int ng_eff, double dt, const double* rho, const double* rhou, const double* E,
             const double* fx, const double* rho_rec, const double* rhou_rec, const double* E_rec,
             const double* fx_rec, double* rho_new, double* rhou_new, double* E_new, double* fx_new,
             cudaStream_t s)
{
    const Box bx = make_box(g, ng_eff);
    dispatch_nd(g.ndim, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        k_godunov<ND><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, dt, rho, rhou, E, fx, rho_rec, rhou_rec, E_rec,
                                                              fx_rec, rho_new, rhou_new, E_new, fx_new);
    });
    ++g_launches;
    if (g.nfx > 0) {
        k_passive_godunov<<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho_new, fx_new);
        ++g_launches;
    }
}

void pressure_fix(const GridDev& g, double dt, double eps, const double* rho, const double* rhou, const double* E,
                  const double* rho_rec, const double* rhou_rec, const double* E_rec, const double* rho_new,
                  const double* rhou_new, double* E_new, cudaStream_t s)
{
    const Box bx = make_box(g, 0);
    dispatch_nd(g.ndim, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        k_pressure_fix<ND><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, dt, eps, rho, rhou, E, rho_rec, rhou_rec,
                                                                   E_rec, rho_new, rhou_new, E_new);
    });
    ++g_launches;
}

void internal_mass_gravity(const GridDev& g, const double* rho, int pitch, double central_mass, double* shell,
                           double* g_r, cudaStream_t s)
{
    k_internal_mass_gravity<<<1, 256, 0, s>>>(g, rho, pitch, central_mass, shell, g_r);
    ++g_launches;
}

void boundaries(const GridDev& g, double* rho, double* rhou, double* E, double* fx, cudaStream_t s)
{
    dispatch_nd(g.ndim, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        k_fill_ghosts<ND><<<grid_for(g.N), kThreads, 0, s>>>(g, rho, rhou, E, fx);
    });
    ++g_launches;
}

void time_step_inv(const GridDev& g, int ng_eff, const double* rho, const double* u, const double* P,
                   unsigned long long* inv_bits, cudaStream_t s)
{
    const Box bx = make_box(g, ng_eff);
    dispatch_nd(g.ndim, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        k_time_step<ND><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho, u, P, inv_bits);
    });
    ++g_launches;
}

void min_internal_energy(const GridDev& g, const double* rho, const double* rhou, const double* E,
                         unsigned long long* key, int* nan_flag, cudaStream_t s)
{
    const Box bx = make_box(g, 0);
    dispatch_nd(g.ndim, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        k_min_evol<ND><<<grid_for(bx.count), kThreads, 0, s>>>(g, bx, rho, rhou, E, key, nan_flag);
    });
    ++g_launches;
}

double decode_min_key(unsigned long long key)
{
    const unsigned long long b = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
    double v;
    static_assert(sizeof(v) == sizeof(b));
    __builtin_memcpy(&v, &b, sizeof(v));
    return v;
}

int integrate_blocks()
{
    return kRedBlocks;
}

void integrate(const GridDev& g, const double* var, double* partials, double* out, cudaStream_t s)
{
    const Box bx = make_box(g, 0);
    k_integrate_partial<<<kRedBlocks, kThreads, 0, s>>>(g, bx, var, partials);
    k_integrate_final<<<1, 32, 0, s>>>(partials, kRedBlocks, out);
    g_launches += 2;
}

} // namespace stage
} // namespace hcl
