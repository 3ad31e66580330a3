// fused_step.cuh -- the fused MUSCL-Hancock step (one kernel per time step).
//
// One CTA owns a tile of T0 x T1 x T2 interior cells.  In one pass it
//   1. stages the FP64 conservative state of the tile plus a 2-cell halo from
//      HBM and converts it to primitives in shared memory,
//   2. computes limited slopes, face primitives, face conservatives and the
//      Hancock half-step predictor for every cell whose faces the tile needs
//      (hydro_reconstruction.hpp:85-129, extrapolation_reconstruction.hpp),
//   3. solves each face's Riemann problem once (the reference solves every
//      face twice, once from each side, godunov_scheme.hpp:141,155),
//   4. applies the Godunov update with geometric and gravity sources
//      (godunov_scheme.hpp:159-260), writes the new state with one FP64 store
//      per variable, writes the ghost-cell images of border cells in place
//      (boundary_distribute.hpp:42-76), checks the internal energy
//      (main.cpp:397-425) and reduces the CFL 1/dt of the new state
//      (time_step.hpp:55-77) by warp shuffles and one atomic per CTA.
// The time-loop control of main.cpp:354-385 (dt from the previous step's
// reduction, output-time and t_end clamps, max_iter) is evaluated by every
// CTA from a small control block, so a chunk of steps replays from a CUDA
// graph without host round trips.
//
// EXACT = true: FP64 with the reference's operation order (built with
// --fmad=false), bitwise-comparable to the reference's FP64 CPU build.
// EXACT = false: the mixed form -- FP32 primitives, slopes, faces, fluxes;
// FP64 state, internal-energy recovery, update accumulation, dt.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <type_traits>

#include "hcl_device.cuh"
#include "per_device.hpp"
#include "physics_exact.cuh"
#include "physics_fast.cuh"
#include "stages.hpp"
#include "tma_ring.cuh"

namespace hcl::fused {

template <int ND, int TX, int TY, int TZ>
struct Shape {
    static constexpr int NV = ND + 2;
    static constexpr int T0 = TX;
    static constexpr int T1 = ND >= 2 ? TY : 1;
    static constexpr int T2 = ND >= 3 ? TZ : 1;
    static constexpr int L0 = T0 + 4;
    static constexpr int L1 = ND >= 2 ? T1 + 4 : 1;
    static constexpr int L2 = ND >= 3 ? T2 + 4 : 1;
    static constexpr int NP = L0 * L1 * L2;
    static constexpr int TVOL = T0 * T1 * T2;
    __host__ __device__ static constexpr int T(int d) { return d == 0 ? T0 : (d == 1 ? T1 : T2); }
    // A_d: cells whose d-faces are needed: T_d + 2 along d, T_e along e != d
    __host__ __device__ static constexpr int Adim(int d, int e) { return e == d ? T(e) + 2 : T(e); }
    __host__ __device__ static constexpr int Asize(int d) { return Adim(d, 0) * Adim(d, 1) * Adim(d, 2); }
    // F_d: faces normal to d
    __host__ __device__ static constexpr int Fdim(int d, int e) { return e == d ? T(e) + 1 : T(e); }
    __host__ __device__ static constexpr int Fsize(int d) { return Fdim(d, 0) * Fdim(d, 1) * Fdim(d, 2); }
    __host__ __device__ static constexpr int Aoff(int d)
    {
        int o = 0;
        for (int e = 0; e < d; ++e) {
            o += 2 * NV * Asize(e);
        }
        return o;
    }
    __host__ __device__ static constexpr int Foff(int d)
    {
        int o = 0;
        for (int e = 0; e < d; ++e) {
            o += NV * Fsize(e);
        }
        return o;
    }
    static constexpr int A_TOTAL = Aoff(ND);
    static constexpr int F_TOTAL = Foff(ND);
    static constexpr int HCOUNT = TVOL + (ND >= 1 ? 2 * TVOL / T0 : 0) + (ND >= 2 ? 2 * TVOL / T1 : 0) +
                                  (ND >= 3 ? 2 * TVOL / T2 : 0);
};

template <class R>
__host__ __device__ constexpr size_t smem_bytes_for(int np, int a_total, int f_total, int nv)
{
    return sizeof(R) * ((size_t)nv * np + (size_t)a_total + (size_t)f_total);
}

// ---------------------------------------------------------------------------
// time-loop control (main.cpp:354-385), evaluated identically by every thread
struct Decision {
    double dt;
    double t;
    int iter;
    int noop;
    int stop;
    int neg_dt;
    int toid_next;
    int ioid_next;
};

__device__ __forceinline__ Decision decide(const StepCtl* ctl, int slot, const RunParamsDev& rp)
{
    Decision d;
    const int p = slot & 1;
    d.t = ctl->t[p];
    d.iter = ctl->iter[p];
    d.noop = ctl->stop[p] || ctl->errflag[p];
    d.stop = 0;
    d.neg_dt = 0;
    d.toid_next = ctl->time_output_id[p];
    d.ioid_next = ctl->iter_output_id[p];
    d.dt = 0;
    if (d.noop) {
        return d;
    }
    double dt;
    if (rp.fixed_dt == 1) {
        dt = rp.dts[d.iter];
    } else if (rp.fixed_dt == 2) {
        dt = rp.dt_value;
    } else {
        const double inv = __longlong_as_double((long long)ctl->inv_dt_bits[slot % 3]);
        dt = rp.cfl * (1 / inv); // main.cpp:355, time_step.hpp:82
    }
    if (rp.iter_frequency > 0) { // main.cpp:358-364
        const int next_output = (d.ioid_next + 1) * rp.iter_frequency;
        if ((d.iter + 1) >= next_output) {
            ++d.ioid_next;
        }
    }
    if (rp.time_frequency > 0) { // main.cpp:365-375
        const double next_output = rp.time_first_output + ((d.toid_next + 1) * rp.time_frequency);
        if ((d.t + dt) >= next_output) {
            dt = next_output - d.t;
            if (dt <= 0) {
                d.neg_dt = 1;
            }
            ++d.toid_next;
        }
    }
    if ((d.t + dt) >= rp.t_end) { // main.cpp:377-381
        dt = rp.t_end - d.t;
        d.stop = 1;
    }
    if ((d.iter + 1) >= rp.max_iter) { // main.cpp:382-385
        d.stop = 1;
    }
    d.dt = dt;
    return d;
}

__device__ __forceinline__ int64_t sidx(const StateDev& st, int n1, int i, int j, int k)
{
    return (int64_t)i + (int64_t)st.pitch * ((int64_t)j + (int64_t)n1 * (int64_t)k);
}

__device__ __forceinline__ double warp_max_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// Ghost images of interior index l along one dim: positions p != l with
// bc_source(p) == l.  Returns the count written to pos/flip (<= 2*ng).
__device__ __forceinline__ int ghost_images(int l, int n, int ng, int bcl, int bcr, int* pos, int* flip)
{
    int cnt = 0;
    if (l >= 2 * ng && l < n - 2 * ng) {
        // far from both faces: no image under any boundary type
        return 0;
    }
    for (int p = 0; p < ng; ++p) {
        int f;
        if (bc_source(p, n, ng, bcl, bcr, &f) == l) {
            pos[cnt] = p;
            flip[cnt] = f;
            ++cnt;
        }
    }
    for (int p = n - ng; p < n; ++p) {
        int f;
        if (bc_source(p, n, ng, bcl, bcr, &f) == l) {
            pos[cnt] = p;
            flip[cnt] = f;
            ++cnt;
        }
    }
    return cnt;
}

// The same images as a mask over the 2*ng ghost slots of a dimension (slot
// k < ng: cell k; slot k >= ng: cell n - 2ng + k): bit k is set when slot k
// takes its value from cell l, bit 16 + k when that image has its normal
// momentum negated (Nghost <= 4, so 2*ng <= 8 slots).
__device__ __forceinline__ unsigned ghost_mask(int l, int n, int ng, int bcl, int bcr)
{
    if (l >= 2 * ng && l < n - 2 * ng) {
        return 0u;
    }
    unsigned m = 0u;
    for (int k = 0; k < 2 * ng; ++k) {
        const int p = k < ng ? k : n - 2 * ng + k;
        int f;
        if (bc_source(p, n, ng, bcl, bcr, &f) == l) {
            m |= (1u << k) | ((unsigned)f << (16 + k));
        }
    }
    return m;
}

__device__ __forceinline__ int ghost_slot(int k, int n, int ng)
{
    return k < ng ? k : n - 2 * ng + k;
}

// Writes a 2-D cell's new state to its ghost images: every (x image or the
// cell's own column) x (y image or its own row) pair except the cell itself.
// xm, ym: ghost_mask of the column and the row.
__device__ __forceinline__ void store_images_2d(double* __restrict__ q, int64_t plane, int pitch, int n0, int n1,
                                                int ng, int col, int r, unsigned xm, unsigned ym, const double qn[4])
{
    unsigned yb = ym & 0xffffu;
    int py = r, fy = 0;
    bool self_y = true;
    for (;;) {
        unsigned xb = xm & 0xffffu;
        int px = col, fx = 0;
        bool self_x = true;
        for (;;) {
            if (!(self_x && self_y)) {
                const int64_t og = (int64_t)py * pitch + px;
                q[og] = qn[0];
                q[og + plane] = fx ? -qn[1] : qn[1];
                q[og + 2 * plane] = fy ? -qn[2] : qn[2];
                q[og + 3 * plane] = qn[3];
            }
            if (xb == 0u) {
                break;
            }
            const int k = __ffs(xb) - 1;
            xb &= xb - 1u;
            px = ghost_slot(k, n0, ng);
            fx = (xm >> (16 + k)) & 1u;
            self_x = false;
        }
        if (yb == 0u) {
            break;
        }
        const int k = __ffs(yb) - 1;
        yb &= yb - 1u;
        py = ghost_slot(k, n1, ng);
        fy = (ym >> (16 + k)) & 1u;
        self_y = false;
    }
}

// 3-D form: every (x image or own column) x (y image or own row) x (z image
// or own plane) triple except the cell itself.
__device__ __forceinline__ void store_images_3d(double* __restrict__ q, int64_t plane, int pitch, int n0, int n1,
                                                int n2, int ng, int col, int row, int z, unsigned xm, unsigned ym,
                                                unsigned zm, const double qn[5])
{
    unsigned zb = zm & 0xffffu;
    int pz = z, fz = 0;
    bool self_z = true;
    for (;;) {
        unsigned yb = ym & 0xffffu;
        int py = row, fy = 0;
        bool self_y = true;
        for (;;) {
            unsigned xb = xm & 0xffffu;
            int px = col, fx = 0;
            bool self_x = true;
            for (;;) {
                if (!(self_x && self_y && self_z)) {
                    const int64_t og = ((int64_t)pz * n1 + py) * pitch + px;
                    q[og] = qn[0];
                    q[og + plane] = fx ? -qn[1] : qn[1];
                    q[og + 2 * plane] = fy ? -qn[2] : qn[2];
                    q[og + 3 * plane] = fz ? -qn[3] : qn[3];
                    q[og + 4 * plane] = qn[4];
                }
                if (xb == 0u) {
                    break;
                }
                const int k = __ffs(xb) - 1;
                xb &= xb - 1u;
                px = ghost_slot(k, n0, ng);
                fx = (xm >> (16 + k)) & 1u;
                self_x = false;
            }
            if (yb == 0u) {
                break;
            }
            const int k = __ffs(yb) - 1;
            yb &= yb - 1u;
            py = ghost_slot(k, n1, ng);
            fy = (ym >> (16 + k)) & 1u;
            self_y = false;
        }
        if (zb == 0u) {
            break;
        }
        const int k = __ffs(zb) - 1;
        zb &= zb - 1u;
        pz = ghost_slot(k, n2, ng);
        fz = (zm >> (16 + k)) & 1u;
        self_z = false;
    }
}

// ---------------------------------------------------------------------------
// EOSK: the EOS as a compile-time constant (EOS_PERFECT_GAS or EOS_RAD_GAS;
// the FP32-mixed variant is perfect gas only), so that the FP64 physics
// carries no run-time EOS branch.
// Occupancy: the tiles' phases wait at barriers and on dependency chains, and
// more resident CTAs fill those waits.  Where the shared memory of a launch
// leaves room for them (no passive scalars), the 2-D FP64 tile runs three CTAs
// per SM (80 registers, some spilled; KH 2048^2: 1.19 -> 1.02 ms per step;
// 16x8 tiles at five CTAs per SM: 1.15 ms).  The other tiles (0 here) keep
// the compiler's register choice, which already gives the FP32-mixed 2-D
// 256-thread tiles three CTAs per SM and the 3-D tile two (asking for a
// minimum of one block instead lets it take more registers: RT 256^2 x 512
// with a passive scalar 8.8 -> 14.3 ms).
template <int ND, bool EXACT, int TX, int TY, int TZ>
constexpr int fused_min_blocks()
{
    return (EXACT && ND == 2) ? 3 : 0;
}

// tma (2-D and 3-D): the FP64 tile plus its halo arrives as one tensor box
// ({L0, L1, L2, NV} of `tmap`, the input state's hydro planes) issued by one
// thread into the face buffer, which phase 2 overwrites only after phase 1
// has read it; otherwise every thread loads its cells directly.
template <int ND, bool EXACT, int TX, int TY, int TZ, int EOSK>
__device__ __forceinline__ void fused_step_body(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl,
                                                const RunParamsDev& rp, int slot, int out_buf,
                                                const CUtensorMap* tmap = nullptr, int tma = 0)
{
    using S = Shape<ND, TX, TY, TZ>;
    using R = std::conditional_t<EXACT, double, float>;
    constexpr int NV = S::NV;
    constexpr int NT = S::TVOL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sp = reinterpret_cast<R*>(smem_raw);     // [NV][NP] primitives
    R* sa = sp + NV * S::NP;                    // faces: per d [2][NV][A_d]
    R* sf = sa + S::A_TOTAL;                    // fluxes: per d [NV][F_d]
    R* sx = sf + S::F_TOTAL;                    // passive scalars: [nfx][NP] primitives, then
                                                // face values per d [2][nfx][A_d]
    const int nfx = g.nfx;
    auto sxa = [&](int d) { return sx + nfx * (S::NP + 2 * (S::Aoff(d) / (2 * NV))); };

    const int tid = threadIdx.x;
    const Decision dec = decide(ctl, slot, rp);
    if (blockIdx.x == 0 && tid == 0) {
        // publish the state seen by step slot+1 (slots other than the ones read)
        const int q = (slot + 1) & 1;
        if (!dec.noop) {
            ctl->t[q] = dec.t + dec.dt; // main.cpp:530
            ctl->iter[q] = dec.iter + 1;
            ctl->time_output_id[q] = dec.toid_next;
            ctl->iter_output_id[q] = dec.ioid_next;
            ctl->stop[q] = dec.stop;
            ctl->last_dt = dec.dt;
            if (dec.stop) {
                ctl->final_buf = out_buf;
            }
            if (dec.neg_dt) {
                ctl->err = 5; // HCL_ERR_NEGATIVE_DT, main.cpp:368-371
                ctl->errflag[q] = 1;
                ctl->t[q] = dec.t;
                ctl->iter[q] = dec.iter;
                ctl->final_buf = out_buf ^ 1;
            }
            if (rp.dt_log && dec.iter < rp.dt_log_cap && !dec.neg_dt) {
                rp.dt_log[dec.iter] = dec.dt;
            }
        } else {
            ctl->t[q] = dec.t;
            ctl->iter[q] = dec.iter;
            ctl->time_output_id[q] = dec.toid_next;
            ctl->iter_output_id[q] = dec.ioid_next;
            ctl->stop[q] = 1;
            ctl->errflag[q] = ctl->errflag[slot & 1];
        }
        ctl->inv_dt_bits[(slot + 2) % 3] = 0ull;
    }
    if (dec.noop || dec.neg_dt) {
        return;
    }
    const double dt = dec.dt;
    const double dth = dt / 2; // main.cpp:431

    // tile origin (tile-local interior cell (0,0,0) at global (gi0, gj0, gk0))
    int ntile[3], tc[3];
    ntile[0] = (g.nx[0] + S::T0 - 1) / S::T0;
    ntile[1] = (g.nx[1] + S::T1 - 1) / S::T1;
    {
        int b = blockIdx.x;
        tc[0] = b % ntile[0];
        b /= ntile[0];
        tc[1] = b % ntile[1];
        tc[2] = b / ntile[1];
    }
    const int t0[3] = {tc[0] * S::T0, tc[1] * S::T1, tc[2] * S::T2};
    const int gorg[3] = {g.ng + t0[0], ND >= 2 ? g.ng + t0[1] : 0, ND >= 3 ? g.ng + t0[2] : 0};
    int nvalid[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int tdim = S::T(d);
        nvalid[d] = d < ND ? min(tdim, g.nx[d] - t0[d]) : 1;
    }

    const exact::Eos eeos{g.gamma, g.gamma_m1, g.mmw, EOSK};
    const fast::Eos feos{(float)g.gamma, (float)g.gamma_m1, (float)(1.0 / g.gamma_m1)};

    // ---- phase 1: state tile + halo -> primitives --------------------------
    // The box lands at the first 128-byte boundary of the face buffer (the
    // alignment a tensor copy's shared-memory destination needs; the dynamic
    // shared memory itself starts after the kernel's static shared memory).
    static_assert(NV * S::NP * sizeof(double) + 128 <= (S::A_TOTAL + S::F_TOTAL) * sizeof(R),
                  "the staged box fits the face and flux buffers");
    const unsigned sa_s = smem_u32(sa);
    double* stage = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(sa) + ((128u - (sa_s & 127u)) & 127u));
    bool staged = false;
    if constexpr (ND >= 2) {
        // uniform over the CTA: the destination and the box's x origin are
        // aligned as a tensor copy needs them, else the direct loads run
        const bool aligned = (smem_u32(stage) & 127u) == 0u && ((gorg[0] - 2) & 1) == 0;
        if (tma && aligned) {
            __shared__ uint64_t tile_bar;
            if (tid == 0) {
                mbar_init(&tile_bar, 1);
                mbar_init_fence();
            }
            __syncthreads();
            if (tid == 0) {
                mbar_arrive_expect_tx(&tile_bar, (unsigned)(NV * S::NP * sizeof(double)));
                if constexpr (ND == 2) {
                    tma_load_3d(stage, tmap, &tile_bar, gorg[0] - 2, gorg[1] - 2, 0);
                } else {
                    tma_load_4d(stage, tmap, &tile_bar, gorg[0] - 2, gorg[1] - 2, gorg[2] - 2, 0);
                }
            }
            staged = true;
            const bool arrived = mbar_wait_bounded(&tile_bar, 0);
            if (__syncthreads_or(!arrived) && tid == 0) {
                // the box never arrived: stop the run with HCL_ERR_TIMEOUT
                ctl->err = 6;
                ctl->errflag[(slot + 1) & 1] = 1;
                ctl->final_buf = out_buf;
            }
        }
    }
    for (int p = tid; p < S::NP; p += NT) {
        const int lx = p % S::L0;
        const int ly = (p / S::L0) % S::L1;
        const int lz = p / (S::L0 * S::L1);
        const int gi = min(max(gorg[0] - 2 + lx, 0), g.n[0] - 1);
        const int gj = ND >= 2 ? min(max(gorg[1] - 2 + ly, 0), g.n[1] - 1) : 0;
        const int gk = ND >= 3 ? min(max(gorg[2] - 2 + lz, 0), g.n[2] - 1) : 0;
        const int64_t o = sidx(in, g.n[1], gi, gj, gk);
        double q[NV];
        if (staged) {
            // the box slot of the same (clamped) cell: cells past the array's
            // end repeat its last cell, as the direct loads do (the box's
            // origin is never below 0)
            const int bp = (gi - (gorg[0] - 2)) +
                           S::L0 * ((ND >= 2 ? gj - (gorg[1] - 2) : 0) + S::L1 * (ND >= 3 ? gk - (gorg[2] - 2) : 0));
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                q[v] = stage[v * S::NP + bp];
            }
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                q[v] = __ldg(in.q + o + in.plane * v);
            }
        }
        if constexpr (EXACT) {
            double pr[NV];
            exact::to_prim<ND>(eeos, q, pr);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                sp[v * S::NP + p] = pr[v];
            }
        } else {
            // FP64 internal-energy recovery e = E - |m|^2/(2 rho)
            double r = (double)__frcp_rn((float)q[0]);
            r = r * (2.0 - q[0] * r);
            double mu = 0.0;
            sp[p] = (float)q[0];
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                const double u = q[1 + d] * r;
                mu = fma(q[1 + d], u, mu);
                sp[(1 + d) * S::NP + p] = (float)u;
            }
            sp[(1 + ND) * S::NP + p] = (float)(g.gamma_m1 * fma(-0.5, mu, q[1 + ND]));
        }
        for (int f = 0; f < nfx; ++f) {
            sx[f * S::NP + p] = (R)__ldg(in.q + o + in.plane * (NV + f));
        }
    }
    __syncthreads();

    // ---- phase 2: slopes, faces, Hancock predictor --------------------------
    for (int h = tid; h < S::HCOUNT; h += NT) {
        int x[3] = {0, 0, 0};
        int own = -1; // -1: interior cell (all dims), else the slab's dim
        {
            int r = h;
            if (r < S::TVOL) {
                x[0] = r % S::T0;
                x[1] = (r / S::T0) % S::T1;
                x[2] = r / (S::T0 * S::T1);
            } else {
                r -= S::TVOL;
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    const int slab = S::TVOL / S::T(d);
                    if (own < 0) {
                        if (r < 2 * slab) {
                            own = d;
                            const int side = r / slab;
                            int rr = r % slab;
                            // coordinates of the other dims in order
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
            }
        }
        // local prim-tile coordinate of the cell and global index
        const int lc = (x[0] + 2) + S::L0 * ((ND >= 2 ? x[1] + 2 : 0) + S::L1 * (ND >= 3 ? x[2] + 2 : 0));
        const int gc[3] = {gorg[0] + x[0], ND >= 2 ? gorg[1] + x[1] : 0, ND >= 3 ? gorg[2] + x[2] : 0};
        const int lstride[3] = {1, S::L0, S::L0 * S::L1};
        // clamped global index for grid arrays (only unused cells get clamped)
        int gcc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            gcc[d] = min(max(gc[d], 1), g.n[d] - 2 >= 1 ? g.n[d] - 2 : 0);
            if (d >= ND) {
                gcc[d] = 0;
            }
        }

        R fp[2][ND][NV]; // face primitives [side][dim][var]
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
            double dl = 0.0, dl_m = 0.0, dl_p = 0.0;
            if (EXACT || !g.uniform_cart) {
                dl = g.dx[idim][gcc[idim]];
                dl_m = g.dx[idim][gcc[idim] - 1];
                dl_p = g.dx[idim][gcc[idim] + 1];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const R vc = sp[v * S::NP + lc];
                const R vp = sp[v * S::NP + lc + lstride[idim]];
                const R vm = sp[v * S::NP + lc - lstride[idim]];
                if constexpr (EXACT && EOSK == EOS_PERFECT_GAS_FAST) {
                    // fast FP64 on a uniform grid: the limiter of the raw
                    // differences, halved (positive homogeneity, as below)
                    if (g.uniform_cart) {
                        const double sh = 0.5 * exact::slope(g.limiter, vp - vc, vc - vm, EOSK);
                        fp[0][idim][v] = vc - sh;
                        fp[1][idim][v] = vc + sh;
                    } else {
                        const double slope =
                            exact::slope(g.limiter, (vp - vc) / ((dl + dl_p) / 2), (vc - vm) / ((dl_m + dl) / 2), EOSK);
                        fp[0][idim][v] = vc - ((dl / 2) * slope);
                        fp[1][idim][v] = vc + ((dl / 2) * slope);
                    }
                } else if constexpr (EXACT) {
                    const double slope = exact::slope(g.limiter, (vp - vc) / ((dl + dl_p) / 2), (vc - vm) / ((dl_m + dl) / 2));
                    fp[0][idim][v] = vc - ((dl / 2) * slope);
                    fp[1][idim][v] = vc + ((dl / 2) * slope);
                } else if (g.uniform_cart) {
                    // dl/2 * limiter(dR/dl, dL/dl) = limiter(dR, dL)/2 (every limiter
                    // is positively homogeneous of degree 1)
                    const float s = 0.5f * fast::limited(g.limiter, vp - vc, vc - vm);
                    fp[0][idim][v] = vc - s;
                    fp[1][idim][v] = vc + s;
                } else {
                    const float fdl = (float)dl;
                    const float hR = 2.f * fast::rcp(fdl + (float)dl_p);
                    const float hL = 2.f * fast::rcp((float)dl_m + fdl);
                    const float s = 0.5f * fdl * fast::limited(g.limiter, (vp - vc) * hR, (vc - vm) * hL);
                    fp[0][idim][v] = vc - s;
                    fp[1][idim][v] = vc + s;
                }
            }
        }
        // face conservatives (hydro_reconstruction.hpp:111-126)
        R fc[2][ND][NV];
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                if constexpr (EXACT) {
                    exact::to_cons<ND>(eeos, fp[s][idim], fc[s][idim]);
                } else {
                    fast::to_cons<ND>(feos, fp[s][idim], fc[s][idim]);
                }
            }
        }
        // Hancock predictor (extrapolation_reconstruction.hpp:222-312).  The
        // reference's rho_old/rhou_old (face conservatives before the update)
        // are recomputed from the face primitives with the same products
        // to_cons used, which gives the same bits without keeping copies.
        const int64_t cgl = lidx(g, gcc[0], gcc[1], gcc[2]);
        double dv_c = 1.0, ds_c[ND], ds_p[ND];
        if (!EXACT && g.uniform_cart) {
#pragma unroll
            for (int idim = 0; idim < ND; ++idim) {
                ds_c[idim] = ds_p[idim] = 1.0;
            }
        } else if (g.geom == GEOM_CARTESIAN) {
            const double dxs[3] = {g.dx[0][gcc[0]], g.dx[1][gcc[1]], g.dx[2][gcc[2]]};
            dv_c = dxs[0] * dxs[1] * dxs[2];
#pragma unroll
            for (int idim = 0; idim < ND; ++idim) {
                double a[3] = {dxs[0], dxs[1], dxs[2]};
                a[idim] = 1;
                ds_c[idim] = a[0] * a[1] * a[2];
                a[idim] = 1;
                ds_p[idim] = ds_c[idim]; // Cartesian ds does not depend on the index along idim
            }
        } else {
            dv_c = g.dv[cgl];
#pragma unroll
            for (int idim = 0; idim < ND; ++idim) {
                ds_c[idim] = g.ds[cgl + g.N * idim];
                const int64_t cp = lidx(g, gcc[0] + (idim == 0), gcc[1] + (idim == 1), gcc[2] + (idim == 2));
                ds_p[idim] = g.ds[cp + g.N * idim];
            }
        }
        R mflux[2][ND]; // mass fluxes of the face states before the update (passive scalars)
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
            R fL[NV], fR[NV];
            if constexpr (EXACT) {
                exact::flux_prim<ND>(eeos, fp[0][idim], idim, fL);
                exact::flux_prim<ND>(eeos, fp[1][idim], idim, fR);
                mflux[0][idim] = fL[0];
                mflux[1][idim] = fR[0];
                const double dtodv = dth / dv_c;
                const double dsc = ds_c[idim];
                const double dsp = ds_p[idim];
#pragma unroll
                for (int ipos = 0; ipos < ND; ++ipos) {
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        fc[0][ipos][v] += dtodv * ((fL[v] * dsc) - (fR[v] * dsp));
                        fc[1][ipos][v] += dtodv * ((fL[v] * dsc) - (fR[v] * dsp));
                    }
                }
                if (g.geom == GEOM_SPHERICAL) {
                    const double PL = fp[0][idim][1 + ND], PR = fp[1][idim][1 + ND];
                    const R* pL = fp[0][idim];
                    const R* pR = fp[1][idim];
#pragma unroll
                    for (int ipos = 0; ipos < ND; ++ipos) {
#pragma unroll
                        for (int s = 0; s < 2; ++s) {
                            if (idim == 0) {
                                fc[s][ipos][1 + idim] += exact::src_grad_pres(dtodv, PL, PR, dsc, dsp);
                                if constexpr (ND >= 2) {
                                    fc[s][ipos][1 + idim] += exact::src_grad_u_r(dtodv, pL[0], pR[0], pL[2], pR[2], dsc, dsp);
                                    fc[s][ipos][2] -= exact::src_grad_u_idir_r(dtodv, g.x[0][gcc[0]], g.x[0][gcc[0] + 1], pL[0],
                                                                               pR[0], pL[1], pR[1], pL[2], pR[2], dsc, dsp);
                                }
                                if constexpr (ND == 3) {
                                    fc[s][ipos][1 + idim] += exact::src_grad_u_r(dtodv, pL[0], pR[0], pL[3], pR[3], dsc, dsp);
                                    fc[s][ipos][3] -= exact::src_grad_u_idir_r(dtodv, g.x[0][gcc[0]], g.x[0][gcc[0] + 1], pL[0],
                                                                               pR[0], pL[1], pR[1], pL[3], pR[3], dsc, dsp);
                                }
                            }
                            if (idim == 1) {
                                fc[s][ipos][1 + idim] += exact::src_grad_pres(dtodv, PL, PR, dsc, dsp);
                                if constexpr (ND == 3) {
                                    fc[s][ipos][1 + idim] += exact::src_grad_u_th(dtodv, g.cot_mid1[gcc[1]], pL[0], pR[0], pL[3],
                                                                                  pR[3], dsc, dsp);
                                    fc[s][ipos][3] -= exact::src_grad_u_phi(dtodv, g.sin1[gcc[1]], g.sin1[gcc[1] + 1], pL[0], pR[0],
                                                                            pL[2], pR[2], pL[3], pR[3], dsc, dsp);
                                }
                            }
                        }
                    }
                }
                const double gd = gravity_at(g, gcc[0], idim);
#pragma unroll
                for (int ipos = 0; ipos < ND; ++ipos) {
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const double rho_old = fp[s][ipos][0];
                        const double rhou_old = fp[s][ipos][0] * fp[s][ipos][1 + idim];
                        fc[s][ipos][1 + idim] += dth * gd * rho_old;
                        fc[s][ipos][1 + ND] += dth * gd * rhou_old;
                    }
                }
            } else {
                fast::flux_prim<ND>(feos, fp[0][idim], idim, fL);
                fast::flux_prim<ND>(feos, fp[1][idim], idim, fR);
                mflux[0][idim] = fL[0];
                mflux[1][idim] = fR[0];
                float inc[NV];
                float dtodv = 0.f;
                float dsc = 1.f, dsp = 1.f;
                if (g.uniform_cart) {
                    const float cth = (float)(dth * g.inv_dx[idim]);
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        inc[v] = cth * (fL[v] - fR[v]);
                    }
                } else {
                    dtodv = (float)(dth / dv_c);
                    dsc = (float)ds_c[idim];
                    dsp = (float)ds_p[idim];
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        inc[v] = dtodv * (fL[v] * dsc - fR[v] * dsp);
                    }
                }
                if (g.geom == GEOM_SPHERICAL) {
                    const float* pL = fp[0][idim];
                    const float* pR = fp[1][idim];
                    const float PL = pL[1 + ND], PR = pR[1 + ND];
                    if (idim == 0) {
                        inc[1] += dtodv * 0.5f * (PL + PR) * (dsp - dsc);
                        if constexpr (ND >= 2) {
                            const float x0 = (float)g.x[0][gcc[0]], x0p = (float)g.x[0][gcc[0] + 1];
                            inc[1] += dtodv * 0.25f * (pL[0] * pL[2] * pL[2] + pR[0] * pR[2] * pR[2]) * (dsp - dsc);
                            inc[2] -= dtodv * (x0p - x0) / (x0p + x0) * (pR[0] * pR[2] * pR[1] * dsp + pL[0] * pL[2] * pL[1] * dsc);
                        }
                        if constexpr (ND == 3) {
                            const float x0 = (float)g.x[0][gcc[0]], x0p = (float)g.x[0][gcc[0] + 1];
                            inc[1] += dtodv * 0.25f * (pL[0] * pL[3] * pL[3] + pR[0] * pR[3] * pR[3]) * (dsp - dsc);
                            inc[3] -= dtodv * (x0p - x0) / (x0p + x0) * (pR[0] * pR[3] * pR[1] * dsp + pL[0] * pL[3] * pL[1] * dsc);
                        }
                    }
                    if (idim == 1) {
                        inc[2] += dtodv * 0.5f * (PL + PR) * (dsp - dsc);
                        if constexpr (ND == 3) {
                            const float cot = (float)g.cot_mid1[gcc[1]];
                            const float sm = (float)g.sin1[gcc[1]], spp = (float)g.sin1[gcc[1] + 1];
                            inc[2] += dtodv * 0.25f * (pL[0] * pL[3] * pL[3] + pR[0] * pR[3] * pR[3]) * cot * (dsp - dsc);
                            inc[3] -= dtodv * (spp - sm) / (spp + sm) * (pR[0] * pR[3] * pR[2] * dsp + pL[0] * pL[3] * pL[2] * dsc);
                        }
                    }
                }
                const float gd = (float)gravity_at(g, gcc[0], idim);
                const float dg = (float)dth * gd;
#pragma unroll
                for (int ipos = 0; ipos < ND; ++ipos) {
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const float rho_old = fp[s][ipos][0];
                        const float rhou_old = fp[s][ipos][0] * fp[s][ipos][1 + idim];
#pragma unroll
                        for (int v = 0; v < NV; ++v) {
                            fc[s][ipos][v] += inc[v];
                        }
                        fc[s][ipos][1 + idim] = fmaf(dg, rho_old, fc[s][ipos][1 + idim]);
                        fc[s][ipos][1 + ND] = fmaf(dg, rhou_old, fc[s][ipos][1 + ND]);
                    }
                }
            }
        }
        // passive scalars: face values with the same limited slopes
        // (hydro_reconstruction.hpp:105-109), made conservative with the face
        // density before the predictor, advanced by the predictor's mass
        // fluxes (extrapolation_reconstruction.hpp:315-337) and turned back
        // into fractions with the predicted face density (:329-339)
        for (int f = 0; f < nfx; ++f) {
            const R* xs = sx + f * S::NP;
            R xf[2][ND];
#pragma unroll
            for (int idim = 0; idim < ND; ++idim) {
                const R vc = xs[lc];
                const R vp = xs[lc + lstride[idim]];
                const R vm = xs[lc - lstride[idim]];
                if constexpr (EXACT) {
                    const double dl = g.dx[idim][gcc[idim]];
                    const double dl_m = g.dx[idim][gcc[idim] - 1];
                    const double dl_p = g.dx[idim][gcc[idim] + 1];
                    const double slope = exact::slope(g.limiter, (vp - vc) / ((dl + dl_p) / 2), (vc - vm) / ((dl_m + dl) / 2),
                                                      EOSK);
                    xf[0][idim] = vc - ((dl / 2) * slope);
                    xf[1][idim] = vc + ((dl / 2) * slope);
                } else if (g.uniform_cart) {
                    const float sl = 0.5f * fast::limited(g.limiter, vp - vc, vc - vm);
                    xf[0][idim] = vc - sl;
                    xf[1][idim] = vc + sl;
                } else {
                    const float fdl = (float)g.dx[idim][gcc[idim]];
                    const float hR = 2.f * fast::rcp(fdl + (float)g.dx[idim][gcc[idim] + 1]);
                    const float hL = 2.f * fast::rcp((float)g.dx[idim][gcc[idim] - 1] + fdl);
                    const float sl = 0.5f * fdl * fast::limited(g.limiter, (vp - vc) * hR, (vc - vm) * hL);
                    xf[0][idim] = vc - sl;
                    xf[1][idim] = vc + sl;
                }
            }
            R xc[2][ND];
#pragma unroll
            for (int ipos = 0; ipos < ND; ++ipos) {
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    xc[s][ipos] = xf[s][ipos] * fp[s][ipos][0];
                }
            }
#pragma unroll
            for (int idim = 0; idim < ND; ++idim) {
                const R ffL = xf[0][idim] * mflux[0][idim];
                const R ffR = xf[1][idim] * mflux[1][idim];
                R inc;
                if constexpr (EXACT) {
                    inc = (dth / dv_c) * ((ffL * ds_c[idim]) - (ffR * ds_p[idim]));
                } else if (g.uniform_cart) {
                    inc = (float)(dth * g.inv_dx[idim]) * (ffL - ffR);
                } else {
                    inc = (float)(dth / dv_c) * (ffL * (float)ds_c[idim] - ffR * (float)ds_p[idim]);
                }
#pragma unroll
                for (int ipos = 0; ipos < ND; ++ipos) {
                    xc[0][ipos] += inc;
                    xc[1][ipos] += inc;
                }
            }
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                if (own >= 0 && own != d) {
                    continue;
                }
                const int a = (x[0] + (d == 0)) + S::Adim(d, 0) * ((x[1] + (d == 1)) + S::Adim(d, 1) * (x[2] + (d == 2)));
                R* xb = sxa(d);
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    xb[(s * nfx + f) * S::Asize(d) + a] = xc[s][d] / fc[s][d][0];
                }
            }
        }
        // store the faces this cell owns
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            if (own >= 0 && own != d) {
                continue;
            }
            const int ax = x[0] + (d == 0 ? 1 : 0);
            const int ay = x[1] + (d == 1 ? 1 : 0);
            const int az = x[2] + (d == 2 ? 1 : 0);
            const int a = ax + S::Adim(d, 0) * (ay + S::Adim(d, 1) * az);
            R* base = sa + S::Aoff(d);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    base[(s * NV + v) * S::Asize(d) + a] = fc[s][d][v];
                }
            }
        }
    }
    __syncthreads();

    // ---- phase 3: one Riemann solve per face --------------------------------
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const R* base = sa + S::Aoff(d);
        R* fbase = sf + S::Foff(d);
        for (int f = tid; f < S::Fsize(d); f += NT) {
            const int fx0 = f % S::Fdim(d, 0);
            const int fx1 = (f / S::Fdim(d, 0)) % S::Fdim(d, 1);
            const int fx2 = f / (S::Fdim(d, 0) * S::Fdim(d, 1));
            // left cell (coordinate f_d - 1) has A-coordinate f_d; right: f_d + 1
            const int aL = fx0 + S::Adim(d, 0) * (fx1 + S::Adim(d, 1) * fx2);
            const int step_d = d == 0 ? 1 : (d == 1 ? S::Adim(d, 0) : S::Adim(d, 0) * S::Adim(d, 1));
            const int aR = aL + step_d;
            R cL[NV], cR[NV], fl[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                cL[v] = base[(NV + v) * S::Asize(d) + aL];
                cR[v] = base[v * S::Asize(d) + aR];
            }
            if constexpr (EXACT) {
                exact::riemann<ND>(eeos, g.riemann, cL, cR, d, fl);
            } else {
                fast::riemann<ND>(feos, g.riemann, cL, cR, d, fl);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                fbase[v * S::Fsize(d) + f] = fl[v];
            }
        }
    }
    __syncthreads();

    // ---- phase 4: Godunov update, ghost images, health, CFL -----------------
    // pressure_fix.hpp:19-172 on one interior cell (FP64; in the FP32-mixed
    // tiles from the FP32 predicted face states): q the old state,
    // qn the Godunov update, whose energy it may replace.  The face states are
    // the predicted ones in shared memory, the neighbours' old states come
    // from global memory; expression order as in the reference (the energy is
    // overwritten in the inner loop and the last value stays).
    auto pressure_fix_cell = [&](int x0, int x1, int x2, int gi, int gj, int gk, int64_t cgl, const double* q,
                                 double* qn) {
        const double ekin = exact::ek_cons<ND>(q);
        const double evol = q[1 + ND] - ekin;
        const double eps = g.eps_pf;
        if (!(evol < eps * ekin)) {
            return;
        }
        double prim[NV];
        exact::to_prim<ND>(eeos, q, prim);
        const double de_god = (qn[1 + ND] - exact::ek_cons<ND>(qn)) - evol;
        const double eps2 = eps / 10;
        double alpha = (evol * evol) / (ekin * ekin * eps * eps);
        if (evol < eps2 * ekin) {
            alpha = 0;
        }
        double sum = 0;
#pragma unroll
        for (int idr = 0; idr < ND; ++idr) {
            sum += q[1 + idr] * q[1 + idr] / q[0];
        }
        double divU = 0, divUE = 0, einL = 0, einR = 0;
        double En = q[1 + ND];
        const int xs3[3] = {x0, x1, x2};
#pragma unroll
        for (int idim = 0; idim < ND; ++idim) {
            const int di = idim == 0, dj = idim == 1, dk = idim == 2;
            const int64_t cp = lidx(g, gi + di, gj + dj, gk + dk);
            const int64_t om = sidx(in, g.n[1], gi - di, gj - dj, gk - dk);
            const int64_t op = sidx(in, g.n[1], gi + di, gj + dj, gk + dk);
            double qm[NV], qp[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                qm[v] = in.q[om + in.plane * v];
                qp[v] = in.q[op + in.plane * v];
            }
            const R* ab = sa + S::Aoff(idim);
            const int a = (xs3[0] + di) + S::Adim(idim, 0) * ((xs3[1] + dj) + S::Adim(idim, 1) * (xs3[2] + dk));
            const int astep = idim == 0 ? 1 : (idim == 1 ? S::Adim(idim, 0) : S::Adim(idim, 0) * S::Adim(idim, 1));
            double vL[NV], vR[NV], mR[NV], pL[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                vL[v] = ab[v * S::Asize(idim) + a];
                vR[v] = ab[(NV + v) * S::Asize(idim) + a];
                mR[v] = ab[(NV + v) * S::Asize(idim) + a - astep];
                pL[v] = ab[v * S::Asize(idim) + a + astep];
            }
            double primL[NV], primR[NV], prim_mR[NV], prim_pL[NV];
            exact::to_prim<ND>(eeos, vL, primL);
            exact::to_prim<ND>(eeos, vR, primR);
            exact::to_prim<ND>(eeos, mR, prim_mR);
            exact::to_prim<ND>(eeos, pL, prim_pL);
            const double dv = g.dv[cgl];
#pragma unroll
            for (int ipos = 0; ipos < ND; ++ipos) {
                const double us = (prim_mR[1 + ipos] + primL[1 + ipos]) / 2;
                const double us_p = (primR[1 + ipos] + prim_pL[1 + ipos]) / 2;
                const double dsp = g.ds[cp + g.N * ipos];
                const double dsc = g.ds[cgl + g.N * ipos];
                divU += ((us_p * dsp) - (us * dsc)) / dv;
                if (us_p > 0) {
                    einR = q[1 + ND] - exact::ek_cons<ND>(q);
                } else {
                    einR = qp[1 + ND] - exact::ek_cons<ND>(qp);
                }
                if (us < 0) {
                    einL = q[1 + ND] - exact::ek_cons<ND>(q);
                } else {
                    einL = qm[1 + ND] - exact::ek_cons<ND>(qm);
                }
                divUE += ((us_p * einR * dsp) - (us * einL * dsc)) / dv;
                const double de_pf = dt * ((-prim[1 + ND] * divU) - divUE);
                const double de_tot = (alpha * de_god) + ((1 - alpha) * de_pf);
                En = evol + de_tot + (1. / 2 * sum);
            }
        }
        qn[1 + ND] = En;
    };
    double inv_local = 0.0;
    for (int c = tid; c < S::TVOL; c += NT) {
        const int x0 = c % S::T0;
        const int x1 = (c / S::T0) % S::T1;
        const int x2 = c / (S::T0 * S::T1);
        if (x0 >= nvalid[0] || x1 >= nvalid[1] || x2 >= nvalid[2]) {
            continue;
        }
        const int gi = gorg[0] + x0, gj = ND >= 2 ? gorg[1] + x1 : 0, gk = ND >= 3 ? gorg[2] + x2 : 0;
        const int64_t so = sidx(in, g.n[1], gi, gj, gk);
        double q[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            q[v] = in.q[so + in.plane * v];
        }
        const int64_t cgl = lidx(g, gi, gj, gk);
        double qn[NV];
        if constexpr (EXACT) {
            // godunov_scheme.hpp:114-260 in the reference's accumulation order
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                qn[v] = q[v];
            }
            double dv_c, ds_c[ND], ds_p[ND];
            if (g.geom == GEOM_CARTESIAN) {
                const double dxs[3] = {g.dx[0][gi], g.dx[1][gj], g.dx[2][gk]};
                dv_c = dxs[0] * dxs[1] * dxs[2];
#pragma unroll
                for (int idim = 0; idim < ND; ++idim) {
                    double a[3] = {dxs[0], dxs[1], dxs[2]};
                    a[idim] = 1;
                    ds_c[idim] = a[0] * a[1] * a[2];
                    ds_p[idim] = ds_c[idim];
                }
            } else {
                dv_c = g.dv[cgl];
#pragma unroll
                for (int idim = 0; idim < ND; ++idim) {
                    ds_c[idim] = g.ds[cgl + g.N * idim];
                    ds_p[idim] = g.ds[lidx(g, gi + (idim == 0), gj + (idim == 1), gk + (idim == 2)) + g.N * idim];
                }
            }
#pragma unroll
            for (int idim = 0; idim < ND; ++idim) {
                const int xs[3] = {x0, x1, x2};
                const int fidx = xs[0] + S::Fdim(idim, 0) * (xs[1] + S::Fdim(idim, 1) * xs[2]);
                const int fstep = idim == 0 ? 1 : (idim == 1 ? S::Fdim(idim, 0) : S::Fdim(idim, 0) * S::Fdim(idim, 1));
                const R* fb = sf + S::Foff(idim);
                const double dtodv = dt / dv_c;
                const double dsc = ds_c[idim];
                const double dsp = ds_p[idim];
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    const double FL = fb[v * S::Fsize(idim) + fidx];
                    const double FR = fb[v * S::Fsize(idim) + fidx + fstep];
                    qn[v] += dtodv * ((FL * dsc) - (FR * dsp));
                }
                if (g.geom == GEOM_SPHERICAL) {
                    // godunov_scheme.hpp:165-256 with the cell's own face states
                    const R* ab = sa + S::Aoff(idim);
                    const int a = (xs[0] + (idim == 0)) + S::Adim(idim, 0) * ((xs[1] + (idim == 1)) + S::Adim(idim, 1) * (xs[2] + (idim == 2)));
                    double vL[NV], vR[NV], pl[NV], pr[NV];
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        vL[v] = ab[v * S::Asize(idim) + a];
                        vR[v] = ab[(NV + v) * S::Asize(idim) + a];
                    }
                    exact::to_prim<ND>(eeos, vL, pl);
                    exact::to_prim<ND>(eeos, vR, pr);
                    if (idim == 0) {
                        qn[1] += exact::src_grad_pres(dtodv, pl[1 + ND], pr[1 + ND], dsc, dsp);
                        if constexpr (ND >= 2) {
                            qn[1] += exact::src_grad_u_r(dtodv, pl[0], pr[0], pl[2], pr[2], dsc, dsp);
                            qn[2] -= exact::src_grad_u_idir_r(dtodv, g.x[0][gi], g.x[0][gi + 1], pl[0], pr[0], pl[1], pr[1],
                                                              pl[2], pr[2], dsc, dsp);
                        }
                        if constexpr (ND == 3) {
                            qn[1] += exact::src_grad_u_r(dtodv, pl[0], pr[0], pl[3], pr[3], dsc, dsp);
                            qn[3] -= exact::src_grad_u_idir_r(dtodv, g.x[0][gi], g.x[0][gi + 1], pl[0], pr[0], pl[1], pr[1],
                                                              pl[3], pr[3], dsc, dsp);
                        }
                    }
                    if constexpr (ND >= 2) {
                        if (idim == 1) {
                            qn[2] += exact::src_grad_pres(dtodv, pl[1 + ND], pr[1 + ND], dsc, dsp);
                            if constexpr (ND == 3) {
                                qn[2] += exact::src_grad_u_th(dtodv, g.cot_mid1[gj], pl[0], pr[0], pl[3], pr[3], dsc, dsp);
                                qn[3] -= exact::src_grad_u_phi(dtodv, g.sin1[gj], g.sin1[gj + 1], pl[0], pr[0], pl[2], pr[2],
                                                               pl[3], pr[3], dsc, dsp);
                            }
                        }
                    }
                }
                const double gd = gravity_at(g, gi, idim);
                qn[1 + idim] += dt * gd * q[0];
                qn[1 + ND] += dt * gd * q[1 + idim];
            }
        } else {
            double acc[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                acc[v] = 0.0;
            }
            const int xs[3] = {x0, x1, x2};
#pragma unroll
            for (int idim = 0; idim < ND; ++idim) {
                const int fidx = xs[0] + S::Fdim(idim, 0) * (xs[1] + S::Fdim(idim, 1) * xs[2]);
                const int fstep = idim == 0 ? 1 : (idim == 1 ? S::Fdim(idim, 0) : S::Fdim(idim, 0) * S::Fdim(idim, 1));
                const R* fb = sf + S::Foff(idim);
                if (g.uniform_cart) {
                    const double cdt = dt * g.inv_dx[idim];
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        const double FL = (double)fb[v * S::Fsize(idim) + fidx];
                        const double FR = (double)fb[v * S::Fsize(idim) + fidx + fstep];
                        acc[v] = fma(cdt, FL - FR, acc[v]);
                    }
                } else {
                    double dv_c, dsc, dsp;
                    if (g.geom == GEOM_CARTESIAN) {
                        const double dxs[3] = {g.dx[0][gi], g.dx[1][gj], g.dx[2][gk]};
                        dv_c = dxs[0] * dxs[1] * dxs[2];
                        double a[3] = {dxs[0], dxs[1], dxs[2]};
                        a[idim] = 1;
                        dsc = a[0] * a[1] * a[2];
                        dsp = dsc;
                    } else {
                        dv_c = g.dv[cgl];
                        dsc = g.ds[cgl + g.N * idim];
                        dsp = g.ds[lidx(g, gi + (idim == 0), gj + (idim == 1), gk + (idim == 2)) + g.N * idim];
                    }
                    const double dtodv = dt / dv_c;
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        const double FL = (double)fb[v * S::Fsize(idim) + fidx];
                        const double FR = (double)fb[v * S::Fsize(idim) + fidx + fstep];
                        acc[v] = fma(dtodv, FL * dsc - FR * dsp, acc[v]);
                    }
                    if (g.geom == GEOM_SPHERICAL) {
                        const R* ab = sa + S::Aoff(idim);
                        const int a = (xs[0] + (idim == 0)) + S::Adim(idim, 0) * ((xs[1] + (idim == 1)) + S::Adim(idim, 1) * (xs[2] + (idim == 2)));
                        float vL[NV], vR[NV], pl[NV], pr[NV];
#pragma unroll
                        for (int v = 0; v < NV; ++v) {
                            vL[v] = ab[v * S::Asize(idim) + a];
                            vR[v] = ab[(NV + v) * S::Asize(idim) + a];
                        }
                        fast::to_prim<ND>(feos, vL, pl);
                        fast::to_prim<ND>(feos, vR, pr);
                        const double dd = dsp - dsc;
                        if (idim == 0) {
                            acc[1] += dtodv * 0.5 * ((double)pl[1 + ND] + pr[1 + ND]) * dd;
                            if constexpr (ND >= 2) {
                                const double x0n = g.x[0][gi], x0p = g.x[0][gi + 1];
                                acc[1] += dtodv * 0.25 * ((double)pl[0] * pl[2] * pl[2] + (double)pr[0] * pr[2] * pr[2]) * dd;
                                acc[2] -= dtodv * (x0p - x0n) / (x0p + x0n) *
                                          ((double)pr[0] * pr[2] * pr[1] * dsp + (double)pl[0] * pl[2] * pl[1] * dsc);
                            }
                            if constexpr (ND == 3) {
                                const double x0n = g.x[0][gi], x0p = g.x[0][gi + 1];
                                acc[1] += dtodv * 0.25 * ((double)pl[0] * pl[3] * pl[3] + (double)pr[0] * pr[3] * pr[3]) * dd;
                                acc[3] -= dtodv * (x0p - x0n) / (x0p + x0n) *
                                          ((double)pr[0] * pr[3] * pr[1] * dsp + (double)pl[0] * pl[3] * pl[1] * dsc);
                            }
                        }
                        if constexpr (ND >= 2) {
                            if (idim == 1) {
                                acc[2] += dtodv * 0.5 * ((double)pl[1 + ND] + pr[1 + ND]) * dd;
                                if constexpr (ND == 3) {
                                    const double sm = g.sin1[gj], spp = g.sin1[gj + 1];
                                    acc[2] += dtodv * 0.25 * ((double)pl[0] * pl[3] * pl[3] + (double)pr[0] * pr[3] * pr[3]) *
                                              g.cot_mid1[gj] * dd;
                                    acc[3] -= dtodv * (spp - sm) / (spp + sm) *
                                              ((double)pr[0] * pr[3] * pr[2] * dsp + (double)pl[0] * pl[3] * pl[2] * dsc);
                                }
                            }
                        }
                    }
                }
                const double gd = gravity_at(g, gi, idim);
                acc[1 + idim] = fma(dt * gd, q[0], acc[1 + idim]);
                acc[1 + ND] = fma(dt * gd, q[1 + idim], acc[1 + ND]);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                qn[v] = q[v] + acc[v];
            }
        }

        // FP32-mixed tiles: the same FP64 arithmetic on their FP32 face states
        if (g.pressure_fix) {
            pressure_fix_cell(x0, x1, x2, gi, gj, gk, cgl, q, qn);
        }

        // health check (main.cpp:397-425) and CFL of the new state (time_step.hpp:55-77)
        double evol, inv_rho_u[ND], sound;
        if constexpr (EXACT) {
            evol = qn[1 + ND] - exact::ek_cons<ND>(qn);
            double pr[NV];
            exact::to_prim<ND>(eeos, qn, pr);
            sound = exact::sound(eeos, pr[0], pr[1 + ND]);
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                inv_rho_u[d] = fabs(pr[1 + d]);
            }
        } else {
            double r = (double)__frcp_rn((float)qn[0]);
            r = r * (2.0 - qn[0] * r);
            double mu = 0.0;
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                const double u = qn[1 + d] * r;
                mu = fma(qn[1 + d], u, mu);
                inv_rho_u[d] = fabs(u);
            }
            evol = fma(-0.5, mu, qn[1 + ND]);
            const double c2 = g.gamma * g.gamma_m1 * evol * r;
            double y = (double)rsqrtf((float)c2);
            y = y * (1.5 - 0.5 * c2 * y * y);
            sound = c2 * y;
        }
        if (!(evol >= 0.0)) {
            atomicMin(&ctl->bad_cell, (unsigned long long)cgl);
            ctl->err = 4; // HCL_ERR_INVALID_STATE
            ctl->errflag[(slot + 1) & 1] = 1;
            ctl->final_buf = out_buf;
        }

        // store + ghost images
        int pos[3][9];
        int flp[3][9];
        int cnt[3] = {1, 1, 1};
        const int gidx[3] = {gi, gj, gk};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            pos[d][0] = gidx[d];
            flp[d][0] = 0;
            if (d < ND) {
                cnt[d] += ghost_images(gidx[d], g.n[d], g.ng, g.bc[2 * d], g.bc[2 * d + 1], &pos[d][1], &flp[d][1]);
            }
        }
        for (int a2 = 0; a2 < cnt[2]; ++a2) {
            for (int a1 = 0; a1 < cnt[1]; ++a1) {
                for (int a0 = 0; a0 < cnt[0]; ++a0) {
                    const int pi = pos[0][a0], pj = pos[1][a1], pk = pos[2][a2];
                    const int64_t oo = sidx(out, g.n[1], pi, pj, pk);
                    const int fl[3] = {flp[0][a0], flp[1][a1], flp[2][a2]};
                    out.q[oo] = qn[0];
#pragma unroll
                    for (int d = 0; d < ND; ++d) {
                        out.q[oo + out.plane * (1 + d)] = fl[d] ? -qn[1 + d] : qn[1 + d];
                    }
                    out.q[oo + out.plane * (1 + ND)] = qn[1 + ND];
                    // CFL contribution at this position (all_ghosts range)
                    double dxg[3] = {g.dx[0][pi], g.dx[1][pj], g.dx[2][pk]};
                    if (g.geom == GEOM_SPHERICAL) {
                        if (ND == 2) {
                            dxg[1] *= g.xc[0][pi];
                        }
                        if (ND == 3) {
                            dxg[1] *= g.xc[0][pi];
                            dxg[2] *= g.xc[0][pi] * g.sin_xc1[pj];
                        }
                    }
                    double cell = 0;
                    if (!EXACT && g.uniform_cart) {
#pragma unroll
                        for (int d = 0; d < ND; ++d) {
                            cell = fma(inv_rho_u[d] + sound, g.inv_dx[d], cell);
                        }
                    } else {
#pragma unroll
                        for (int d = 0; d < ND; ++d) {
                            cell += (inv_rho_u[d] + sound) / dxg[d];
                        }
                    }
                    if (isnan(cell)) {
                        inv_local = __longlong_as_double(0x7ff8000000000000ll);
                    } else if (!isnan(inv_local)) {
                        inv_local = inv_local > cell ? inv_local : cell;
                    }
                }
            }
        }

        // passive scalars (godunov_scheme.hpp:118-123, :262-301): fx rho plus
        // the upwind face values times the Riemann mass fluxes, divided by the
        // new density and clamped to [0, 1]; ghost images copy the value
        if (nfx > 0) {
            double dv_c = 1.0, ds_c[ND], ds_p[ND];
            if (EXACT || !g.uniform_cart) {
                if (g.geom == GEOM_CARTESIAN) {
                    const double dxs[3] = {g.dx[0][gi], g.dx[1][gj], g.dx[2][gk]};
                    dv_c = dxs[0] * dxs[1] * dxs[2];
#pragma unroll
                    for (int idim = 0; idim < ND; ++idim) {
                        double a[3] = {dxs[0], dxs[1], dxs[2]};
                        a[idim] = 1;
                        ds_c[idim] = a[0] * a[1] * a[2];
                        ds_p[idim] = ds_c[idim];
                    }
                } else {
                    dv_c = g.dv[cgl];
#pragma unroll
                    for (int idim = 0; idim < ND; ++idim) {
                        ds_c[idim] = g.ds[cgl + g.N * idim];
                        ds_p[idim] = g.ds[lidx(g, gi + (idim == 0), gj + (idim == 1), gk + (idim == 2)) + g.N * idim];
                    }
                }
            }
            const int xs3[3] = {x0, x1, x2};
            for (int f = 0; f < nfx; ++f) {
                double xn = in.q[so + in.plane * (NV + f)] * q[0];
                double xacc = 0.0;
#pragma unroll
                for (int idim = 0; idim < ND; ++idim) {
                    const int fidx = xs3[0] + S::Fdim(idim, 0) * (xs3[1] + S::Fdim(idim, 1) * xs3[2]);
                    const int fstep = idim == 0 ? 1 : (idim == 1 ? S::Fdim(idim, 0) : S::Fdim(idim, 0) * S::Fdim(idim, 1));
                    const R* fb = sf + S::Foff(idim);
                    const R FL = fb[fidx];
                    const R FR = fb[fidx + fstep];
                    const int a = (xs3[0] + (idim == 0)) +
                                  S::Adim(idim, 0) * ((xs3[1] + (idim == 1)) + S::Adim(idim, 1) * (xs3[2] + (idim == 2)));
                    const int astep = idim == 0 ? 1 : (idim == 1 ? S::Adim(idim, 0) : S::Adim(idim, 0) * S::Adim(idim, 1));
                    const R* side0 = sxa(idim) + f * S::Asize(idim);
                    const R* side1 = sxa(idim) + (nfx + f) * S::Asize(idim);
                    const R xL = FL < 0 ? side0[a] : side1[a - astep];
                    const R xR = FR < 0 ? side0[a + astep] : side1[a];
                    if constexpr (EXACT) {
                        const double ffL = xL * FL;
                        const double ffR = xR * FR;
                        xn += (dt / dv_c) * ((ffL * ds_c[idim]) - (ffR * ds_p[idim]));
                    } else if (g.uniform_cart) {
                        xacc = fma(dt * g.inv_dx[idim], (double)xL * FL - (double)xR * FR, xacc);
                    } else {
                        xacc = fma(dt / dv_c, (double)xL * FL * ds_c[idim] - (double)xR * FR * ds_p[idim], xacc);
                    }
                }
                if constexpr (!EXACT) {
                    xn += xacc;
                }
                double v = xn / qn[0];
                v = v < 0. ? 0. : (v > 1. ? 1. : v);
                for (int a2 = 0; a2 < cnt[2]; ++a2) {
                    for (int a1 = 0; a1 < cnt[1]; ++a1) {
                        for (int a0 = 0; a0 < cnt[0]; ++a0) {
                            out.q[sidx(out, g.n[1], pos[0][a0], pos[1][a1], pos[2][a2]) + out.plane * (NV + f)] = v;
                        }
                    }
                }
            }
        }
    }
    // CTA max of 1/dt -> one atomic
    __shared__ double red[32];
    bool nan_seen = isnan(inv_local);
    double m = nan_seen ? 0.0 : inv_local;
    m = warp_max_d(m);
    const int lane = tid & 31, w = tid >> 5;
    if (lane == 0) {
        red[w] = m;
    }
    __syncthreads();
    if (w == 0) {
        m = lane < (NT + 31) / 32 ? red[lane] : 0.0;
        m = warp_max_d(m);
        if (lane == 0) {
            atomicMax(&ctl->inv_dt_bits[(slot + 1) % 3], dbl_bits(m));
        }
    }
    if (nan_seen) {
        atomicMax(&ctl->inv_dt_bits[(slot + 1) % 3], 0x7ff8000000000000ull);
    }
}

template <int ND, bool EXACT, int TX, int TY, int TZ, int EOSK = EOS_PERFECT_GAS>
__global__ void __launch_bounds__(TX*(ND >= 2 ? TY : 1)*(ND >= 3 ? TZ : 1))
k_fused_step(GridDev g, StateDev in, StateDev out, StepCtl* ctl, RunParamsDev rp, int slot, int out_buf,
             const __grid_constant__ CUtensorMap tmap, int tma)
{
    fused_step_body<ND, EXACT, TX, TY, TZ, EOSK>(g, in, out, ctl, rp, slot, out_buf, &tmap, tma);
}

// the same step with the occupancy bound above (instantiated where it is > 0)
template <int ND, bool EXACT, int TX, int TY, int TZ, int EOSK = EOS_PERFECT_GAS>
__global__ void __launch_bounds__(TX*(ND >= 2 ? TY : 1)*(ND >= 3 ? TZ : 1),
                                  fused_min_blocks<ND, EXACT, TX, TY, TZ>() > 0 ? fused_min_blocks<ND, EXACT, TX, TY, TZ>() : 1)
k_fused_step_occ(GridDev g, StateDev in, StateDev out, StepCtl* ctl, RunParamsDev rp, int slot, int out_buf,
                 const __grid_constant__ CUtensorMap tmap, int tma)
{
    fused_step_body<ND, EXACT, TX, TY, TZ, EOSK>(g, in, out, ctl, rp, slot, out_buf, &tmap, tma);
}

template <int ND, bool EXACT, int TX, int TY, int TZ>
struct FusedLauncher {
    using S = Shape<ND, TX, TY, TZ>;
    using R = std::conditional_t<EXACT, double, float>;
    // dynamic shared memory of a launch with nfx passive scalars
    static size_t smem(int nfx = 0)
    {
        return smem_bytes_for<R>(S::NP, S::A_TOTAL, S::F_TOTAL, S::NV) +
               sizeof(R) * (size_t)nfx * (S::NP + 2 * (S::A_TOTAL / (2 * S::NV)));
    }
    static int threads() { return S::TVOL; }
    // Opts the kernel into the device's largest dynamic shared memory per
    // block (launches without passive scalars use smem(0) and keep their
    // occupancy); called once per process before any launch (never during
    // stream capture).
    static constexpr int kMinBlocks = fused_min_blocks<ND, EXACT, TX, TY, TZ>();
    static void configure()
    {
        set_max_dynamic(reinterpret_cast<const void*>(k_fused_step<ND, EXACT, TX, TY, TZ>));
        if constexpr (EXACT) {
            set_max_dynamic(reinterpret_cast<const void*>(k_fused_step<ND, EXACT, TX, TY, TZ, EOS_RAD_GAS>));
        }
        if constexpr (kMinBlocks > 0) {
            set_max_dynamic(reinterpret_cast<const void*>(k_fused_step_occ<ND, EXACT, TX, TY, TZ>));
            if constexpr (EXACT) {
                set_max_dynamic(reinterpret_cast<const void*>(k_fused_step_occ<ND, EXACT, TX, TY, TZ, EOS_RAD_GAS>));
            }
        }
    }
    // the occupancy-bounded kernel pays off when that many CTAs fit the SM's
    // shared memory (1 KB reserved per CTA, up to 512 B static)
    static bool use_occ(int nfx)
    {
        if constexpr (kMinBlocks > 0) {
            static PerDevice cache;
            int dev = 0;
            cudaGetDevice(&dev);
            const int per_sm = cache.get(dev, [dev] {
                int v = 0;
                cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
                return v;
            });
            return (size_t)kMinBlocks * (smem(nfx) + 1024 + 512) <= (size_t)per_sm;
        }
        return false;
    }
    // the per-block opt-in limit less the kernel's static shared memory
    static void set_max_dynamic(const void* fn)
    {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, fn);
        const int bytes = std::max(optin - (int)fa.sharedSizeBytes, (int)smem());
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    }
    // the kernel of one compile-time EOS kind (occupancy-bounded when it pays)
    template <int EOSK>
    static void launch_kind(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl,
                            const RunParamsDev& rp, int slot, int out_buf, cudaStream_t s)
    {
        const size_t sm = smem(g.nfx);
        const int nt0 = (g.nx[0] + S::T0 - 1) / S::T0;
        const int nt1 = (g.nx[1] + S::T1 - 1) / S::T1;
        const int nt2 = (g.nx[2] + S::T2 - 1) / S::T2;
        const int blocks = nt0 * nt1 * nt2;
        // the tile + halo box of the input state for TMA staging (2-D and 3-D;
        // its x origin gorg[0] - 2 = ng - 2 + T0 k is 16-byte aligned for an
        // even ghost width)
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        const int box[3] = {S::L0, S::L1, S::L2};
        const int tma = (ND >= 2 && g.ng % 2 == 0 && encode_tile_map(g, in, S::NV, box, &map)) ? 1 : 0;
        if (use_occ(g.nfx)) {
            k_fused_step_occ<ND, EXACT, TX, TY, TZ, EOSK>
                <<<blocks, S::TVOL, sm, s>>>(g, in, out, ctl, rp, slot, out_buf, map, tma);
        } else {
            k_fused_step<ND, EXACT, TX, TY, TZ, EOSK><<<blocks, S::TVOL, sm, s>>>(g, in, out, ctl, rp, slot, out_buf, map, tma);
        }
        ++g_launches;
    }
    static void launch(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                       int slot, int out_buf, cudaStream_t s)
    {
        if constexpr (EXACT) {
            if (g.eos == EOS_RAD_GAS) {
                launch_kind<EOS_RAD_GAS>(g, in, out, ctl, rp, slot, out_buf, s);
                return;
            }
        }
        launch_kind<EOS_PERFECT_GAS>(g, in, out, ctl, rp, slot, out_buf, s);
    }
    // fast FP64: the perfect gas in its fast forms (translation units built
    // with FMA contraction)
    static void configure_fast()
    {
        static_assert(EXACT, "fast FP64 runs the FP64 kernels");
        set_max_dynamic(reinterpret_cast<const void*>(k_fused_step<ND, EXACT, TX, TY, TZ, EOS_PERFECT_GAS_FAST>));
        if constexpr (kMinBlocks > 0) {
            set_max_dynamic(reinterpret_cast<const void*>(k_fused_step_occ<ND, EXACT, TX, TY, TZ, EOS_PERFECT_GAS_FAST>));
        }
    }
};

} // namespace hcl::fused
