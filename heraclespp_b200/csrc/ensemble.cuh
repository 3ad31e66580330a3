// ensemble.cuh -- batched ensemble of independent 2-D problems in one
// persistent launch.
//
// Every problem keeps its own grid, state buffers, CFL time step and control
// block (the one its handle uses).  Work items are warp strips of all
// problems; each persistent warp takes items round-robin, and a grid-wide
// barrier separates time steps (each problem's step n+1 needs its whole step n
// and its 1/dt reduction).  The barrier spins with an iteration limit: when
// the limit runs out it records HCL_ERR_TIMEOUT and every CTA returns, so a
// scheduling fault turns into an error status, not a hang.  The launch is
// cooperative, so all CTAs are co-resident by construction.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fused_strip2d.cuh"
#include "hcl_device.cuh"
#include "stages.hpp"

namespace hcl::ensemble {

// Returns the same answer to every thread of the CTA (thread 0 decides), so a
// CTA leaves the step loop as a whole and no warp is left half-exited.
// Thread 0 polls at most spin_limit times (each poll sleeps ~64 ns), then
// records HCL_ERR_TIMEOUT; a CTA that sees any error recorded stops waiting.
__device__ __forceinline__ bool grid_barrier(unsigned int* count, unsigned int target, int* status,
                                             long long spin_limit = kSpinLimit)
{
    __shared__ int go_on;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(count, 1u);
        long long spins = 0;
        int ok = 1;
        while (*(volatile unsigned int*)count < target) {
            if (*(volatile int*)status != 0) {
                ok = 0;
                break;
            }
            if (++spins > spin_limit) {
                atomicExch(status, 6); // HCL_ERR_TIMEOUT
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
        go_on = ok && *(volatile int*)status == 0;
    }
    __syncthreads();
    return go_on != 0;
}

// NW warps per CTA (4 or 16); each warp's row ring lives in dynamic shared
// memory (NW x kStripRingDoubles doubles).
template <int LIM, int RS, int NW>
__global__ void __launch_bounds__(32 * NW, NW == 16 ? 1 : 4)
k_ensemble(const Prob* __restrict__ probs, const int* __restrict__ item_prob, Params ep, unsigned int* barrier,
           int* status)
{
    extern __shared__ __align__(16) double s_ens_ring[];
    const int lane = threadIdx.x & 31;
    const int warps_total = gridDim.x * (blockDim.x >> 5);
    const int wid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const fused::StripRing ring =
        reinterpret_cast<fused::StripRing>(s_ens_ring + (threadIdx.x >> 5) * fused::kStripRingDoubles);
    for (int s = 0; s < ep.nsteps; ++s) {
        const int gs = ep.step0 + s;
        // per-problem bookkeeping: t, iteration, dt log, clear the slot two ahead
        if (blockIdx.x == 0) {
            for (int p = threadIdx.x; p < ep.nprob; p += blockDim.x) {
                const Prob& P = probs[p];
                const int it = P.ctl->iter[gs & 1];
                const double dt = ep.fixed_dt ? ep.dts[(int64_t)p * ep.dts_stride + it]
                                              : ep.cfl * (1 / __longlong_as_double((long long)P.ctl->inv_dt_bits[gs % 3]));
                P.ctl->t[(gs + 1) & 1] = P.ctl->t[gs & 1] + dt;
                P.ctl->iter[(gs + 1) & 1] = it + 1;
                P.ctl->last_dt = dt;
                if (P.dt_log && it < P.dt_cap) {
                    P.dt_log[it] = dt;
                }
                P.ctl->inv_dt_bits[(gs + 2) % 3] = 0ull;
            }
        }
        for (int w = wid; w < ep.nitems; w += warps_total) {
            const int p = item_prob[w];
            const Prob& P = probs[p];
            const int it = P.ctl->iter[gs & 1];
            const double dt = ep.fixed_dt ? ep.dts[(int64_t)p * ep.dts_stride + it]
                                          : ep.cfl * (1 / __longlong_as_double((long long)P.ctl->inv_dt_bits[gs % 3]));
            const int local = w - P.item0;
            double inv_max = 0.0;
            int64_t bad_cell = -1;
            const double* qin = ep.seg_mode ? P.q[0] + (int64_t)s * P.seg_stride : P.q[gs & 1];
            double* qout = ep.seg_mode ? P.q[0] + (int64_t)(s + 1) * P.seg_stride : P.q[(gs + 1) & 1];
            fused::strip_work<LIM, RS, 0, 2>(P.g, qin, qout, P.plane, P.pitch, dt, local % P.ncolw, local / P.ncolw, ep.L,
                                       inv_max, bad_cell, ring);
            const bool nan_seen = isnan(inv_max);
            double m = nan_seen ? 0.0 : inv_max;
            m = fused::warp_max_d(m);
            const unsigned nanv = __ballot_sync(0xffffffffu, nan_seen);
            if (lane == 0) {
                atomicMax(&P.ctl->inv_dt_bits[(gs + 1) % 3], dbl_bits(m));
                if (nanv) {
                    atomicMax(&P.ctl->inv_dt_bits[(gs + 1) % 3], 0x7ff8000000000000ull);
                }
            }
            if (bad_cell >= 0) {
                atomicMin(&P.ctl->bad_cell, (unsigned long long)bad_cell);
                P.ctl->err = 4;
                P.ctl->errflag[(gs + 1) & 1] = 1;
                atomicExch(status, 4);
            }
        }
        if (!grid_barrier(barrier, (unsigned)((s + 1) * gridDim.x) + ep.extra_arrivals, status, ep.spin_limit)) {
            return;
        }
    }
}

} // namespace hcl::ensemble
