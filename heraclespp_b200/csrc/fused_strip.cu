// fused_strip.cu -- instantiations of the warp-strip 2-D mixed step for every
// limiter x Riemann solver pair (same flags as fused_mixed.cu).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "fused_strip2d.cuh"
#include "per_device.hpp"
#include "stages.hpp"

namespace hcl::fused {

bool strip2d_eligible(const GridDev& g)
{
    return g.ndim == 2 && g.uniform_cart && g.geom == GEOM_CARTESIAN && g.gravity == GRAV_UNIFORM && g.nfx == 0;
}

// Strips with one or two passive scalars (schedules 3-6 only).
bool strip2d_fx_eligible(const GridDev& g)
{
    return g.ndim == 2 && g.uniform_cart && g.geom == GEOM_CARTESIAN && g.gravity == GRAV_UNIFORM &&
           (g.nfx == 1 || g.nfx == 2);
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda), looked
// up once per process; null when the driver does not offer it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The TMA ring's box starts at column c0 - 2 = ng - 2 + 28 k, which is
// 16-byte aligned for an even ghost width; the box carries the 4 hydro planes.
bool strip2d_tma_eligible(const GridDev& g)
{
    return strip2d_eligible(g) && g.ng % 2 == 0 && tensor_map_encoder() != nullptr;
}

bool encode_tile_map(const GridDev& g, const StateDev& st, int nv, const int box[3], CUtensorMap* map)
{
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || g.ndim < 2 || (reinterpret_cast<uintptr_t>(st.q) & 15u) != 0 || (st.pitch * sizeof(double)) % 16 != 0 ||
        (st.plane * sizeof(double)) % 16 != 0) {
        return false;
    }
    const int rank = g.ndim + 1;
    cuuint64_t dims[4], strides[3];
    cuuint32_t bx[4], estr[4] = {1, 1, 1, 1};
    dims[0] = (cuuint64_t)g.n[0];
    dims[1] = (cuuint64_t)g.n[1];
    bx[0] = (cuuint32_t)box[0];
    bx[1] = (cuuint32_t)box[1];
    strides[0] = (cuuint64_t)st.pitch * sizeof(double);
    if (g.ndim == 3) {
        dims[2] = (cuuint64_t)g.n[2];
        bx[2] = (cuuint32_t)box[2];
        strides[1] = (cuuint64_t)st.pitch * g.n[1] * sizeof(double);
    }
    dims[rank - 1] = (cuuint64_t)nv;
    bx[rank - 1] = (cuuint32_t)nv;
    strides[rank - 2] = (cuuint64_t)st.plane * sizeof(double);
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, st.q, dims, strides, bx, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

namespace {

// dynamic shared memory of the 4-warp strip kernel with nfx passive scalars
// (the rings of one scalar are static)
constexpr int fx_ring_smem(int nfx)
{
    return nfx > 1 ? 4 * 8 * (4 + nfx) * 32 * (int)sizeof(double) : 0;
}

// Resident CTAs of a strip kernel on the current device (`blocks` threads,
// `smem` bytes of dynamic shared memory, opted in first when non-zero),
// computed once per device.
int resident_on_device(PerDevice& cache, const void* fn, int threads, int smem)
{
    int dev = 0;
    cudaGetDevice(&dev);
    return cache.get(dev, [&] {
        if (smem > 0) {
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        }
        int per_sm = 0, nsm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, (size_t)smem);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        return per_sm > 0 && nsm > 0 ? per_sm * nsm : 148;
    });
}

template <int LIM, int RS>
int resident_blocks()
{
    static PerDevice cache;
    return resident_on_device(cache, reinterpret_cast<const void*>(k_strip2d<LIM, RS>), 128, 0);
}

template <int LIM, int RS, int NFX>
int resident_blocks_fx()
{
    static PerDevice cache;
    return resident_on_device(cache, reinterpret_cast<const void*>(k_strip2d<LIM, RS, NFX>), 128, fx_ring_smem(NFX));
}

// Resident CTAs of the in-step strip kernel (one per SM).
template <int LIM, int RS, bool TMA>
int resident_blocks_sync()
{
    static PerDevice cache;
    return resident_on_device(cache, reinterpret_cast<const void*>(k_strip2d_sync<LIM, RS, TMA>),
                              32 * kStripSyncWarps, TMA ? kStripSyncSmemTma : kStripSyncSmem);
}

// 3-D tiled map of a 2-D FP64 state (columns, rows, the 4 hydro planes) with
// the strip ring's box {32 columns, 2 rows, 4 variables}; columns past n0 and
// rows past n1 read as zeros (they feed only lanes and rows that write
// nothing).
bool encode_strip_map(const GridDev& g, const StateDev& st, CUtensorMap* map)
{
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) {
        return false;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)g.n[0], (cuuint64_t)g.n[1], 4};
    const cuuint64_t strides[2] = {(cuuint64_t)st.pitch * sizeof(double), (cuuint64_t)st.plane * sizeof(double)};
    const cuuint32_t box[3] = {32, kTmaBoxRows, 4};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, st.q, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// sync: CTAs of 16 warps marching in step (k_strip2d_sync); otherwise CTAs
// of 4 independent warps (k_strip2d).  L <= 0: strips fitted so that one wave
// of resident warps covers the grid (no warp waits for a second wave).
template <int LIM, int RS>
void launch_lr(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp, int slot,
               int out_buf, int L, bool sync, bool tma, cudaStream_t s)
{
    const int ncolw = (g.nx[0] + kStripLanesOut - 1) / kStripLanesOut;
    const bool fx = g.nfx > 0;
    sync = sync && !fx;
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    tma = tma && sync && strip2d_tma_eligible(g) && encode_strip_map(g, in, &map);
    const int wpb = sync ? kStripSyncWarps : 4;
    const int resident = sync ? (tma ? resident_blocks_sync<LIM, RS, true>() : resident_blocks_sync<LIM, RS, false>())
                              : (fx ? (g.nfx == 2 ? resident_blocks_fx<LIM, RS, 2>() : resident_blocks_fx<LIM, RS, 1>())
                                    : resident_blocks<LIM, RS>());
    if (L <= 0) {
        const int per_col = std::max(1, resident * wpb / ncolw);
        L = std::max(8, (g.nx[1] + per_col - 1) / per_col);
    }
    const int nstrip = (g.nx[1] + L - 1) / L;
    const int warps = ncolw * nstrip;
    const int blocks = std::min((warps + wpb - 1) / wpb, resident);
    if (sync && tma) {
        k_strip2d_sync<LIM, RS, true>
            <<<blocks, 32 * kStripSyncWarps, kStripSyncSmemTma, s>>>(g, in, out, ctl, rp, slot, out_buf, L, map);
    } else if (sync) {
        k_strip2d_sync<LIM, RS, false>
            <<<blocks, 32 * kStripSyncWarps, kStripSyncSmem, s>>>(g, in, out, ctl, rp, slot, out_buf, L, map);
    } else if (fx && g.nfx == 2) {
        k_strip2d<LIM, RS, 2><<<blocks, 128, fx_ring_smem(2), s>>>(g, in, out, ctl, rp, slot, out_buf, L);
    } else if (fx) {
        k_strip2d<LIM, RS, 1><<<blocks, 128, 0, s>>>(g, in, out, ctl, rp, slot, out_buf, L);
    } else {
        k_strip2d<LIM, RS><<<blocks, 128, 0, s>>>(g, in, out, ctl, rp, slot, out_buf, L);
    }
}

template <int LIM>
void launch_l(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp, int slot,
              int out_buf, int L, bool sync, bool tma, cudaStream_t s)
{
    if (g.riemann == RS_HLL) {
        launch_lr<LIM, RS_HLL>(g, in, out, ctl, rp, slot, out_buf, L, sync, tma, s);
    } else if (g.riemann == RS_HLLC) {
        launch_lr<LIM, RS_HLLC>(g, in, out, ctl, rp, slot, out_buf, L, sync, tma, s);
    } else {
        launch_lr<LIM, RS_SPLITTING>(g, in, out, ctl, rp, slot, out_buf, L, sync, tma, s);
    }
}

} // namespace

void step_strip2d(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                  int slot, int out_buf, int L, bool sync, bool tma, cudaStream_t s)
{
    switch (g.limiter) {
    case LIM_CONSTANT:
        launch_l<LIM_CONSTANT>(g, in, out, ctl, rp, slot, out_buf, L, sync, tma, s);
        break;
    case LIM_VANLEER:
        launch_l<LIM_VANLEER>(g, in, out, ctl, rp, slot, out_buf, L, sync, tma, s);
        break;
    case LIM_MINMOD:
        launch_l<LIM_MINMOD>(g, in, out, ctl, rp, slot, out_buf, L, sync, tma, s);
        break;
    default:
        launch_l<LIM_VANALBADA>(g, in, out, ctl, rp, slot, out_buf, L, sync, tma, s);
        break;
    }
    ++g_launches;
}

} // namespace hcl::fused
