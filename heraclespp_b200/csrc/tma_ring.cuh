// tma_ring.cuh -- TMA staging helpers (sm_100a): the row rings of the
// warp-strip kernels and the tile + halo box of the fused tile kernels.
//
// A warp's row ring (4 slots of two x-row segments: 4 variables x 2 rows x 32
// doubles, 2 KB) is filled by the Tensor Memory Accelerator: one lane issues a
// single 3-D cp.async.bulk.tensor per pair of rows (box {32 doubles, 2 rows,
// 4 variables} of the FP64 state, whose planes are the tensor's third
// dimension), and completion is tracked by one mbarrier per slot (expect-tx
// of the box's bytes).  The lanes wait on the slot's mbarrier phase before
// reading it.  The tensor map covers this GPU's own state buffer only and the
// copies carry no cluster multicast.
//
// Every wait is bounded: after kTmaWaitPolls failed polls it gives up and
// reports false, and the kernel records HCL_ERR_TIMEOUT instead of hanging.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace hcl::fused {

// one ring slot: 32 lanes x 2 rows x 4 variables of FP64
constexpr unsigned kTmaBoxRows = 2u;
constexpr unsigned kTmaBoxBytes = 4u * kTmaBoxRows * 32u * 8u;
// polls of one mbarrier wait before it gives up (each try_wait also
// suspends the thread for a hardware-defined time)
constexpr int kTmaWaitPolls = 1 << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes initialised mbarriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One box of a 3-D tiled tensor map into shared memory; completes `bar`'s
// transaction count.  x * 8 bytes must be a multiple of 16 (x even for FP64).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// One box of a 4-D tiled tensor map (x * 8 bytes a multiple of 16).
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z,
                                            int w)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6}], [%2];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map)
{
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// On shared-memory addresses computed once: one box into shared memory by
// one elected lane of the (converged) warp:
// expect-tx on the slot's mbarrier and the copy, both predicated on the
// election, so the warp takes no divergent branch.  The proxy fence orders
// the warp's earlier generic reads of the slot before the async write.
__device__ __forceinline__ void tma_box_elected(unsigned dst, const CUtensorMap* map, unsigned bar, unsigned bytes,
                                                int x, int y, int z)
{
    asm volatile(
        "{\n"
        " .reg .pred P;\n"
        " .reg .b32 L;\n"
        " elect.sync L|P, 0xffffffff;\n"
        " @P fence.proxy.async.shared::cta;\n"
        " @P mbarrier.arrive.expect_tx.shared::cta.b64 _, [%2], %3;\n"
        " @P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%4, %5, "
        "%6}], [%2];\n"
        "}\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(bytes), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_s(unsigned bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0u;
}
__device__ __forceinline__ bool mbar_wait_bounded_s(unsigned bar, unsigned parity)
{
    for (int i = 0; i < kTmaWaitPolls; ++i) {
        if (mbar_try_wait_s(bar, parity)) {
            return true;
        }
    }
    return false;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Waits for the phase of `bar` with the given parity to complete; false when
// kTmaWaitPolls polls were not enough.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) {
        return true;
    }
    for (int i = 1; i < kTmaWaitPolls; ++i) {
        if (mbar_try_wait(bar, parity)) {
            return true;
        }
    }
    return false;
}

} // namespace hcl::fused
