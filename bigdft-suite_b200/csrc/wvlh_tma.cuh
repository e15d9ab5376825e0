// Tensor-memory-accelerator (TMA) staging of the z kernel's tiles.
//
// A z tile is 32 x 2 columns of a plane stack times the whole z extent; in
// shared memory it is stored z-major, column (y, x) at z * 64 + y * 32 + x,
// which is exactly the dense layout of a TMA box {32, 2, Z, 1} over the
// 4-D tensor (x, y, z, orbital) of a batch's scratch planes.  One thread
// issues the box load (cp.async.bulk.tensor, completion counted in bytes on
// an mbarrier) and, at the end, the box store of the result; elements past
// the plane's edge are zero-filled on load and skipped on store.  No
// multicast is used (the source is this GPU's own memory).
//
// Every wait on the mbarrier is bounded: after kTmaSpinLimit polls the CTA
// records an error in the batch's flag and returns without using the tile.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace wvlh {

constexpr unsigned kTmaSpinLimit = 1u << 26;

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// poll phase `parity` of the barrier at most kTmaSpinLimit times
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
    const unsigned a = smem_addr(bar);
    for (unsigned i = 0; i < kTmaSpinLimit; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// box store from shared memory; the caller fences the generic-proxy writes
// (fence_async_smem) and a barrier precedes the call
__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3, const void *src)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];\n" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}

// the issuing thread waits until the stores have read shared memory
__device__ __forceinline__ void tma_store_drain() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }

// shared-memory writes by ordinary stores become visible to the TMA unit
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Host: encode a 4-D map (x, y, z, orbital) over a batch's scratch planes,
// box {32, 2, Z, 1}; false when the shapes or alignments do not allow TMA.
bool encode_tile_map(CUtensorMap *map, const void *base, int elem_bytes, long long W, long long H, long long Z,
                     long long norb, long long orb_stride_elems);

}  // namespace wvlh
