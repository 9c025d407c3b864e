// bulk.cuh -- TMA bulk copies (cp.async.bulk) between global and shared memory
// with an mbarrier for load completion.  Every wait is bounded: on timeout the
// caller gets `false` and records PIBM_ERR_TIMEOUT instead of hanging.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pibm {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *mb, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mb)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One thread: announce `bytes` and start a global -> shared bulk copy (16-byte multiples, 16-byte aligned).
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *mb) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mb)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst_smem)),
                 "l"(src_gmem), "r"(bytes), "r"(smem_u32(mb))
                 : "memory");
}

// One warp: lane 0 announces n*bytes on mb, then the lanes start n
// global -> shared bulk copies of `bytes` each, copy r from src + r*src_pitch
// to dst + r*dst_pitch (byte pitches; addresses, pitches and bytes 16-byte
// multiples).  The copies complete on mb like one bulk_load of n*bytes.
__device__ __forceinline__ void bulk_load_rows(void *dst, uint32_t dst_pitch, const void *src, size_t src_pitch,
                                               uint32_t bytes, int n, uint64_t *mb) {
    const int lane = threadIdx.x & 31;
    if (lane == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mb)), "r"(bytes * (uint32_t)n)
                     : "memory");
    __syncwarp();
    for (int r = lane; r < n; r += 32)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_u32((char *)dst + (size_t)r * dst_pitch)),
                     "l"((const char *)src + (size_t)r * src_pitch), "r"(bytes), "r"(smem_u32(mb))
                     : "memory");
}

// All threads: wait for the phase with parity `phase` to complete (bounded).
__device__ __forceinline__ bool mbar_wait(uint64_t *mb, uint32_t phase) {
    const uint32_t a = smem_u32(mb);
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(phase)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// One thread: shared -> global bulk store of data the CTA wrote (call after a
// __syncthreads; the proxy fence orders the generic writes before the copy).
__device__ __forceinline__ void bulk_store(void *dst_gmem, const void *src_smem, uint32_t bytes) {
    fence_async_smem();
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem), "r"(smem_u32(src_smem)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// One thread: wait until every committed bulk store has finished reading shared
// memory.  A CTA may exit after it: the global writes complete with the grid.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// One thread: wait until every committed bulk store has completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---- tensor-map (tiled) copies, this GPU's memory only, no multicast ----
// One thread: arrive on mb announcing `bytes` of transaction.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *mb, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mb)), "r"(bytes) : "memory");
}
// One thread: plain arrive (completes a phase that expects no bytes).
__device__ __forceinline__ void mbar_arrive(uint64_t *mb) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mb)) : "memory");
}
// One thread: load the box at element coordinates (x, y, z) of a 3-D tensor
// map into shared memory (completes on mb).  x * element size must be a
// multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, int x, int y, int z, uint64_t *mb) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(mb))
        : "memory");
}
// One thread: store a shared-memory box to coordinates (x, y, z) (bulk group;
// commit with bulk_commit).  Writers of the box fence (fence_async_smem) and
// synchronise with the issuing thread first.
__device__ __forceinline__ void tma_store_3d(const void *tmap, const void *src, int x, int y, int z) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(tmap),
                 "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Barrier over `count` threads (whole warps) on hardware barrier `id` that
// also returns the AND of v over them (the same answer in every thread).
__device__ __forceinline__ bool named_bar_and(int id, int count, bool v) {
    int r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.s32 q, %1, 0;\n\tbar.red.and.pred p, %2, %3, q;\n\tselp.s32 %0, 1, 0, p;\n\t}"
                 : "=r"(r)
                 : "r"((int)v), "r"(id), "r"(count)
                 : "memory");
    return r != 0;
}
// Barrier over `count` threads (whole warps) on hardware barrier `id` (1..15; 0 is __syncthreads').
__device__ __forceinline__ void named_bar_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Programmatic dependent launch: wait until the grids this one depends on
// have completed and their writes are visible (a no-op in a grid launched
// without the programmatic-serialization attribute).  Code before it may
// read only data no earlier kernel of the stream writes.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace pibm
