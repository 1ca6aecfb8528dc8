// Thin inline-PTX wrappers for the sm_100a Tensor Memory Accelerator (TMA)
// and shared-memory mbarriers, plus host-side tensor-map creation through the
// driver entry point (no link-time dependency on libcuda).
//
// Only plain (non-multicast) tiled loads and stores are used, always on this
// GPU's own memory.  Every wait on an mbarrier is bounded in time: once the
// global nanosecond timer has advanced by the caller's limit the waiting
// thread records SPM_DEVERR_TIMEOUT in the device error word and gives up.
#pragma once

#include <cuda.h>

#include "spm_common.cuh"

namespace spm {

constexpr unsigned int       SPM_DEVERR_TIMEOUT = 1u << 4;
constexpr unsigned long long kWaitLimitNs       = 1000000000ull;  // default bound of one wait: 1 s

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Wait for phase `parity` of an mbarrier for at most limit_ns nanoseconds of
// the global timer.  Returns false on timeout (and records it in *err when
// err is given).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned int *err,
                                          unsigned long long limit_ns) {
    const unsigned           a  = smem_addr(bar);
    const unsigned long long t0 = global_ns();
    for (;;) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > limit_ns) break;
    }
    if (err) atomicOr(err, SPM_DEVERR_TIMEOUT);
    return false;
}

// 4D tiled TMA load global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// 4D tiled TMA store shared -> global (bulk async group).
__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                             const void *src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until at most N bulk groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// Wait until all bulk groups completed (writes visible).
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// 16-byte asynchronous global -> shared copy (both addresses 16-byte
// aligned), its commit and a wait for all of this thread's copies.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Host: tensor maps
// ---------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void                           *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 4D map over a field array of element type T (float/double), dims given
// innermost first in elements, strides (dims 1..3) in bytes.
template <typename T>
inline bool make_map_4d(CUtensorMap *map, void *base, const uint64_t dims[4], const uint64_t strides_bytes[3],
                        const uint32_t box[4]) {
    EncodeTiledFn fn = encode_tiled_fn();
    if (!fn) return false;
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const CUresult r = fn(map, dt, 4, base, reinterpret_cast<const cuuint64_t *>(dims),
                          reinterpret_cast<const cuuint64_t *>(strides_bytes), reinterpret_cast<const cuuint32_t *>(box),
                          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace spm
