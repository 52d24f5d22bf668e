// tma.cuh -- tensor-memory-accelerator (TMA) tile loads into shared memory,
// completed on shared-memory barriers, and the host-side tensor-map
// encoding (sm_100a; loads only, each CTA fetching its own tiles).
//
// Rules the callers keep: the global base is 16-byte aligned, every stride
// is a multiple of 16 bytes, the box's innermost extent in bytes is a
// multiple of 16, and the innermost start coordinate times the element size
// is a multiple of 16 bytes (for doubles: an even x). Out-of-range box cells
// are filled with zeros. Every wait is bounded: a barrier that has not
// completed after kTmaSpinLimit polls sets *err (a plain store: the word may
// be mapped host memory) and the caller goes on (its results are then
// invalid and the host reports the error). A wait still polling after each
// kTmaErrPoll polls reads *err and gives up at once if another wait already
// did, so the remaining waits of a failed launch end quickly.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace tl {

constexpr long kTmaSpinLimit = 1L << 26;
constexpr long kTmaErrPoll = 1L << 20;   // power of two; far beyond any wait of a working copy

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// Orders shared-memory accesses of the generic proxy -- this thread's and,
// after a barrier, the block's -- before the async proxy's next ones.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// Arms `bar` for `bytes` of TMA transactions. Every arming precedes loads
// into a buffer the block's threads may have just read (a ring stage or a
// staging area freed by a barrier), so it first orders those generic reads
// before the async proxy's writes: without the fence a refill could land
// under a late read (observed as rare, run-to-run differences of a staged
// persistent kernel).
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    fence_proxy_async();
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `parity` to complete; false (and *err = 1) after
// `limit` polls.
__device__ __forceinline__ bool mbar_wait_limited(unsigned long long* bar, unsigned parity, int* err, long limit)
{
    for (long n = 0; n < limit; ++n) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((n & (kTmaErrPoll - 1)) == kTmaErrPoll - 1 && err && *(volatile int*)err) break;
    }
    if (err) *(volatile int*)err = 1;
    return false;
}

__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int* err)
{
    return mbar_wait_limited(bar, parity, err, kTmaSpinLimit);
}

// 3D tile load: box of the map at element coordinates (x, y, z) into dst,
// completing `bytes` of transaction count on bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// Host: a 3D map of doubles (esize 8) or floats (esize 4) over an
// (nx, ny, nz) array (x fastest) with the given box, out-of-range cells read
// as zero; false when the driver entry point is missing or the encoding is
// refused (alignment, sizes).
inline bool tma_encode_3d(CUtensorMap* map, const void* base, long nx, long ny, long nz, unsigned bx, unsigned by,
                          unsigned bz, int esize = 8)
{
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<Encode>(fn);
        else
            cudaGetLastError();
    }
    if (!encode) return false;
    if ((reinterpret_cast<unsigned long long>(base) & 15u) != 0 || ((nx * esize) & 15) != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)(nx * esize), (cuuint64_t)(nx * ny * esize)};
    const cuuint32_t box[3] = {bx, by, bz};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUtensorMapDataType dt = esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    return encode(map, dt, 3, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tl
