// tma.cuh -- tensor-memory-access (TMA) staging helpers for sm_100a: tensor
// maps of the Fourier arrays, bulk tensor copies global <-> shared, and the
// shared-memory transaction barrier that the loads complete on.
//
// Rules the callers keep (the hardware does not check them at run time):
//   * the innermost coordinate times the element size is a multiple of 16
//     bytes (the Fourier maps count reals, so kx0 must be even);
//   * stores start at non-negative coordinates (elements beyond the tensor's
//     extent are not written);
//   * shared-memory destinations are 128-byte aligned;
//   * no multicast: every CTA loads its own tiles.
#pragma once

#include <cuda.h>   // CUtensorMap and its enums (types only; the encoder comes from the runtime)
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <stdexcept>

#include "common.cuh"

namespace gev {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Wait for phase `parity` of the barrier; gives up (returns false) after a
// bounded number of polls, each of which suspends for at most the hardware's
// own short time limit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < (1 << 22); it++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// global -> shared tile of a 4-D tensor map; completes bytes on `bar`
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "r"(smem_u32(bar))
        : "memory");
}

// shared -> global tile of a 4-D tensor map (bulk group of the issuing thread)
__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3, const void *src)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
                 : "memory");
}

// the issuing thread's bulk stores have finished reading shared memory
__device__ __forceinline__ void tma_store_drain()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// shared-memory writes of this thread become visible to the bulk-copy engine
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

inline PFN_cuTensorMapEncodeTiled_v12000 tma_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            throw std::runtime_error("cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// A Fourier array (rows of P = N/2+1 complex values at the pitch N/2+2,
// components `nk` complex values apart) as the 4-D tensor
// {2P reals, ky, kz, component}; box {2T reals, yb, zb, 1}.
template <class R>
CUtensorMap fourier_tensor_map(const void *base, int N, int64_t nk, int ncomp, int T, int yb, int zb)
{
    CUtensorMap m;
    const cuuint64_t row = (cuuint64_t)(N / 2 + 2) * 2 * sizeof(R);
    const cuuint64_t dims[4] = {(cuuint64_t)2 * (N / 2 + 1), (cuuint64_t)N, (cuuint64_t)N, (cuuint64_t)ncomp};
    const cuuint64_t strides[3] = {row, row * (cuuint64_t)N, (cuuint64_t)nk * 2 * sizeof(R)};
    const cuuint32_t box[4] = {(cuuint32_t)(2 * T), (cuuint32_t)yb, (cuuint32_t)zb, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = tma_encoder()(&m, sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                                     4, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("tensor map encoding failed");
    return m;
}

}  // namespace gev
