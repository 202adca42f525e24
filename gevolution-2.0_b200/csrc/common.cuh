// common.cuh -- shared types and helpers for the sm_100a PM-cycle kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gev {

// ---------------------------------------------------------------------------
// precision traits: R is the field/FFT type (float in mixed mode, double in FP64)
// ---------------------------------------------------------------------------
template <class R> struct CT;
template <> struct CT<float> { using C = float2; };
template <> struct CT<double> { using C = double2; };

__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <class C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <class C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <class C> __device__ __forceinline__ C cmul(C a, C b)
{
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <class C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <class C, class S> __device__ __forceinline__ C cscale(C a, S s) { a.x *= s; a.y *= s; return a; }
// multiply by s*i (s = +1 or -1)
template <int S, class C> __device__ __forceinline__ C cmul_si(C a)
{
    C r;
    if (S > 0) { r.x = -a.y; r.y = a.x; }
    else { r.x = a.y; r.y = -a.x; }
    return r;
}

// ---------------------------------------------------------------------------
// lattice geometry.  Real fields: x + N*(y + N*z).  Fourier fields (half
// spectrum along x): kx + PP*(ky + N*kz), kx < P = N/2 + 1, with the even row
// pitch PP = N/2 + 2.
// Particle tiles: 8^3 cells; a particle's bucket is 8*tile + class, where the
// class bits mark cells on the tile's upper faces (x, y, z == 7) whose
// particles also deposit into the next tile along that axis.
// ---------------------------------------------------------------------------
constexpr int TILE = 8;

struct Geom {
    int N;
    int P;        // N/2 + 1
    int PP;       // N/2 + 2, row pitch of the Fourier arrays
    int nt;       // tiles per side
    int64_t n3;   // N^3
    int64_t nk;   // PP*N*N
    int64_t ntiles;
};

__host__ __device__ __forceinline__ int wrapi(int i, int N) { return i < 0 ? i + N : (i >= N ? i - N : i); }

// Division of 32-bit unsigned values by a divisor fixed at launch time, as a
// multiply-high and a shift (Granlund & Montgomery, "Division by invariant
// integers using multiplication", 1994: with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, n / d = (umulhi(m, n) + n) >> l, exact
// for every 32-bit n).  Replaces the runtime-divisor division sequence in the
// per-particle cell decode.
struct FastDiv {
    uint32_t d, m;
    int l;
    FastDiv() = default;
    __host__ explicit FastDiv(uint32_t div) : d(div)
    {
        l = 0;
        while ((1ull << l) < div) l++;
        m = (uint32_t)((((1ull << l) - div) << 32) / div + 1);
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const
    {
#ifdef __CUDA_ARCH__
        const uint32_t hi = __umulhi(m, n);
#else
        const uint32_t hi = (uint32_t)(((uint64_t)m * n) >> 32);
#endif
        return (uint32_t)(((uint64_t)hi + n) >> l);
    }
};

// cell index x + N*(y + N*z) -> (x, y, z)
__host__ __device__ __forceinline__ void decode_cell(uint32_t cell, const FastDiv &fN, int &x, int &y, int &z)
{
    const uint32_t q = fN.div(cell);
    x = (int)(cell - q * fN.d);
    z = (int)fN.div(q);
    y = (int)(q - (uint32_t)z * fN.d);
}

__host__ __device__ __forceinline__ int64_t sidx(int N, int x, int y, int z)
{
    return (int64_t)x + (int64_t)N * ((int64_t)y + (int64_t)N * (int64_t)z);
}

__host__ __device__ __forceinline__ uint32_t bucket_of_cell(int N, int nt, int x, int y, int z)
{
    int tx = x >> 3, ty = y >> 3, tz = z >> 3;
    uint32_t cls = ((x & 7) == 7 ? 1u : 0u) | ((y & 7) == 7 ? 2u : 0u) | ((z & 7) == 7 ? 4u : 0u);
    uint32_t tile = (uint32_t)tx + (uint32_t)nt * ((uint32_t)ty + (uint32_t)nt * (uint32_t)tz);
    return tile * 8u + cls;
}

// Raises a kernel's dynamic shared-memory limit once per device: the attribute
// belongs to the current device, so a process with contexts on several GPUs
// sets it on each.  done: the call site's flags, one per device ordinal.
constexpr int SMEM_ATTR_DEVICES = 64;
template <class K> inline void raise_smem_limit(K kernel, size_t bytes, bool (&done)[SMEM_ATTR_DEVICES])
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SMEM_ATTR_DEVICES) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        return;
    }
    if (!done[dev]) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        done[dev] = true;
    }
}

// x-pass load modes (fused source preparation)
enum { FX_COPY = 0, FX_PREP_T00 = 1, FX_PREP_TIJ = 2, FX_PREP_T0I = 3 };
// z-pass Fourier-space operators
enum { OP_POISSON = 0, OP_SCALAR = 1, OP_VECTOR = 2, OP_BIN = 3, OP_ZELD = 4, OP_ICS = 5 };
// optional extras of OP_SCALAR
enum { EXTRA_TENSOR_PROJECT = 1, EXTRA_TENSOR_EVOLVE = 2, EXTRA_VECTOR_EVOLVE = 4 };

// device error word bits (read back by the host at synchronising calls)
constexpr int ERR_NONFINITE = 1;       // a particle coordinate became non-finite
constexpr int ERR_LC_OVERFLOW = 2;     // lightcone output exceeded its capacity
constexpr int ERR_BAD_CELL = 4;        // a particle cell index outside the lattice
constexpr int ERR_TMA_TIMEOUT = 8;     // a bulk tensor copy did not complete within the wait limit
constexpr int ERR_BAD_ORDER = 16;      // a deposit found a cell's particles not contiguous in their bucket
constexpr int ERR_DOMAIN = 32;         // a tabulated function was evaluated outside its table

// kernel launch helper
inline unsigned int cdiv(int64_t a, int64_t b) { return (unsigned int)((a + b - 1) / b); }

}  // namespace gev
