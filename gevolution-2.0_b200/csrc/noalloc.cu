// noalloc.cu -- gev_poisson_noalloc: the Poisson solve of the phi update on
// caller-owned device arrays, with all scratch in static device memory.
//
// Why it exists: gev_solve_phi works on fields that a context allocated.  Some
// callers cannot allocate device memory at the point where they want the
// solve: a host code that owns every device buffer through its own memory
// pool (a caching allocator that must see every allocation), or a caller in
// the middle of recording work into a stream where a cudaMalloc would either
// synchronise the device or be refused.  This entry point takes the source and
// the output as plain device pointers and keeps its one large temporary -- the
// complex half spectrum of the transform -- in a file-scope __device__ array
// of fixed size, so a call launches kernels and nothing else.
//
// Limits and rules (the same text is in include/gev.h):
//   * N in {16, 32, 64, 128}: the static scratch holds the half spectrum of a
//     128^3 grid in FP64 (N/2+2)*N*N*16 bytes = 17,301,504 bytes, plus the FFT
//     and k tables and one error word.  Larger N is rejected with GEV_ERR_SIZE.
//   * Nothing in the scratch has to start at zero: every call first writes the
//     tables, clears the error word and then writes the whole spectrum before
//     any of it is read.
//   * There is one scratch per device, shared by every caller of this entry
//     point in the process: two calls on the same device whose work overlaps
//     in time (different streams, no ordering between them) race on it.
//     Order such calls on one stream or synchronise between them.
//   * The host needs the device address of the scratch: the first call on a
//     device (and the first call after that device's context was destroyed and
//     re-created, e.g. by cudaDeviceReset) looks it up with
//     cudaGetSymbolAddress, which can also load the library's device code;
//     make that first call before any stream capture begins.
//   * A bulk tensor copy of the y or z pass that does not complete within its
//     wait limit sets the error word; the last kernel of the call then fills
//     phi with NaN, so the failure shows in the output without a
//     synchronising status read (the next call clears the word).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "gev.h"
#include "kernels.h"

namespace gev {
namespace {

constexpr int NA_MAX_N = 128;
constexpr size_t na_align(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t NA_SPEC_BYTES = na_align((size_t)(NA_MAX_N / 2 + 2) * NA_MAX_N * NA_MAX_N * sizeof(double2));
constexpr size_t NA_TWF_BYTES = na_align((size_t)NA_MAX_N * sizeof(double2));
constexpr size_t NA_TWH_BYTES = na_align((size_t)(NA_MAX_N / 2) * sizeof(double2));
constexpr size_t NA_K2_BYTES = na_align((size_t)NA_MAX_N * sizeof(double));
constexpr size_t NA_KS_BYTES = na_align((size_t)NA_MAX_N * sizeof(double2));
constexpr size_t NA_ERR_BYTES = na_align(sizeof(int));
constexpr size_t NA_SCRATCH_BYTES = NA_SPEC_BYTES + NA_TWF_BYTES + NA_TWH_BYTES + NA_K2_BYTES + NA_KS_BYTES + NA_ERR_BYTES;

static __device__ __align__(256) unsigned char na_scratch[NA_SCRATCH_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex na_mutex;
// per device: the scratch address and the unique id of the context it was
// resolved in (a device address is only valid inside its own context)
struct NaSlot {
    unsigned long long ctx_id = 0;
    void *ptr = nullptr;
};
NaSlot na_slot[NA_MAX_DEVICES];

// the unique id of the calling thread's current context (0 if there is none)
int na_current_context_id(unsigned long long *id)
{
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    if (!get_current || !get_id) {
        void *p1 = nullptr, *p2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p1, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess || !p1 ||
            cudaGetDriverEntryPoint("cuCtxGetId", &p2, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess || !p2)
            return GEV_ERR_CUDA;
        get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p1);
        get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p2);
    }
    CUcontext cur = nullptr;
    if (get_current(&cur) != CUDA_SUCCESS) return GEV_ERR_CUDA;
    *id = 0;
    if (cur && get_id(cur, id) != CUDA_SUCCESS) return GEV_ERR_CUDA;
    return GEV_OK;
}

// device address of the scratch in the current context of device `dev`,
// resolved once per context
int na_scratch_address(int dev, unsigned char **base)
{
    std::lock_guard<std::mutex> lock(na_mutex);
    unsigned long long id = 0;
    if (na_current_context_id(&id) != GEV_OK) return GEV_ERR_CUDA;
    NaSlot &s = na_slot[dev];
    if (id == 0 || !s.ptr || s.ctx_id != id) {
        void *p = nullptr;
        // makes the device's primary context current if no context is yet
        if (cudaGetSymbolAddress(&p, na_scratch) != cudaSuccess || !p) return GEV_ERR_CUDA;
        if (na_current_context_id(&id) != GEV_OK || id == 0) return GEV_ERR_CUDA;
        s.ptr = p;
        s.ctx_id = id;
    }
    *base = static_cast<unsigned char *>(s.ptr);
    return GEV_OK;
}

// FFT twiddles and the k tables of gevolution.hpp:269-275 for grid size N
template <class R>
__global__ void k_na_tables(int N, typename CT<R>::C *tw_full, typename CT<R>::C *tw_half, double *k2, double2 *ks, int *err)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) *err = 0;
    if (k >= N) return;
    double s, c;
    sincospi(2.0 * (double)k / (double)N, &s, &c);   // exp(-2 pi i k / N)
    tw_full[k] = mk((R)c, (R)-s);
    if (k < N / 2) {
        sincospi(4.0 * (double)k / (double)N, &s, &c);   // exp(-2 pi i k / (N/2))
        tw_half[k] = mk((R)c, (R)-s);
    }
    sincospi((double)k / (double)N, &s, &c);
    const double gk = 2.0 * (double)N * s;
    k2[k] = gk * gk;
    ks[k] = make_double2(gk * c, -gk * s);
}

// a Fourier pass gave up waiting for its data: phi is not the solution, so
// it becomes NaN everywhere (the next call's table kernel clears the word)
template <class R>
__global__ void k_na_poison(const int *err, R *dst, int64_t n3)
{
    if (*err == 0) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (R)NAN;
}

template <class R>
int na_solve(int N, const R *src, R *dst, double coeff, double modif, unsigned char *base, cudaStream_t st)
{
    using C = typename CT<R>::C;
    C *spec = reinterpret_cast<C *>(base);
    C *twf = reinterpret_cast<C *>(base + NA_SPEC_BYTES);
    C *twh = reinterpret_cast<C *>(base + NA_SPEC_BYTES + NA_TWF_BYTES);
    double *k2 = reinterpret_cast<double *>(base + NA_SPEC_BYTES + NA_TWF_BYTES + NA_TWH_BYTES);
    double2 *ks = reinterpret_cast<double2 *>(base + NA_SPEC_BYTES + NA_TWF_BYTES + NA_TWH_BYTES + NA_K2_BYTES);
    int *err = reinterpret_cast<int *>(base + NA_SPEC_BYTES + NA_TWF_BYTES + NA_TWH_BYTES + NA_K2_BYTES + NA_KS_BYTES);
    const int64_t n3 = (int64_t)N * N * N, nk = (int64_t)(N / 2 + 2) * N * N;   // Fourier rows of pitch N/2+2

    k_na_tables<R><<<cdiv(N, 128), 128, 0, st>>>(N, twf, twh, k2, ks, err);
    const FftTables<R> tb{twf, twh, k2, ks};
    // same pass sequence as the context's phi update without prepareFTsource
    fx_forward<R>(N, FX_COPY, src, n3, 1, 0, nullptr, nullptr, 0.0, 0.0, 0.0, 0.0, spec, nk, nullptr, tb, st);
    fy_pass<R>(N, -1, spec, nk, 1, err, tb, st);
    FzParams fp{};
    fp.op = OP_POISSON;
    fp.p0 = coeff / -((double)N * (double)N * (double)N);
    fp.p1 = modif;
    fp.phi_hom = nullptr;
    fp.err = err;
    fz_pass<R>(N, fp, spec, nk, nullptr, nullptr, nullptr, tb, st);
    fy_pass<R>(N, 1, spec, nk, 1, err, tb, st);
    fx_inverse<R>(N, spec, nk, dst, n3, 1, tb, st);
    k_na_poison<R><<<(unsigned)std::min<int64_t>(cdiv(n3, 256), 148 * 8), 256, 0, st>>>(err, dst, n3);
    return cudaGetLastError() == cudaSuccess ? GEV_OK : GEV_ERR_CUDA;
}

}  // namespace
}  // namespace gev

extern "C" int gev_poisson_noalloc(int32_t N, int32_t precision, const void *source, void *phi, double poisson_coeff,
                                   double modif, void *stream)
{
    using namespace gev;
    if (!source || !phi || (precision != GEV_FP64 && precision != GEV_MIXED)) return GEV_ERR_ARG;
    if (N != 16 && N != 32 && N != 64 && N != 128) {
        if (N == 256 || N == 384 || N == 512 || N == 768) return GEV_ERR_SIZE;
        return GEV_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GEV_ERR_CUDA;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return GEV_ERR_ARG;
    unsigned char *base = nullptr;
    if (na_scratch_address(dev, &base) != GEV_OK) return GEV_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        if (precision == GEV_FP64)
            return na_solve<double>(N, static_cast<const double *>(source), static_cast<double *>(phi), poisson_coeff,
                                    modif, base, st);
        return na_solve<float>(N, static_cast<const float *>(source), static_cast<float *>(phi), poisson_coeff, modif,
                               base, st);
    } catch (...) {
        return GEV_ERR_CUDA;
    }
}
