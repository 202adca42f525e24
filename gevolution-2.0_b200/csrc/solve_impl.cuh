// solve_impl.cuh -- launchers of the pencil passes for every supported grid
// size; included once per precision (solve_f32.cu, solve_f64.cu).
#pragma once

#include <algorithm>
#include <stdexcept>

#include "fftpass.cuh"
#include "kernels.h"

namespace gev {

// Tile shapes of the pencil passes (FP32 values; FP64 uses half the columns).
#ifndef GEV_TX_F
#define GEV_TX_F 16
#endif
#ifndef GEV_TY_F
#define GEV_TY_F 16
#endif
#ifndef GEV_TZ1_F
#define GEV_TZ1_F 8
#endif
#ifndef GEV_TZ3_F
#define GEV_TZ3_F 4
#endif
#ifndef GEV_TZ6_F
#define GEV_TZ6_F 4
#endif
#ifndef GEV_NT_Y
#define GEV_NT_Y 512
#endif
#ifndef GEV_NT_Z
#define GEV_NT_Z 256
#endif
#ifndef GEV_FY_TMA
#define GEV_FY_TMA 1     // y pass staged by bulk tensor copies
#endif
#ifndef GEV_FZ_TMA
#define GEV_FZ_TMA 1     // z pass staged by bulk tensor copies
#endif
#ifndef GEV_TZC_F
#define GEV_TZC_F 4      // columns of the contracted scalar z pass
#endif
#ifndef GEV_TIJ6_T_F
#define GEV_TIJ6_T_F 4   // rows of the six-component Tij x pass
#endif
template <class R> struct PassCfg {
    static constexpr int TX = sizeof(R) == 4 ? GEV_TX_F : GEV_TX_F / 2;     // rows per x-pass CTA
    static constexpr int TY = sizeof(R) == 4 ? GEV_TY_F : GEV_TY_F / 2;     // columns per y-pass CTA
    static constexpr int TZ1 = sizeof(R) == 4 ? GEV_TZ1_F : GEV_TZ1_F / 2;  // Poisson
    static constexpr int TZ3 = sizeof(R) == 4 ? GEV_TZ3_F : GEV_TZ3_F / 2;  // vector
    static constexpr int TZ6 = sizeof(R) == 4 ? GEV_TZ6_F : GEV_TZ6_F / 2;  // scalar / tensor
    static constexpr int NTY = GEV_NT_Y;                                    // threads per y-pass CTA
    static constexpr int NTZ = GEV_NT_Z;                                    // threads per z-pass CTA
    static constexpr int TZC = sizeof(R) == 4 ? GEV_TZC_F : GEV_TZC_F / 2;  // contracted scalar
    static constexpr int TIJ6 = sizeof(R) == 4 ? GEV_TIJ6_T_F : GEV_TIJ6_T_F / 2;
};

// CTAs of `bytes` dynamic shared memory that fit one SM (228 KB, 1 KB reserved per CTA)
constexpr int smem_ctas(size_t bytes) { return (int)(233472 / (bytes + 1024)); }

template <class K> inline void set_smem(K kernel, size_t bytes)
{
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

#define GEV_SWITCH_N(N, CALL)                          \
    switch (N) {                                       \
    case 16: { constexpr int NN = 16; CALL; } break;   \
    case 32: { constexpr int NN = 32; CALL; } break;   \
    case 64: { constexpr int NN = 64; CALL; } break;   \
    case 128: { constexpr int NN = 128; CALL; } break; \
    case 256: { constexpr int NN = 256; CALL; } break; \
    case 384: { constexpr int NN = 384; CALL; } break; \
    case 512: { constexpr int NN = 512; CALL; } break; \
    case 768: { constexpr int NN = 768; CALL; } break; \
    default: throw std::runtime_error("unsupported grid size"); \
    }

template <class R, int N, int MODE>
void fx_fwd_n(const FxArgs<R> &a, int ncomp, int64_t in_stride, int64_t out_stride, const FftTables<R> &tb, cudaStream_t st)
{
    using C = typename CT<R>::C;
    constexpr int T = PassCfg<R>::TX, NT = 256;
    size_t smem = (size_t)(N / 2) * (T + 1) * sizeof(C);
    auto k = k_fx_fwd<R, N, T, NT, MODE>;
    set_smem(k, smem);
    k<<<dim3(N / T, N, ncomp), NT, smem, st>>>(a, in_stride, out_stride, tb.tw_half, tb.tw_full);
}

template <class R, int N>
void fx_tij6_n(const FxArgs<R> &a, int64_t in_stride, int64_t out_stride, const FftTables<R> &tb, cudaStream_t st)
{
    using C = typename CT<R>::C;
    constexpr int T = PassCfg<R>::TIJ6, NT = 256;
    size_t smem = (size_t)(N / 2) * (6 * T + 1) * sizeof(C);
    auto k = k_fx_fwd_tij6<R, N, T, NT>;
    set_smem(k, smem);
    k<<<dim3(N / T, N), NT, smem, st>>>(a.in, in_stride, a.phi, a.c, a.out, out_stride, tb.tw_half, tb.tw_full);
}

template <class R>
void fx_forward(int N, int mode, const R *in, int64_t in_stride, int ncomp, int comp0, const R *phi, const R *chi,
                double bg, double c, double c2, double c3, typename CT<R>::C *out, int64_t out_stride,
                double *partial, const FftTables<R> &tb, cudaStream_t st)
{
    FxArgs<R> a;
    a.in = in; a.phi = phi; a.chi = chi;
    a.bg = bg; a.c = c; a.c2 = c2; a.c3 = c3;
    a.comp0 = comp0; a.out = out; a.partial = partial;
    if (mode == FX_COPY) { GEV_SWITCH_N(N, (fx_fwd_n<R, NN, FX_COPY>(a, ncomp, in_stride, out_stride, tb, st))) }
    else if (mode == FX_PREP_T00) { GEV_SWITCH_N(N, (fx_fwd_n<R, NN, FX_PREP_T00>(a, ncomp, in_stride, out_stride, tb, st))) }
    else if (mode == FX_PREP_T0I) { GEV_SWITCH_N(N, (fx_fwd_n<R, NN, FX_PREP_T0I>(a, ncomp, in_stride, out_stride, tb, st))) }
    else if (ncomp == 6 && comp0 == 0) { GEV_SWITCH_N(N, (fx_tij6_n<R, NN>(a, in_stride, out_stride, tb, st))) }
    else { GEV_SWITCH_N(N, (fx_fwd_n<R, NN, FX_PREP_TIJ>(a, ncomp, in_stride, out_stride, tb, st))) }
}

template <class R, int N, int S>
void fy_n(typename CT<R>::C *data, int64_t stride, int ncomp, int *err, const FftTables<R> &tb, cudaStream_t st)
{
    using C = typename CT<R>::C;
    constexpr int T = PassCfg<R>::TY, NT = PassCfg<R>::NTY;
#if GEV_FY_TMA
    const size_t smem = (size_t)N * T * sizeof(C) + 128;
    const CUtensorMap map = fourier_tensor_map<R>(data, N, stride, ncomp, T, ZBox<N>::ZB, 1);
    auto k = k_fy_tma<R, N, T, NT, S>;
    set_smem(k, smem);
    k<<<dim3((N / 2 + 1 + T - 1) / T, N, ncomp), NT, smem, st>>>(tb.tw_full, err, map);
#else
    size_t smem = (size_t)N * (T + 1) * sizeof(C);
    auto k = k_fy<R, N, T, NT, S>;
    set_smem(k, smem);
    k<<<dim3((N / 2 + 1 + T - 1) / T, N, ncomp), NT, smem, st>>>(data, stride, tb.tw_full);
#endif
}

template <class R>
void fy_pass(int N, int sign, typename CT<R>::C *data, int64_t stride, int ncomp, int *err, const FftTables<R> &tb,
             cudaStream_t st)
{
    if (sign < 0) { GEV_SWITCH_N(N, (fy_n<R, NN, -1>(data, stride, ncomp, err, tb, st))) }
    else { GEV_SWITCH_N(N, (fy_n<R, NN, 1>(data, stride, ncomp, err, tb, st))) }
}

template <class R, int N>
void fxi_n(const typename CT<R>::C *in, int64_t in_stride, R *out, int64_t out_stride, int ncomp, const FftTables<R> &tb,
           cudaStream_t st)
{
    using C = typename CT<R>::C;
    constexpr int T = PassCfg<R>::TX, NT = 256;
    size_t smem = (size_t)(N / 2) * (T + 1) * sizeof(C);
    auto k = k_fx_inv<R, N, T, NT>;
    set_smem(k, smem);
    k<<<dim3(N / T, N, ncomp), NT, smem, st>>>(in, in_stride, out, out_stride, tb.tw_half, tb.tw_full);
}

template <class R>
void fx_inverse(int N, const typename CT<R>::C *in, int64_t in_stride, R *out, int64_t out_stride, int ncomp,
                const FftTables<R> &tb, cudaStream_t st)
{
    GEV_SWITCH_N(N, (fxi_n<R, NN>(in, in_stride, out, out_stride, ncomp, tb, st)))
}

template <class R, int N, int OP, int EXTRA>
void fz_n(const FzArgs<R> &a, const FftTables<R> &tb, cudaStream_t st)
{
    using C = typename CT<R>::C;
    constexpr int T = OpShape<OP, EXTRA>::CONTRACT ? PassCfg<R>::TZC
                      : (OP == OP_POISSON || OP == OP_BIN || OP == OP_ICS) ? PassCfg<R>::TZ1
                      : ((OP == OP_VECTOR || OP == OP_ZELD) ? PassCfg<R>::TZ3 : PassCfg<R>::TZ6);
    constexpr int NT = PassCfg<R>::NTZ;
#if GEV_FZ_TMA
    static_assert(T % 2 == 0 || sizeof(R) == 8, "TMA boxes need 16-byte rows");
    constexpr int CMAX = OpShape<OP, EXTRA>::CMAX;
    constexpr int CTMA = OpShape<OP, EXTRA>::CTMA;
    constexpr size_t dense = (size_t)CTMA * N * T * sizeof(C) + 128;
    constexpr size_t padded = (size_t)CTMA * (N + N / 8) * T * sizeof(C) + 128;
    // padded rows where they spread the banks, keep every component buffer on
    // a 128-byte boundary, and cost no resident CTA
    constexpr bool PAD = pad_helps<T, C>() && ((N + N / 8) * T * sizeof(C)) % 128 == 0 &&
                         smem_ctas(padded) >= std::min(FzMinBlocks<R, OP, EXTRA, NT>::v, smem_ctas(dense));
    const size_t smem = PAD ? padded : dense;
    const CUtensorMap map = fourier_tensor_map<R>(a.data, N, a.stride, CMAX, T, 1, ZBox<N>::ZB);
    auto k = k_fz_tma<R, N, T, NT, OP, EXTRA, PAD>;
    set_smem(k, smem);
    k<<<dim3((N / 2 + 1 + T - 1) / T, N), NT, smem, st>>>(a, tb.tw_full, map);
#else
    constexpr int CBUF = OpShape<OP, EXTRA>::CBUF;
    size_t smem = (size_t)N * (CBUF * T + 1) * sizeof(C);
    auto k = k_fz<R, N, T, NT, OP, EXTRA>;
    set_smem(k, smem);
    k<<<dim3((N / 2 + 1 + T - 1) / T, N), NT, smem, st>>>(a, tb.tw_full);
#endif
}

template <class R, int N>
void fz_dispatch(const FzParams &fp, const FzArgs<R> &a, const FftTables<R> &tb, cudaStream_t st)
{
    if (fp.op == OP_POISSON) fz_n<R, N, OP_POISSON, 0>(a, tb, st);
    else if (fp.op == OP_ZELD) fz_n<R, N, OP_ZELD, 0>(a, tb, st);
    else if (fp.op == OP_ICS) fz_n<R, N, OP_ICS, 0>(a, tb, st);
    else if (fp.op == OP_BIN) fz_n<R, N, OP_BIN, 0>(a, tb, st);
    else if (fp.op == OP_VECTOR) fz_n<R, N, OP_VECTOR, 0>(a, tb, st);
    else {
        switch (fp.extra) {
        case 0: fz_n<R, N, OP_SCALAR, 0>(a, tb, st); break;
        case EXTRA_TENSOR_PROJECT: fz_n<R, N, OP_SCALAR, EXTRA_TENSOR_PROJECT>(a, tb, st); break;
        case EXTRA_TENSOR_EVOLVE: fz_n<R, N, OP_SCALAR, EXTRA_TENSOR_EVOLVE>(a, tb, st); break;
        case EXTRA_VECTOR_EVOLVE: fz_n<R, N, OP_SCALAR, EXTRA_VECTOR_EVOLVE>(a, tb, st); break;
        case EXTRA_TENSOR_PROJECT | EXTRA_VECTOR_EVOLVE: fz_n<R, N, OP_SCALAR, EXTRA_TENSOR_PROJECT | EXTRA_VECTOR_EVOLVE>(a, tb, st); break;
        case EXTRA_TENSOR_EVOLVE | EXTRA_VECTOR_EVOLVE: fz_n<R, N, OP_SCALAR, EXTRA_TENSOR_EVOLVE | EXTRA_VECTOR_EVOLVE>(a, tb, st); break;
        default: throw std::runtime_error("unsupported solver combination");
        }
    }
}

template <class R>
void fz_pass(int N, const FzParams &fp, typename CT<R>::C *data, int64_t stride, typename CT<R>::C *hij,
             typename CT<R>::C *hijp, typename CT<R>::C *bstate, const FftTables<R> &tb, cudaStream_t st)
{
    FzArgs<R> a;
    a.data = data; a.stride = stride;
    a.k2 = tb.k2; a.ks = tb.ks;
    a.p0 = fp.p0; a.p1 = fp.p1; a.p2 = fp.p2; a.p3 = fp.p3;
    a.extra = fp.extra;
    a.hij = hij; a.hijp = hijp; a.bstate = bstate;
    a.phi_hom = fp.phi_hom;
    a.bins = fp.bins;
    a.occ = fp.occ;
    a.err = fp.err;
    a.tab = fp.tab;
    a.ntab = fp.ntab;
    a.modes = fp.modes;
    GEV_SWITCH_N(N, (fz_dispatch<R, NN>(fp, a, tb, st)))
}

// prepareFTsource as standalone passes, in place (the reference's call shape,
// main.cu:725, :822): T00 form into the source field with per-block sums of
// the source (row blocks of N points, one partial per (y, z) row); Tij form
// on the six Sij planes
template <class R>
__global__ void k_prep_t00(FxArgs<R> a, int N, R *out, double *partial)
{
    __shared__ double red[256 / 32];
    const int y = blockIdx.x, z = blockIdx.y;
    double lsum = 0.0;
    for (int x = threadIdx.x; x < N; x += blockDim.x) {
        double src;
        const double r = prep_t00(a, N, x, y, z, src);
        lsum += src;
        out[sidx(N, x, y, z)] = (R)r;   // the same point was read above: in place is safe
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) s += red[w];
        partial[y + (int64_t)N * z] = s;
    }
}

template <class R>
__global__ void k_prep_tij(R *Sij, int64_t n3, const R *__restrict__ phi, R coeff, int N)
{
    const int y = blockIdx.x, z = blockIdx.y;
    for (int x = threadIdx.x; x < N; x += blockDim.x) {
        R o[6];
#pragma unroll
        for (int c = 0; c < 6; c++) o[c] = prep_tij(Sij + c * n3, phi, coeff, c, N, x, y, z);
#pragma unroll
        for (int c = 0; c < 6; c++) Sij[c * n3 + sidx(N, x, y, z)] = o[c];
    }
}

template <class R>
void prep_t00_pass(int N, R *source, const R *phi, const R *chi, double bg, double c, double c2, double c3, double *partial,
                   cudaStream_t st)
{
    FxArgs<R> a{};
    a.in = source; a.phi = phi; a.chi = chi;
    a.bg = bg; a.c = c; a.c2 = c2; a.c3 = c3;
    k_prep_t00<R><<<dim3(N, N), 256, 0, st>>>(a, N, source, partial);
}

template <class R>
void prep_tij_pass(int N, R *Sij, const R *phi, double coeff, cudaStream_t st)
{
    k_prep_tij<R><<<dim3(N, N), 128, 0, st>>>(Sij, (int64_t)N * N * N, phi, (R)coeff, N);
}

#define GEV_SOLVE_INST(R)                                                                                            \
    template void fx_forward<R>(int, int, const R *, int64_t, int, int, const R *, const R *, double, double, double, \
                                double, CT<R>::C *, int64_t, double *, const FftTables<R> &, cudaStream_t);          \
    template void fy_pass<R>(int, int, CT<R>::C *, int64_t, int, int *, const FftTables<R> &, cudaStream_t);                \
    template void fx_inverse<R>(int, const CT<R>::C *, int64_t, R *, int64_t, int, const FftTables<R> &,             \
                                cudaStream_t);                                                                       \
    template void fz_pass<R>(int, const FzParams &, CT<R>::C *, int64_t, CT<R>::C *, CT<R>::C *, CT<R>::C *,          \
                             const FftTables<R> &, cudaStream_t);                                                    \
    template void prep_t00_pass<R>(int, R *, const R *, const R *, double, double, double, double, double *,          \
                                   cudaStream_t);                                                                    \
    template void prep_tij_pass<R>(int, R *, const R *, double, cudaStream_t);

}  // namespace gev
