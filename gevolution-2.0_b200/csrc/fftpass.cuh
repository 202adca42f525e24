// fftpass.cuh -- pencil passes of the 3-D real-to-complex transforms with the
// reference's pointwise physics fused into their load and solve stages.
//
// Fourier layout: kx + PP*(ky + N*kz) for kx < P = N/2 + 1 (half spectrum
// along x); the row pitch PP = N/2 + 2 is even so that every row starts on a
// 16-byte boundary (tensor-memory-access copies need 16-byte-aligned strides).
//   fx_fwd : R2C along x for T rows (y0..y0+T-1, z); fused prepareFTsource
//   fy     : complex FFT along y for T kx-columns at one z (in place)
//   fz     : FFT along z, pointwise Fourier-space solver, inverse FFT along z,
//            for T kx-columns at one y and all components of the solve
//   fx_inv : C2R along x for T rows
#pragma once

#include "common.cuh"
#include "fft.cuh"
#include "tma.cuh"

namespace gev {

// occupancy the z pass and the six-component x pass are compiled for
#ifndef GEV_FZ_MINB
#define GEV_FZ_MINB 4   // resident CTAs of 256 threads per SM (FP32)
#endif
#ifndef GEV_FZ_MINB_D
#define GEV_FZ_MINB_D 3   // the same for FP64
#endif
#ifndef GEV_TIJ6_MINB
#define GEV_TIJ6_MINB 3
#endif
// resident CTAs per SM of the FP32 x passes (256 threads) and of the FP32 bulk-copy y pass (512 threads)
#ifndef GEV_FX_MINB
#define GEV_FX_MINB 4
#endif
#ifndef GEV_FXI_MINB
#define GEV_FXI_MINB 4
#endif
#ifndef GEV_FY_MINB
#define GEV_FY_MINB 2
#endif

// ---------------------------------------------------------------------------
// fused source preparation (PHINONLINEAR): T00 in FP64, Tij in the field precision
// ---------------------------------------------------------------------------
// FX_COPY, FX_PREP_T00, FX_PREP_TIJ: common.cuh

template <class R> struct FxArgs {
    const R *in;          // field (component plane) to transform
    const R *phi;
    const R *chi;
    double bg, c, c2, c3; // prepareFTsource_T00 params (bgmodel, coeff, coeff2, coeff3) / Tij coeff in c
    int comp0;            // first Tij component of the batch (gridDim.z = number of components)
    typename CT<R>::C *out;
    double *partial;      // per-block partial sums of the source (FX_PREP_T00)
};

template <class R>
__device__ __forceinline__ double ld(const R *f, int N, int x, int y, int z)
{
    return (double)f[sidx(N, wrapi(x, N), wrapi(y, N), wrapi(z, N))];
}

template <class R>
__device__ __forceinline__ R ldr(const R *f, int N, int x, int y, int z)
{
    return __ldg(f + sidx(N, wrapi(x, N), wrapi(y, N), wrapi(z, N)));
}

// Strided fill of TOT elements (element idx = threadIdx.x + k*NT): each thread
// issues B loads before the matching B stores, so B global loads per thread are
// in flight instead of one (the passes are bound by load latency otherwise).
template <int TOT, int NT, int B, class V, class LOAD, class STORE>
__device__ __forceinline__ void staged_fill(LOAD &&load, STORE &&store)
{
    constexpr int PER = (TOT + NT - 1) / NT;
#pragma unroll
    for (int k0 = 0; k0 < PER; k0 += B) {
        V v[B];
#pragma unroll
        for (int k = 0; k < B; k++) {
            const int idx = threadIdx.x + (k0 + k) * NT;
            if (k0 + k < PER && (PER * NT == TOT || idx < TOT)) v[k] = load(idx);
        }
#pragma unroll
        for (int k = 0; k < B; k++) {
            const int idx = threadIdx.x + (k0 + k) * NT;
            if (k0 + k < PER && (PER * NT == TOT || idx < TOT)) store(idx, v[k]);
        }
    }
}

// prepareFTsource_T00: gevolution.hpp:160-171
template <class R>
__device__ __forceinline__ double prep_t00(const FxArgs<R> &a, int N, int x, int y, int z, double &src)
{
    int64_t i = sidx(N, x, y, z);
    double s = (double)a.in[i];
    double ph = (double)a.phi[i];
    src = s;
    double r = a.c2 * (s - a.bg);
    r *= 1.0 - 2.0 * ph * (1.0 - ph);
    double g;
    g = ld(a.phi, N, x - 1, y, z) - ld(a.phi, N, x + 1, y, z); r += 0.125 * g * g;
    g = ld(a.phi, N, x, y - 1, z) - ld(a.phi, N, x, y + 1, z); r += 0.125 * g * g;
    g = ld(a.phi, N, x, y, z - 1) - ld(a.phi, N, x, y, z + 1); r += 0.125 * g * g;
    r += (a.c3 * (1.0 - 3.0 * ph) - a.c) * ph - a.c3 * (double)a.chi[i];
    return r;
}

// prepareFTsource_Tij for one symmetric component c (00,01,02,11,12,22),
// gevolution.hpp:64-107, in the field precision R.  Diagonal:
// (phi(x+e_i) - phi(x-e_i))^2 / 2 + coeff T_ii.  Off-diagonal, the reference's
//   pi pj - p0 pij + (p0^2 - pi^2 - pj^2 + pij^2) / 2
// is evaluated in the algebraically identical form 2uv + w (u + v + w/2), with
// u = pi - p0, v = pj - p0, w = pij - pi - pj + p0: the squares of the
// potential cancel exactly in that form, so it keeps full relative accuracy in
// FP32 where the reference's form loses (phi / grad phi)^2 to cancellation.
template <class R>
__device__ __forceinline__ R prep_tij(const R *T, const R *phi, R coeff, int c, int N, int x, int y, int z)
{
    const int64_t i = sidx(N, x, y, z);
    const R t = __ldg(T + i);
    const int ai = (c == 0 || c == 1 || c == 2) ? 0 : (c == 5 ? 2 : 1);
    const int aj = (c == 0) ? 0 : (c == 1 ? 1 : ((c == 2 || c == 4 || c == 5) ? 2 : 1));
    const int ei[3] = {ai == 0, ai == 1, ai == 2}, ej[3] = {aj == 0, aj == 1, aj == 2};
    if (ai == aj) {
        const R g = ldr(phi, N, x + ei[0], y + ei[1], z + ei[2]) - ldr(phi, N, x - ei[0], y - ei[1], z - ei[2]);
        return (R)0.5 * g * g + coeff * t;
    }
    const R p0 = __ldg(phi + i);
    const R pi_ = ldr(phi, N, x + ei[0], y + ei[1], z + ei[2]);
    const R pj = ldr(phi, N, x + ej[0], y + ej[1], z + ej[2]);
    const R pij = ldr(phi, N, x + ei[0] + ej[0], y + ei[1] + ej[1], z + ei[2] + ej[2]);
    const R u = pi_ - p0, v = pj - p0, w = (pij - pi_) - (pj - p0);
    return (R)2 * u * v + w * (u + v + (R)0.5 * w) + coeff * t;
}

// T0i component c completed from its potential-free sum S_c at vertex x:
// T0i_c(x) = (1 + phi(x) + phi(x + e_c)) S_c(x) -- the per-vertex factor of
// particle_T0i_project (gevolution.hpp:2031-2201), which does not depend on
// the particle, applied once per vertex with the current phi
template <class R>
__device__ __forceinline__ R prep_t0i(const R *S, const R *phi, int c, int N, int x, int y, int z)
{
    const int64_t i = sidx(N, x, y, z);
    const R f = (R)1 + __ldg(phi + i) + ldr(phi, N, x + (c == 0), y + (c == 1), z + (c == 2));
    return f * __ldg(S + i);
}

// ---------------------------------------------------------------------------
// x pass, forward: real rows -> half spectrum.  grid (N/T, N, ncomp)
// ---------------------------------------------------------------------------
template <class R, int N, int T, int NT, int MODE>
__global__ void __launch_bounds__(NT, sizeof(R) == 4 ? GEV_FX_MINB : 1) k_fx_fwd(FxArgs<R> a, int64_t in_stride, int64_t out_stride,
                                               const typename CT<R>::C *__restrict__ tw_half,
                                               const typename CT<R>::C *__restrict__ tw_full)
{
    using C = typename CT<R>::C;
    constexpr int M = N / 2, P = N / 2 + 1, PP = N / 2 + 2, LD = T + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *buf = reinterpret_cast<C *>(smem_raw);
    __shared__ double red[NT / 32];

    const int y0 = blockIdx.x * T, z = blockIdx.y, comp = blockIdx.z;
    const R *in = a.in + (int64_t)comp * in_stride;
    C *out = a.out + (int64_t)comp * out_stride;
    double lsum = 0.0;

    staged_fill<M * T, NT, (MODE == FX_COPY ? 8 : 4), C>(
        [&](int idx) {
            const int n = idx % M, t = idx / M, y = y0 + t;
            R v0, v1;
            if constexpr (MODE == FX_COPY) {
                const R *row = in + sidx(N, 0, y, z);
                v0 = __ldg(row + 2 * n);
                v1 = __ldg(row + 2 * n + 1);
            } else if constexpr (MODE == FX_PREP_T00) {
                double s0, s1;
                v0 = (R)prep_t00(a, N, 2 * n, y, z, s0);
                v1 = (R)prep_t00(a, N, 2 * n + 1, y, z, s1);
                lsum += s0 + s1;
            } else if constexpr (MODE == FX_PREP_T0I) {
                v0 = prep_t0i(in, a.phi, a.comp0 + comp, N, 2 * n, y, z);
                v1 = prep_t0i(in, a.phi, a.comp0 + comp, N, 2 * n + 1, y, z);
            } else {
                v0 = prep_tij(in, a.phi, (R)a.c, a.comp0 + comp, N, 2 * n, y, z);
                v1 = prep_tij(in, a.phi, (R)a.c, a.comp0 + comp, N, 2 * n + 1, y, z);
            }
            return mk(v0, v1);
        },
        [&](int idx, C v) { buf[(idx % M) * LD + idx / M] = v; });
    __syncthreads();
    fft_lines<M, -1, T, NT>(buf, LD, tw_half);

    for (int idx = threadIdx.x; idx < P * T; idx += NT) {
        int k = idx % P, t = idx / P, y = y0 + t;
        C zk = buf[(k == M ? 0 : k) * LD + t];
        C zm = buf[(k == 0 ? 0 : M - k) * LD + t];
        zm.y = -zm.y;                                  // conj(Z[M-k])
        C ze = cscale(cadd(zk, zm), R(0.5));
        C d = csub(zk, zm);
        C zo = mk(R(0.5) * d.y, R(-0.5) * d.x);        // (zk - conj(zm)) / (2i)
        C w = __ldg(tw_full + k);
        out[k + (int64_t)PP * (y + (int64_t)N * z)] = cadd(ze, cmul(w, zo));
    }

    if constexpr (MODE == FX_PREP_T00) {
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < NT / 32; w++) s += red[w];
            a.partial[blockIdx.x + gridDim.x * blockIdx.y] = s;
        }
    }
}

// prepareFTsource_Tij for all six components at one point from the ten
// potential values they share (p0 = phi(x), pxp = phi(x + e_x), ..., pxy =
// phi(x + e_x + e_y)); the arithmetic of each component is that of prep_tij
// (same expressions, same order), so the results are identical.
template <class R>
__device__ __forceinline__ void tij6_point(R p0, R pxp, R pxm, R pyp, R pym, R pzp, R pzm, R pxy, R pxz, R pyz,
                                           const R t[6], R coeff, R o[6])
{
    R g;
    g = pxp - pxm; o[0] = (R)0.5 * g * g + coeff * t[0];
    g = pyp - pym; o[3] = (R)0.5 * g * g + coeff * t[3];
    g = pzp - pzm; o[5] = (R)0.5 * g * g + coeff * t[5];
    R u, v, w;
    u = pxp - p0; v = pyp - p0; w = (pxy - pxp) - (pyp - p0);
    o[1] = (R)2 * u * v + w * (u + v + (R)0.5 * w) + coeff * t[1];
    u = pxp - p0; v = pzp - p0; w = (pxz - pxp) - (pzp - p0);
    o[2] = (R)2 * u * v + w * (u + v + (R)0.5 * w) + coeff * t[2];
    u = pyp - p0; v = pzp - p0; w = (pyz - pyp) - (pzp - p0);
    o[4] = (R)2 * u * v + w * (u + v + (R)0.5 * w) + coeff * t[4];
}

// two adjacent values (x even: 8- or 16-byte aligned) in one load
template <class R> __device__ __forceinline__ typename CT<R>::C ld_pair(const R *p)
{
    return __ldg(reinterpret_cast<const typename CT<R>::C *>(p));
}

// x pass, forward, for the six Tij components at once: each potential value
// is loaded once for all six sources.  grid (N/T, N)
template <class R, int N, int T, int NT>
__global__ void __launch_bounds__(NT, GEV_TIJ6_MINB) k_fx_fwd_tij6(const R *__restrict__ Tij, int64_t n3, const R *__restrict__ phi,
                                                    double coeff, typename CT<R>::C *out, int64_t out_stride,
                                                    const typename CT<R>::C *__restrict__ tw_half,
                                                    const typename CT<R>::C *__restrict__ tw_full)
{
    using C = typename CT<R>::C;
    // the six components' rows side by side: 6T lines of one batched transform,
    // element n of line c*T + t at buf[n*LD + c*T + t]
    constexpr int M = N / 2, P = N / 2 + 1, PP = N / 2 + 2, T6 = 6 * T, LD = T6 + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *buf = reinterpret_cast<C *>(smem_raw);
    const int y0 = blockIdx.x * T, z = blockIdx.y;
    const R rc = (R)coeff;
    struct Six { C v[6]; };
    staged_fill<M * T, NT, 2, Six>(
        [&](int idx) {
            // the points x0 = 2n and x0 + 1 of row (y, z): the potential rows
            // they touch are read as aligned pairs plus the four values beyond
            const int n = idx % M, t = idx / M, y = y0 + t;
            const int x0 = 2 * n, xm = x0 == 0 ? N - 1 : x0 - 1, x2 = x0 + 2 == N ? 0 : x0 + 2;
            const int ym = y == 0 ? N - 1 : y - 1, yp = y == N - 1 ? 0 : y + 1;
            const int zm = z == 0 ? N - 1 : z - 1, zp = z == N - 1 ? 0 : z + 1;
            const R *r00 = phi + sidx(N, 0, y, z), *rm0 = phi + sidx(N, 0, ym, z), *rp0 = phi + sidx(N, 0, yp, z);
            const R *r0p = phi + sidx(N, 0, y, zp), *r0m = phi + sidx(N, 0, y, zm), *rpp = phi + sidx(N, 0, yp, zp);
            const C c00 = ld_pair(r00 + x0), cm0 = ld_pair(rm0 + x0), cp0 = ld_pair(rp0 + x0);
            const C c0p = ld_pair(r0p + x0), c0m = ld_pair(r0m + x0), cpp = ld_pair(rpp + x0);
            const R f00m = __ldg(r00 + xm), f002 = __ldg(r00 + x2), fp02 = __ldg(rp0 + x2), f0p2 = __ldg(r0p + x2);
            const int64_t i0 = sidx(N, x0, y, z);
            R t0[6], t1[6];
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const C tv = ld_pair(Tij + c * n3 + i0);
                t0[c] = tv.x;
                t1[c] = tv.y;
            }
            R a0[6], a1[6];
            tij6_point(c00.x, c00.y, f00m, cp0.x, cm0.x, c0p.x, c0m.x, cp0.y, c0p.y, cpp.x, t0, rc, a0);
            tij6_point(c00.y, f002, c00.x, cp0.y, cm0.y, c0p.y, c0m.y, fp02, f0p2, cpp.y, t1, rc, a1);
            Six s;
#pragma unroll
            for (int c = 0; c < 6; c++) s.v[c] = mk(a0[c], a1[c]);
            return s;
        },
        [&](int idx, Six s) {
            const int o = (idx % M) * LD + idx / M;
#pragma unroll
            for (int c = 0; c < 6; c++) buf[o + c * T] = s.v[c];
        });
    __syncthreads();
    fft_lines<M, -1, T6, NT>(buf, LD, tw_half);
    for (int idx = threadIdx.x; idx < 6 * P * T; idx += NT) {
        const int k = idx % P, r = idx / P, t = r % T, c = r / T, y = y0 + t;
        const C *b = buf + c * T;
        C zk = b[(k == M ? 0 : k) * LD + t];
        C zm = b[(k == 0 ? 0 : M - k) * LD + t];
        zm.y = -zm.y;
        C ze = cscale(cadd(zk, zm), R(0.5));
        C d = csub(zk, zm);
        C zo = mk(R(0.5) * d.y, R(-0.5) * d.x);
        C w = __ldg(tw_full + k);
        out[c * out_stride + k + (int64_t)PP * (y + (int64_t)N * z)] = cadd(ze, cmul(w, zo));
    }
}

// ---------------------------------------------------------------------------
// y pass (in place), complex.  grid (ceil(P/T), N, ncomp)
// ---------------------------------------------------------------------------
template <class R, int N, int T, int NT, int S>
__global__ void __launch_bounds__(NT, 1024 / NT) k_fy(typename CT<R>::C *data, int64_t stride,
                                           const typename CT<R>::C *__restrict__ tw)
{
    using C = typename CT<R>::C;
    constexpr int P = N / 2 + 1, PP = N / 2 + 2, LD = T + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *buf = reinterpret_cast<C *>(smem_raw);
    const int kx0 = blockIdx.x * T, z = blockIdx.y;
    C *d = data + (int64_t)blockIdx.z * stride;
    staged_fill<N * T, NT, 8, C>(
        [&](int idx) {
            const int t = idx % T, n = idx / T, kx = kx0 + t;
            return (kx < P) ? d[kx + (int64_t)PP * (n + (int64_t)N * z)] : mk(R(0), R(0));
        },
        [&](int idx, C v) { buf[(idx / T) * LD + idx % T] = v; });
    __syncthreads();
    fft_lines<N, S, T, NT>(buf, LD, tw);
    for (int idx = threadIdx.x; idx < N * T; idx += NT) {
        int t = idx % T, n = idx / T, kx = kx0 + t;
        if (kx < P) d[kx + (int64_t)PP * (n + (int64_t)N * z)] = buf[n * LD + t];
    }
}

// ---------------------------------------------------------------------------
// x pass, inverse: half spectrum -> real rows (imaginary parts of the kx = 0
// and kx = N/2 entries do not contribute).  grid (N/T, N, ncomp)
// ---------------------------------------------------------------------------
template <class R, int N, int T, int NT>
__global__ void __launch_bounds__(NT, sizeof(R) == 4 ? GEV_FXI_MINB : 1) k_fx_inv(const typename CT<R>::C *in, int64_t in_stride, R *out,
                                               int64_t out_stride,
                                               const typename CT<R>::C *__restrict__ tw_half,
                                               const typename CT<R>::C *__restrict__ tw_full)
{
    using C = typename CT<R>::C;
    constexpr int M = N / 2, PP = N / 2 + 2, LD = T + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *buf = reinterpret_cast<C *>(smem_raw);
    const int y0 = blockIdx.x * T, z = blockIdx.y;
    const C *src = in + (int64_t)blockIdx.z * in_stride;
    R *dst = out + (int64_t)blockIdx.z * out_stride;
    staged_fill<M * T, NT, 4, C>(
        [&](int idx) {
            const int k = idx % M, t = idx / M, y = y0 + t;
            const C *row = src + (int64_t)PP * (y + (int64_t)N * z);
            C A = __ldg(row + k), B = __ldg(row + M - k);
            if (k == 0) { A.y = R(0); B.y = R(0); }
            B.y = -B.y;
            C w = __ldg(tw_full + k);
            w.y = -w.y;                                // exp(+2 pi i k / N)
            C dd = cmul(csub(A, B), w);
            C s = cadd(A, B);
            return mk(s.x - dd.y, s.y + dd.x);         // (A+B) + i (A-B) w
        },
        [&](int idx, C v) { buf[(idx % M) * LD + idx / M] = v; });
    __syncthreads();
    fft_lines<M, 1, T, NT>(buf, LD, tw_half);
    for (int idx = threadIdx.x; idx < M * T; idx += NT) {
        int n = idx % M, t = idx / M, y = y0 + t;
        C v = buf[n * LD + t];
        R *row = dst + sidx(N, 0, y, z);
        row[2 * n] = v.x;
        row[2 * n + 1] = v.y;
    }
}

// ---------------------------------------------------------------------------
// z pass with the Fourier-space solvers (gevolution.hpp:251-852).  All solver
// arithmetic is FP64; k tables hold gridk2[i] = (2N sin(pi i/N))^2 and
// kshift[i] = 2N sin(pi i/N) exp(-i pi i/N) (gevolution.hpp:269-275).
// ---------------------------------------------------------------------------
// OP_POISSON, OP_SCALAR, OP_VECTOR, OP_BIN and the EXTRA_* flags: common.cuh
// optional extras of OP_SCALAR

template <class R> struct FzArgs {
    typename CT<R>::C *data;   // component planes (stride nk)
    int64_t stride;
    const double *k2;          // gridk2[N]
    const double2 *ks;         // kshift[N]
    double p0, p1, p2, p3;     // op parameters
    int extra;
    typename CT<R>::C *hij;    // tensor state (6 planes) / B state (3 planes)
    typename CT<R>::C *hijp;
    typename CT<R>::C *bstate;
    double *phi_hom;           // k = 0 mode after the Poisson solve
    double *bins;              // OP_BIN: 4*numbins accumulators (k, k^2, P, P^2)
    unsigned long long *occ;   // OP_BIN: mode counts
    int *err;                  // device error word (may be null)
    const double *tab;         // OP_ZELD: ln k [h/Mpc] (ntab values) then ln P(k) (ntab values)
    int ntab;
    const double2 *modes;      // OP_ICS: [kz][ky][kx] numerators of the displacement potential
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zsc(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 zcj(double2 a) { return make_double2(a.x, -a.y); }
template <class C> __device__ __forceinline__ double2 z2d(C a) { return make_double2((double)a.x, (double)a.y); }

// transverse-traceless numerators of projectFTtensor (gevolution.hpp:744-769)
__device__ __forceinline__ void tt_num(const double *g, const double2 *k, double k2, const double2 *S, double2 *o)
{
    double2 Sxx = S[0], Sxy = S[1], Sxz = S[2], Syy = S[3], Syz = S[4], Szz = S[5];
    o[0] = zadd(zadd(zsc(zadd(zsc(Sxx, g[0] - k2), zsc(zmul(k[0], zadd(zmul(k[1], Sxy), zmul(k[2], Sxz))), 2.0)), g[0] - k2),
                     zsc(Syy, (g[0] + k2) * (g[1] + k2) - 2.0 * k2 * k2)),
                zadd(zsc(Szz, (g[0] + k2) * (g[2] + k2) - 2.0 * k2 * k2), zsc(zmul(zmul(k[1], k[2]), Syz), 2.0 * (g[0] + k2))));
    o[1] = zadd(zadd(zsc(Sxy, 2.0 * (g[0] - k2) * (g[1] - k2)), zsc(zmul(zmul(zcj(k[0]), zcj(k[1])), Szz), g[2] + k2)),
                zadd(zsc(zmul(zcj(k[1]), zadd(zmul(zcj(k[0]), Sxx), zsc(zmul(k[2], Sxz), 2.0))), g[0] - k2),
                     zsc(zmul(zcj(k[0]), zadd(zmul(zcj(k[1]), Syy), zsc(zmul(k[2], Syz), 2.0))), g[1] - k2)));
    o[2] = zadd(zadd(zsc(Sxz, 2.0 * (g[0] - k2) * (g[2] - k2)), zsc(zmul(zmul(zcj(k[0]), zcj(k[2])), Syy), g[1] + k2)),
                zadd(zsc(zmul(zcj(k[2]), zadd(zmul(zcj(k[0]), Sxx), zsc(zmul(k[1], Sxy), 2.0))), g[0] - k2),
                     zsc(zmul(zcj(k[0]), zadd(zmul(zcj(k[2]), Szz), zsc(zmul(k[1], Syz), 2.0))), g[2] - k2)));
    o[3] = zadd(zadd(zsc(zadd(zsc(Syy, g[1] - k2), zsc(zmul(k[1], zadd(zmul(k[0], Sxy), zmul(k[2], Syz))), 2.0)), g[1] - k2),
                     zsc(Sxx, (g[1] + k2) * (g[0] + k2) - 2.0 * k2 * k2)),
                zadd(zsc(Szz, (g[1] + k2) * (g[2] + k2) - 2.0 * k2 * k2), zsc(zmul(zmul(k[0], k[2]), Sxz), 2.0 * (g[1] + k2))));
    o[4] = zadd(zadd(zsc(Syz, 2.0 * (g[1] - k2) * (g[2] - k2)), zsc(zmul(zmul(zcj(k[1]), zcj(k[2])), Sxx), g[0] + k2)),
                zadd(zsc(zmul(zcj(k[2]), zadd(zmul(zcj(k[1]), Syy), zsc(zmul(k[0], Sxy), 2.0))), g[1] - k2),
                     zsc(zmul(zcj(k[1]), zadd(zmul(zcj(k[2]), Szz), zsc(zmul(k[0], Sxz), 2.0))), g[2] - k2)));
    o[5] = zadd(zadd(zsc(zadd(zsc(Szz, g[2] - k2), zsc(zmul(k[2], zadd(zmul(k[0], Sxz), zmul(k[1], Syz))), 2.0)), g[2] - k2),
                     zsc(Sxx, (g[2] + k2) * (g[0] + k2) - 2.0 * k2 * k2)),
                zadd(zsc(Syy, (g[2] + k2) * (g[1] + k2) - 2.0 * k2 * k2), zsc(zmul(zmul(k[0], k[1]), Sxy), 2.0 * (g[2] + k2))));
}

template <int OP, int EXTRA> struct OpShape {
    static constexpr int CIN = (OP == OP_POISSON || OP == OP_BIN || OP == OP_ZELD || OP == OP_ICS) ? 1 : (OP == OP_SCALAR ? 6 : 3);
    static constexpr int COUT = (OP == OP_BIN) ? 0 : ((OP == OP_POISSON || OP == OP_ICS) ? 1 : (OP == OP_SCALAR ? ((EXTRA & EXTRA_VECTOR_EVOLVE) ? 4 : 1) : 3));
    static constexpr int CMAX = CIN > COUT ? CIN : COUT;   // columns the pass holds at once
    // projectFTscalar alone needs only three kz-independent combinations of the
    // six S_ij (see k_fz), so the z pass transforms three columns instead of six
    static constexpr bool CONTRACT = (OP == OP_SCALAR && EXTRA == 0);
    static constexpr int CBUF = CONTRACT ? 3 : CMAX;
    static constexpr int CTMA = CONTRACT ? 4 : CMAX;   // buffers of the bulk-copy z pass (k_fz_tma)
};

// Element-wise solver for one (kx, ky, kz): reads CIN values from v, writes
// COUT values back into v[0..COUT-1].
template <class R, int OP, int EXTRA>
__device__ __forceinline__ void fz_apply(const FzArgs<R> &a, int N, int kx, int ky, int kz, int64_t kidx, double2 *v)
{
    using C = typename CT<R>::C;
    const double g[3] = {__ldg(a.k2 + kx), __ldg(a.k2 + ky), __ldg(a.k2 + kz)};
    const double2 k[3] = {__ldg(a.ks + kx), __ldg(a.ks + ky), __ldg(a.ks + kz)};
    const double k2 = g[0] + g[1] + g[2];
    if constexpr (OP == OP_BIN) {
        // extractCrossSpectrum binning, KTYPE_LINEAR with CIC deconvolution
        // (tools.hpp:105-215); p0 = numbins, p1 = kmax
        if (kx == 0 && ky == 0 && kz == 0) return;
        const int weight = (kx == 0 || (kx == N / 2 && (N % 2) == 0)) ? 1 : 2;
        // k^2 and the bin index with separately rounded operations (no fused
        // multiply-add), as the reference evaluates them on the host: modes on a
        // bin edge (|n|^2 = 3 m^2 for the default kmax) land in the same bin
        auto lin = [&](int i) {
            const double t = __dmul_rn(2.0 * 3.14159265358979323846, (double)(i <= N / 2 ? i : N - i));
            return __dmul_rn(t, t);
        };
        auto snc = [&](int i) {
            int j = i <= N / 2 ? i : N - i;
            if (j == 0) return 1.0;
            return sin(3.14159265358979323846 * (double)(float)j / (double)(float)N) * (double)(float)N / (3.14159265358979323846 * (double)(float)j);
        };
        double kk2 = __dadd_rn(__dadd_rn(lin(kx), lin(ky)), lin(kz));
        double s = snc(kx) * snc(ky) * snc(kz);
        s *= s;
        double pw = v[0].x * v[0].x + v[0].y * v[0].y;
        double sk = sqrt(kk2);
        int nb = (int)a.p0;
        int bin = (int)floor(__ddiv_rn(__dmul_rn((double)nb, sk), a.p1));
        if (bin < nb) {
            atomicAdd(a.bins + bin, weight * sk);
            atomicAdd(a.bins + nb + bin, weight * kk2);
            atomicAdd(a.bins + 2 * nb + bin, weight * pw * kk2 * sk / s);
            atomicAdd(a.bins + 3 * nb + bin, weight * pw * pw * kk2 * kk2 * kk2 / s / s);
            atomicAdd(a.occ + bin, (unsigned long long)weight);
        }
    } else if constexpr (OP == OP_ZELD) {
        // Zel'dovich displacement of a white-noise spectrum (the generator's
        // counterpart of generateDisplacementField, ic_basic.hpp:1165-1610):
        // psi_c = i 2 pi n_c / |2 pi n|^2 * sqrt(P(k) N^3 / L^3) * w / N^3 in box
        // units, n the signed integer wavevector (numpy fftfreq convention),
        // k = 2 pi |n| / L.  p0 = L [Mpc/h], p1 != 0 cuts |n| > N/2 (k-sphere).
        const int n0 = kx, n1 = (ky < N / 2) ? ky : ky - N, n2 = (kz < N / 2) ? kz : kz - N;
        const double kk = (double)n0 * n0 + (double)n1 * n1 + (double)n2 * n2;
        const double2 w = v[0];
        v[0] = v[1] = v[2] = make_double2(0.0, 0.0);
        if (kk == 0.0 || (a.p1 != 0.0 && 4.0 * kk > (double)N * N)) return;
        const double lk = log(2.0 * 3.14159265358979323846 * sqrt(kk) / a.p0);
        int lo = 0, hi = a.ntab - 1;
        double lp;
        if (lk <= a.tab[0]) lp = a.tab[a.ntab];
        else if (lk >= a.tab[hi]) lp = a.tab[a.ntab + hi];
        else {
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (a.tab[mid] <= lk) lo = mid; else hi = mid;
            }
            const double t = (lk - a.tab[lo]) / (a.tab[hi] - a.tab[lo]);
            lp = a.tab[a.ntab + lo] + t * (a.tab[a.ntab + hi] - a.tab[a.ntab + lo]);
        }
        const double n3 = (double)N * N * N;
        const double amp = sqrt(exp(lp) * n3 / (a.p0 * a.p0 * a.p0)) / n3 / (2.0 * 3.14159265358979323846 * kk);
        const double nc[3] = {(double)n0, (double)n1, (double)n2};
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = make_double2(-nc[c] * amp * w.y, nc[c] * amp * w.x);   // i nc amp w
    } else if constexpr (OP == OP_ICS) {
        // generateDisplacementField's last factor (ic_basic.hpp:1270-1281):
        // potFT(k) = numerator(k) / potFT(k), the field holding the Fourier
        // transform of the CIC kernel; modes the generator sets to zero stay
        // zero (their numerator is exactly zero).  Complex division as
        // (n ker*) / |ker|^2.
        const double2 num = __ldg(a.modes + (int64_t)kx + (int64_t)(N / 2 + 1) * ((int64_t)ky + (int64_t)N * kz));
        if (num.x == 0.0 && num.y == 0.0) {
            v[0] = make_double2(0.0, 0.0);
        } else {
            const double2 ker = v[0];
            const double den = ker.x * ker.x + ker.y * ker.y;
            v[0] = make_double2((num.x * ker.x + num.y * ker.y) / den, (num.y * ker.x - num.x * ker.y) / den);
        }
    } else if constexpr (OP == OP_POISSON) {
        // solveModifiedPoissonFT: gevolution.hpp:806-852; p0 = coeff / (-N^3), p1 = modif;
        // p2 != 0 removes the k = 0 mode first (ic_basic.hpp:2419-2421)
        double den = k2 + a.p1;
        v[0] = (den != 0.0) ? zsc(v[0], a.p0 / den) : make_double2(0.0, 0.0);
        if (kx == 0 && ky == 0 && kz == 0) {
            if (a.p1 == 0.0 || a.p2 != 0.0) v[0] = make_double2(0.0, 0.0);
            if (a.phi_hom) *a.phi_hom = v[0].x;
        }
    } else if constexpr (OP == OP_VECTOR) {
        // projectFTvector: gevolution.hpp:449-515; p0 = coeff, p1 = modif
        if (k2 > 0.0) {
            double2 tmp = zsc(zadd(zadd(zmul(k[0], v[0]), zmul(k[1], v[1])), zmul(k[2], v[2])), 1.0 / k2);
            double f = 4.0 * a.p0 / (k2 + a.p1);
            for (int c = 0; c < 3; c++) v[c] = zsc(zsub(v[c], zmul(zcj(k[c]), tmp)), f);
        } else {
            v[0] = v[1] = v[2] = make_double2(0.0, 0.0);
        }
    } else {
        // projectFTscalar: gevolution.hpp:251-340 (add = 0)
        double2 S[6] = {v[0], v[1], v[2], v[3], v[4], v[5]};
        double2 chi = make_double2(0.0, 0.0);
        if (k2 > 0.0) {
            chi = zadd(zadd(zsc(S[0], g[1] + g[2] - 2.0 * g[0]), zsc(S[3], g[0] + g[2] - 2.0 * g[1])), zsc(S[5], g[0] + g[1] - 2.0 * g[2]));
            chi = zsub(chi, zsc(zmul(zmul(k[0], k[1]), S[1]), 6.0));
            chi = zsub(chi, zsc(zmul(zmul(k[0], k[2]), S[2]), 6.0));
            chi = zsub(chi, zsc(zmul(zmul(k[1], k[2]), S[4]), 6.0));
            chi = zsc(chi, 1.0 / (2.0 * k2 * k2 * N));
        }
        if constexpr ((EXTRA & EXTRA_TENSOR_PROJECT) != 0) {
            // projectFTtensor: gevolution.hpp:693-787
            double2 o[6];
            if (k2 > 0.0) {
                tt_num(g, k, k2, S, o);
                double k6 = k2 * k2 * k2 * N;
                for (int c = 0; c < 6; c++) a.hij[c * a.stride + kidx] = mk(R(o[c].x / k6), R(o[c].y / k6));
            } else {
                for (int c = 0; c < 6; c++) a.hij[c * a.stride + kidx] = mk(R(0), R(0));
            }
        }
        if constexpr ((EXTRA & EXTRA_TENSOR_EVOLVE) != 0) {
            // evolveFTtensor: gevolution.hpp:537-674; p0 = hubble, p1 = dtau, p2 = dtau_old
            const double dm = 0.5 * (a.p2 + a.p1), opd = 1.0 + a.p0 * dm, omd = 1.0 - a.p0 * dm;
            const double k4 = k2 * k2 * N;
            double2 h[6], hp[6], o[6];
            for (int c = 0; c < 6; c++) { h[c] = z2d(a.hij[c * a.stride + kidx]); hp[c] = z2d(a.hijp[c * a.stride + kidx]); }
            if (k2 * dm * dm < 1.0) {
                for (int c = 0; c < 6; c++) h[c] = zadd(h[c], zsc(hp[c], a.p2));
                if (k2 > 0.0) {
                    tt_num(g, k, k2, S, o);
                    for (int c = 0; c < 6; c++) hp[c] = zsc(zadd(zsc(hp[c], omd), zsc(zsub(zsc(o[c], 1.0 / k4), zsc(h[c], k2)), dm)), 1.0 / opd);
                } else {
                    double2 tr = zadd(zadd(S[0], S[3]), S[5]);
                    double2 Sm[6] = {zsub(S[0], zsc(tr, 1.0 / 3.0)), S[1], S[2], zsub(S[3], zsc(tr, 1.0 / 3.0)), S[4], zsub(S[5], zsc(tr, 1.0 / 3.0))};
                    for (int c = 0; c < 6; c++) hp[c] = zsc(zadd(zsc(hp[c], omd), zsc(Sm[c], 2.0 * dm / N)), 1.0 / opd);
                }
            } else {
                tt_num(g, k, k2, S, o);
                for (int c = 0; c < 6; c++) {
                    hp[c] = make_double2(0.0, 0.0);
                    h[c] = zsc(zadd(zsc(o[c], a.p2 / k4), zsc(h[c], 2.0 * a.p0)), 1.0 / (k2 * a.p2 + 2.0 * a.p0));
                }
            }
            for (int c = 0; c < 6; c++) {
                a.hij[c * a.stride + kidx] = mk(R(h[c].x), R(h[c].y));
                a.hijp[c * a.stride + kidx] = mk(R(hp[c].x), R(hp[c].y));
            }
        }
        if constexpr ((EXTRA & EXTRA_VECTOR_EVOLVE) != 0) {
            // evolveFTvector: gevolution.hpp:359-429; p3 = a^2 dtau
            double2 B[3];
            for (int c = 0; c < 3; c++) B[c] = z2d(a.bstate[c * a.stride + kidx]);
            double k4 = k2 * k2;
            if (k4 > 0.0) {
                double2 fac = make_double2(0.0, -2.0 * a.p3 / k4);
                B[0] = zadd(B[0], zmul(fac, zadd(zmul(zcj(k[0]), zsub(zsub(zsub(zsc(S[0], g[1] + g[2]), zsc(S[3], g[1])), zsc(S[5], g[2])), zsc(zmul(zmul(k[1], k[2]), S[4]), 2.0))),
                                                 zsc(zadd(zmul(k[1], S[1]), zmul(k[2], S[2])), g[1] + g[2] - g[0]))));
                B[1] = zadd(B[1], zmul(fac, zadd(zmul(zcj(k[1]), zsub(zsub(zsub(zsc(S[3], g[0] + g[2]), zsc(S[0], g[0])), zsc(S[5], g[2])), zsc(zmul(zmul(k[0], k[2]), S[2]), 2.0))),
                                                 zsc(zadd(zmul(k[0], S[1]), zmul(k[2], S[4])), g[0] + g[2] - g[1]))));
                B[2] = zadd(B[2], zmul(fac, zadd(zmul(zcj(k[2]), zsub(zsub(zsub(zsc(S[5], g[0] + g[1]), zsc(S[0], g[0])), zsc(S[3], g[1])), zsc(zmul(zmul(k[0], k[1]), S[1]), 2.0))),
                                                 zsc(zadd(zmul(k[0], S[2]), zmul(k[1], S[4])), g[0] + g[1] - g[2]))));
            } else {
                B[0] = B[1] = B[2] = make_double2(0.0, 0.0);
            }
            for (int c = 0; c < 3; c++) {
                a.bstate[c * a.stride + kidx] = mk(R(B[c].x), R(B[c].y));
                v[1 + c] = B[c];
            }
        }
        v[0] = chi;
    }
}

// grid (ceil(P/T), N); T kx-columns at one ky, all CIN components of the solve.
//
// projectFTscalar (gevolution.hpp:251-340) without tensor or vector extras:
//   chi 2 k^4 N = S00 (g1+g2-2g0) + S11 (g0+g2-2g1) + S22 (g0+g1-2g2)
//                 - 6 (k0 k1 S01 + k0 k2 S02 + k1 k2 S12)
//               = A + g2 B - 6 k2 C, with
//   A = S00 (g1-2g0) + S11 (g0-2g1) + S22 (g0+g1) - 6 k0 k1 S01,
//   B = S00 + S11 - 2 S22,   C = k0 S02 + k1 S12.
// A, B, C have coefficients that depend on kx, ky only, so they are formed
// (in FP64) while the pencils load and the z transform -- linear, along kz --
// acts on three columns instead of six.
template <class R, int N, int T, int NT, int OP, int EXTRA>
__global__ void __launch_bounds__(NT, GEV_FZ_MINB * 256 / NT) k_fz(FzArgs<R> a, const typename CT<R>::C *__restrict__ tw)
{
    using C = typename CT<R>::C;
    constexpr int P = N / 2 + 1, PP = N / 2 + 2;
    constexpr int CIN = OpShape<OP, EXTRA>::CIN, COUT = OpShape<OP, EXTRA>::COUT;
    constexpr bool CONTRACT = OpShape<OP, EXTRA>::CONTRACT;
    constexpr int CBUF = OpShape<OP, EXTRA>::CBUF;
    constexpr int LD = CBUF * T + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *buf = reinterpret_cast<C *>(smem_raw);
    const int kx0 = blockIdx.x * T, ky = blockIdx.y;

    if constexpr (CONTRACT) {
        struct ABC { C v[3]; };
        staged_fill<N * T, NT, 2, ABC>(
            [&](int idx) {
                const int t = idx % T, n = idx / T, kx = kx0 + t;
                ABC o;
                if (kx >= P) {
                    o.v[0] = o.v[1] = o.v[2] = mk(R(0), R(0));
                    return o;
                }
                const int64_t k = kx + (int64_t)PP * (ky + (int64_t)N * n);
                double2 S[6];
#pragma unroll
                for (int c = 0; c < 6; c++) S[c] = z2d(a.data[c * a.stride + k]);
                const double g0 = __ldg(a.k2 + kx), g1 = __ldg(a.k2 + ky);
                const double2 k0 = __ldg(a.ks + kx), k1 = __ldg(a.ks + ky);
                const double2 A = zsub(zadd(zadd(zsc(S[0], g1 - 2.0 * g0), zsc(S[3], g0 - 2.0 * g1)), zsc(S[5], g0 + g1)),
                                       zsc(zmul(zmul(k0, k1), S[1]), 6.0));
                const double2 B = zsub(zadd(S[0], S[3]), zsc(S[5], 2.0));
                const double2 Cc = zadd(zmul(k0, S[2]), zmul(k1, S[4]));
                o.v[0] = mk(R(A.x), R(A.y));
                o.v[1] = mk(R(B.x), R(B.y));
                o.v[2] = mk(R(Cc.x), R(Cc.y));
                return o;
            },
            [&](int idx, ABC o) {
                const int t = idx % T, n = idx / T;
#pragma unroll
                for (int c = 0; c < 3; c++) buf[n * LD + c * T + t] = o.v[c];
            });
    } else {
        staged_fill<N * CIN * T, NT, 8, C>(
            [&](int idx) {
                const int t = idx % T, r = idx / T, c = r % CIN, n = r / CIN, kx = kx0 + t;
                return (kx < P) ? a.data[c * a.stride + kx + (int64_t)PP * (ky + (int64_t)N * n)] : mk(R(0), R(0));
            },
            [&](int idx, C v) {
                const int t = idx % T, r = idx / T, c = r % CIN, n = r / CIN;
                buf[n * LD + c * T + t] = v;
            });
    }
    __syncthreads();
    // one component at a time keeps the butterfly registers per thread small
#pragma unroll 1
    for (int c = 0; c < (CONTRACT ? 3 : CIN); c++) fft_lines<N, -1, T, NT>(buf + c * T, LD, tw);

    if constexpr (CONTRACT) {
        for (int idx = threadIdx.x; idx < N * T; idx += NT) {
            const int t = idx % T, n = idx / T, kx = kx0 + t;
            if (kx >= P) continue;
            const double g0 = __ldg(a.k2 + kx), g1 = __ldg(a.k2 + ky), g2 = __ldg(a.k2 + n);
            const double2 k2c = __ldg(a.ks + n);
            const double k2 = g0 + g1 + g2;
            double2 chi = make_double2(0.0, 0.0);
            if (k2 > 0.0) {
                const double2 A = z2d(buf[n * LD + t]), B = z2d(buf[n * LD + T + t]), Cc = z2d(buf[n * LD + 2 * T + t]);
                chi = zsub(zadd(A, zsc(B, g2)), zsc(zmul(k2c, Cc), 6.0));
                chi = zsc(chi, 1.0 / (2.0 * k2 * k2 * N));
            }
            buf[n * LD + t] = mk(R(chi.x), R(chi.y));
        }
    } else {
        for (int idx = threadIdx.x; idx < N * T; idx += NT) {
            int t = idx % T, n = idx / T, kx = kx0 + t;
            if (kx >= P) continue;
            double2 v[6];
#pragma unroll
            for (int c = 0; c < CIN; c++) v[c] = z2d(buf[n * LD + c * T + t]);
            int64_t kidx = kx + (int64_t)PP * (ky + (int64_t)N * n);
            fz_apply<R, OP, EXTRA>(a, N, kx, ky, n, kidx, v);
#pragma unroll
            for (int c = 0; c < COUT; c++) buf[n * LD + c * T + t] = mk(R(v[c].x), R(v[c].y));
        }
    }
    if constexpr (COUT > 0) {
        __syncthreads();
#pragma unroll 1
        for (int c = 0; c < COUT; c++) fft_lines<N, 1, T, NT>(buf + c * T, LD, tw);
        for (int idx = threadIdx.x; idx < N * COUT * T; idx += NT) {
            int t = idx % T, r = idx / T, c = r % COUT, n = r / COUT, kx = kx0 + t;
            if (kx < P) a.data[c * a.stride + kx + (int64_t)PP * (ky + (int64_t)N * n)] = buf[n * LD + c * T + t];
        }
    }
}

// z pass with tensor-memory-access staging: one elected thread loads the
// CTA's T kx-columns of every input component over all kz as bulk tensor
// copies (boxes of at most 256 kz) into dense per-component shared buffers,
// the CTA transforms, solves and inverse-transforms them, and the results
// leave by bulk tensor stores.  Columns kx >= P of the last CTA are zero-filled
// on load and clipped on store.  Same arithmetic as k_fz.
template <int N> struct ZBox {
    static constexpr int ZB = N <= 256 ? N : (N % 256 == 0 ? 256 : 128);
    static constexpr int NZB = N / ZB;
};

// the tensor extras keep six components in registers through the solve:
// compiled for one resident CTA instead of GEV_FZ_MINB
template <class R, int OP, int EXTRA, int NT> struct FzMinBlocks {
    static constexpr int v = (OpShape<OP, EXTRA>::CIN == 6 && !OpShape<OP, EXTRA>::CONTRACT)
                                 ? 1
                                 : (sizeof(R) == 4 ? GEV_FZ_MINB : GEV_FZ_MINB_D) * 256 / NT;
};

// PAD: the transforms use padded rows (fft.cuh), each component buffer then
// holds N + N / 8 rows of T values
template <class R, int N, int T, int NT, int OP, int EXTRA, bool PAD>
__global__ void __launch_bounds__(NT, (FzMinBlocks<R, OP, EXTRA, NT>::v))
    k_fz_tma(FzArgs<R> a, const typename CT<R>::C *__restrict__ tw, const __grid_constant__ CUtensorMap tmap)
{
    using C = typename CT<R>::C;
    constexpr int P = N / 2 + 1, PP = N / 2 + 2;
    constexpr int CIN = OpShape<OP, EXTRA>::CIN, COUT = OpShape<OP, EXTRA>::COUT;
    constexpr bool CONTRACT = OpShape<OP, EXTRA>::CONTRACT;
    constexpr int ZB = ZBox<N>::ZB, NZB = ZBox<N>::NZB;
    constexpr int CS = N * T;   // one component: [kz][t], dense
    constexpr int CSTR = PAD ? (N + N / 8) * T : CS;   // component buffer stride
    // bulk tensor copies want 128-byte aligned shared addresses: the launch
    // adds 128 bytes of slack and the buffers start at the next boundary
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *buf = reinterpret_cast<C *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t bar;
    const int kx0 = blockIdx.x * T, ky = blockIdx.y;

    // the contracted scalar solve loads S00, S01, S11, S22 into buffers 0..3,
    // folds them into A and B (buffers 0, 1), then loads S02, S12 into
    // buffers 2, 3 and folds them into C (buffer 2): four buffers instead of six
    constexpr int NL1 = CONTRACT ? 4 : CIN;
    auto first_comp = [](int s) { return CONTRACT ? (s == 2 ? 3 : (s == 3 ? 5 : s)) : s; };
    auto load = [&](int slot, int comp) {
#pragma unroll 1
        for (int zc = 0; zc < NZB; zc++) tma_load_4d(buf + slot * CSTR + zc * ZB * T, &tmap, 2 * kx0, ky, zc * ZB, comp, &bar);
    };
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (uint32_t)(NL1 * CS * sizeof(C)));
#pragma unroll 1
        for (int s = 0; s < NL1; s++) load(s, first_comp(s));
    }
    bool ok = mbar_wait(&bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0 && a.err) atomicOr(a.err, ERR_TMA_TIMEOUT);
        return;
    }

    if constexpr (CONTRACT) {
        // A, B, C of k_fz's projectFTscalar factorisation
        for (int idx = threadIdx.x; idx < CS; idx += NT) {
            const int t = idx % T, kx = kx0 + t;
            double2 A = make_double2(0.0, 0.0), B = A;
            if (kx < P) {
                const double2 S0 = z2d(buf[idx]), S1 = z2d(buf[CSTR + idx]);
                const double2 S3 = z2d(buf[2 * CSTR + idx]), S5 = z2d(buf[3 * CSTR + idx]);
                const double g0 = __ldg(a.k2 + kx), g1 = __ldg(a.k2 + ky);
                const double2 k0 = __ldg(a.ks + kx), k1 = __ldg(a.ks + ky);
                A = zsub(zadd(zadd(zsc(S0, g1 - 2.0 * g0), zsc(S3, g0 - 2.0 * g1)), zsc(S5, g0 + g1)),
                         zsc(zmul(zmul(k0, k1), S1), 6.0));
                B = zsub(zadd(S0, S3), zsc(S5, 2.0));
            }
            buf[idx] = mk(R(A.x), R(A.y));
            buf[CSTR + idx] = mk(R(B.x), R(B.y));
        }
        __syncthreads();   // buffers 2 and 3 are free
        if (threadIdx.x == 0) {
            fence_async_smem();
            mbar_expect_tx(&bar, (uint32_t)(2 * CS * sizeof(C)));
            load(2, 2);
            load(3, 4);
        }
        ok = mbar_wait(&bar, 1);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0 && a.err) atomicOr(a.err, ERR_TMA_TIMEOUT);
            return;
        }
        for (int idx = threadIdx.x; idx < CS; idx += NT) {
            const int t = idx % T, kx = kx0 + t;
            double2 Cc = make_double2(0.0, 0.0);
            if (kx < P) {
                const double2 S2 = z2d(buf[2 * CSTR + idx]), S4 = z2d(buf[3 * CSTR + idx]);
                const double2 k0 = __ldg(a.ks + kx), k1 = __ldg(a.ks + ky);
                Cc = zadd(zmul(k0, S2), zmul(k1, S4));
            }
            buf[2 * CSTR + idx] = mk(R(Cc.x), R(Cc.y));
        }
        __syncthreads();
    }
#pragma unroll 1
    for (int c = 0; c < (CONTRACT ? 3 : CIN); c++) fft_lines<N, -1, T, NT, PAD>(buf + c * CSTR, T, tw);

    for (int idx = threadIdx.x; idx < CS; idx += NT) {
        const int t = idx % T, n = idx / T, kx = kx0 + t;
        if (kx >= P) continue;
        if constexpr (CONTRACT) {
            const double g0 = __ldg(a.k2 + kx), g1 = __ldg(a.k2 + ky), g2 = __ldg(a.k2 + n);
            const double2 k2c = __ldg(a.ks + n);
            const double k2 = g0 + g1 + g2;
            double2 chi = make_double2(0.0, 0.0);
            if (k2 > 0.0) {
                const double2 A = z2d(buf[idx]), B = z2d(buf[CSTR + idx]), Cc = z2d(buf[2 * CSTR + idx]);
                chi = zsub(zadd(A, zsc(B, g2)), zsc(zmul(k2c, Cc), 6.0));
                chi = zsc(chi, 1.0 / (2.0 * k2 * k2 * N));
            }
            buf[idx] = mk(R(chi.x), R(chi.y));
        } else {
            double2 v[6];
#pragma unroll
            for (int c = 0; c < CIN; c++) v[c] = z2d(buf[c * CSTR + idx]);
            const int64_t kidx = kx + (int64_t)PP * (ky + (int64_t)N * n);
            fz_apply<R, OP, EXTRA>(a, N, kx, ky, n, kidx, v);
#pragma unroll
            for (int c = 0; c < COUT; c++) buf[c * CSTR + idx] = mk(R(v[c].x), R(v[c].y));
        }
    }
    if constexpr (COUT > 0) {
        __syncthreads();
#pragma unroll 1
        for (int c = 0; c < COUT; c++) fft_lines<N, 1, T, NT, PAD>(buf + c * CSTR, T, tw);
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll 1
            for (int c = 0; c < COUT; c++)
#pragma unroll 1
                for (int zc = 0; zc < NZB; zc++) tma_store_4d(&tmap, 2 * kx0, ky, zc * ZB, c, buf + c * CSTR + zc * ZB * T);
            tma_store_drain();
        }
    }
}

// y pass with bulk-tensor-copy staging: T kx-columns over all ky at one kz,
// in place.  grid (ceil(P/T), N, ncomp)
template <class R, int N, int T, int NT, int S>
__global__ void __launch_bounds__(NT, (sizeof(R) == 4 ? GEV_FY_MINB : 2) * 512 / NT) k_fy_tma(const typename CT<R>::C *__restrict__ tw,
                                                        int *err, const __grid_constant__ CUtensorMap tmap)
{
    using C = typename CT<R>::C;
    constexpr int YB = ZBox<N>::ZB, NYB = ZBox<N>::NZB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *buf = reinterpret_cast<C *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t bar;
    const int kx0 = blockIdx.x * T, z = blockIdx.y, comp = blockIdx.z;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (uint32_t)(N * T * sizeof(C)));
#pragma unroll 1
        for (int yc = 0; yc < NYB; yc++) tma_load_4d(buf + yc * YB * T, &tmap, 2 * kx0, yc * YB, z, comp, &bar);
    }
    const bool ok = mbar_wait(&bar, 0);
    if (__syncthreads_or(!ok)) {   // the data never arrived: leave the array untouched and say so
        if (threadIdx.x == 0 && err) atomicOr(err, ERR_TMA_TIMEOUT);
        return;
    }
    fft_lines<N, S, T, NT>(buf, T, tw);
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll 1
        for (int yc = 0; yc < NYB; yc++) tma_store_4d(&tmap, 2 * kx0, yc * YB, z, comp, buf + yc * YB * T);
        tma_store_drain();
    }
}

}  // namespace gev
