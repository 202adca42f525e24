// fft.cuh -- batched in-shared-memory FFTs for the pencil passes.
//
// T independent lines of length L sit in shared memory as buf[n*ld + t]
// (n = position along the transform, t = line, ld >= T).  The transform is the
// self-sorting Stockham formulation: every pass reads R points of a butterfly,
// applies twiddles and an R-point DFT in registers, and writes them back in
// place between two block-wide barriers, so no bit-reversal pass is needed.
// Lengths are compile-time constants factored into radices 2, 3, 4 and 8.
// Twiddles come from a table tw[k] = exp(-2 pi i k / L) computed on the host in
// double precision; inverse transforms use the conjugates.
//
// Padded rows (PAD): between two passes, row n lives at row n + n / 8, so the
// buffer needs L + L / 8 rows.  For dense buffers (ld = T) whose rows are
// narrower than a 128-byte bank line this makes the first pass's scattered
// writes (rows R j + r, a multiple of 128 bytes apart) conflict-free, while
// the other accesses of a warp (8 consecutive rows aligned to 8) stay
// contiguous.  The transform's input and output stay dense, in natural order.
#pragma once

#include "common.cuh"

namespace gev {

template <int L> struct Plan;
#define GEV_PLAN(LV, NS, R0, R1, R2, R3)                                                   \
    template <> struct Plan<LV> {                                                          \
        static constexpr int ns = NS;                                                      \
        __host__ __device__ static constexpr int r(int i) { return i == 0 ? R0 : (i == 1 ? R1 : (i == 2 ? R2 : R3)); } \
    };
GEV_PLAN(8, 1, 8, 1, 1, 1)
GEV_PLAN(16, 2, 4, 4, 1, 1)
GEV_PLAN(32, 2, 4, 8, 1, 1)
GEV_PLAN(64, 2, 8, 8, 1, 1)
// radix-8 passes first: with padded rows every pass of a dense buffer is then
// free of bank conflicts
GEV_PLAN(128, 3, 8, 8, 2, 1)
GEV_PLAN(192, 3, 3, 8, 8, 1)
GEV_PLAN(256, 3, 4, 8, 8, 1)
GEV_PLAN(384, 4, 8, 8, 2, 3)
GEV_PLAN(512, 3, 8, 8, 8, 1)
GEV_PLAN(768, 4, 8, 8, 4, 3)
#undef GEV_PLAN

// ---- R-point DFTs in registers, exponent sign S (-1 forward, +1 inverse) ----
template <int S, class C> __device__ __forceinline__ void dft2(C &a, C &b)
{
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int S, class C> __device__ __forceinline__ void dft4(C &x0, C &x1, C &x2, C &x3)
{
    C a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), d = cmul_si<S>(csub(x1, x3));
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd(b, d);
    x3 = csub(b, d);
}

template <int R, int S, class C> __device__ __forceinline__ void dft(C *v);

template <> __device__ __forceinline__ void dft<2, -1, float2>(float2 *v) { dft2<-1>(v[0], v[1]); }
template <> __device__ __forceinline__ void dft<2, 1, float2>(float2 *v) { dft2<1>(v[0], v[1]); }
template <> __device__ __forceinline__ void dft<2, -1, double2>(double2 *v) { dft2<-1>(v[0], v[1]); }
template <> __device__ __forceinline__ void dft<2, 1, double2>(double2 *v) { dft2<1>(v[0], v[1]); }

template <int S, class C> __device__ __forceinline__ void dft4v(C *v) { dft4<S>(v[0], v[1], v[2], v[3]); }

template <int S, class C> __device__ __forceinline__ void dft3v(C *v)
{
    using R = decltype(v[0].x);
    const R h = R(0.8660254037844386467637231707529362);  // sqrt(3)/2
    C t1 = cadd(v[1], v[2]);
    C t2 = cmul_si<S>(cscale(csub(v[1], v[2]), h));
    C m = csub(v[0], cscale(t1, R(0.5)));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, t2);
    v[2] = csub(m, t2);
}

template <int S, class C> __device__ __forceinline__ void dft8v(C *v)
{
    using R = decltype(v[0].x);
    const R r2 = R(0.7071067811865475244008443621048490);  // sqrt(2)/2
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<S>(e0, e1, e2, e3);
    dft4<S>(o0, o1, o2, o3);
    // o_k *= exp(S 2 pi i k / 8)
    C t;
    t.x = r2 * (o1.x - S * o1.y);
    t.y = r2 * (o1.y + S * o1.x);
    o1 = t;
    o2 = cmul_si<S>(o2);
    t.x = r2 * (-o3.x - S * o3.y);
    t.y = r2 * (-o3.y + S * o3.x);
    o3 = t;
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <int R, int S, class C> __device__ __forceinline__ void dftR(C *v)
{
    if constexpr (R == 2) { dft2<S>(v[0], v[1]); }
    else if constexpr (R == 3) { dft3v<S>(v); }
    else if constexpr (R == 4) { dft4v<S>(v); }
    else if constexpr (R == 8) { dft8v<S>(v); }
}

// row n0 + r * STRIDE of the buffer, padded if PAD; n0 + (n0 >> 3) is hoisted
// out of the loop over r where the block of 8 rows of each r is known:
// STRIDE a multiple of 8, or STRIDE = 1 with n0 a multiple of a radix RAD
// that divides 8 (the rows n0 .. n0 + RAD - 1 share their block)
template <bool PAD, int STRIDE, int RAD> __device__ __forceinline__ int pad_row(int n0, int r)
{
    if constexpr (!PAD) return n0 + r * STRIDE;
    else if constexpr (STRIDE % 8 == 0) return n0 + (n0 >> 3) + r * (STRIDE + STRIDE / 8);
    else if constexpr (STRIDE == 1 && 8 % RAD == 0) return n0 + (n0 >> 3) + r;
    else {
        const int n = n0 + r * STRIDE;
        return n + (n >> 3);
    }
}

// One Stockham pass of radix R with span NS over T lines; rows are read
// padded if PI and written padded if PO.
template <int L, int R, int NS, int S, int T, int NT, bool PI, bool PO, class C>
__device__ __forceinline__ void stockham_pass(C *buf, int ld, const C *__restrict__ tw)
{
    constexpr int NB = L / R;
    constexpr int TOT = NB * T;
    constexpr int BPT = (TOT + NT - 1) / NT;
    C v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; b++) {
        int idx = threadIdx.x + b * NT;
        if (BPT * NT == TOT || idx < TOT) {
            int t = idx % T, j = idx / T;
#pragma unroll
            for (int r = 0; r < R; r++) v[b][r] = buf[pad_row<PI, NB, R>(j, r) * ld + t];
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < BPT; b++) {
        int idx = threadIdx.x + b * NT;
        if (BPT * NT == TOT || idx < TOT) {
            int t = idx % T, j = idx / T;
            int jm = j % NS;
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    C w = __ldg(tw + r * jm * (L / (NS * R)));
                    if constexpr (S > 0) w.y = -w.y;
                    v[b][r] = cmul(v[b][r], w);
                }
            }
            dftR<R, S>(v[b]);
            int idxD = (j / NS) * NS * R + jm;
#pragma unroll
            for (int r = 0; r < R; r++) buf[pad_row<PO, NS, R>(idxD, r) * ld + t] = v[b][r];
        }
    }
    __syncthreads();
}

template <int L, int S, int T, int NT, bool PAD, int STAGE, int NS> struct FftStages {
    template <class C> static __device__ __forceinline__ void run(C *buf, int ld, const C *__restrict__ tw)
    {
        if constexpr (STAGE < Plan<L>::ns) {
            constexpr int R = Plan<L>::r(STAGE);
            constexpr bool PI = PAD && STAGE > 0, PO = PAD && STAGE < Plan<L>::ns - 1;
            stockham_pass<L, R, NS, S, T, NT, PI, PO>(buf, ld, tw);
            FftStages<L, S, T, NT, PAD, STAGE + 1, NS * R>::run(buf, ld, tw);
        }
    }
};

// Transform T lines of length L in place (unnormalised).  Caller must have
// issued __syncthreads() after filling buf; returns after a barrier.  With
// PAD the buffer holds L + L / 8 rows.
template <int L, int S, int T, int NT, bool PAD = false, class C>
__device__ __forceinline__ void fft_lines(C *buf, int ld, const C *__restrict__ tw)
{
    FftStages<L, S, T, NT, PAD, 0, 1>::run(buf, ld, tw);
}

// rows of a dense buffer (ld = T) that padding spreads over the banks
template <int T, class C> constexpr bool pad_helps() { return T * (int)sizeof(C) < 128; }

}  // namespace gev
