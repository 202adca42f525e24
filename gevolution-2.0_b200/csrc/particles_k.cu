// particles_k.cu -- geodesic kick + drift, tile re-bucketing, particle I/O.
//
// Kick and drift follow update_q (gevolution.hpp:888-1011, GRADIENT_ORDER 2)
// and update_pos (:1162-1232) term by term, in the field precision R (FP32 in
// mixed mode) with the in-cell offsets updated in FP64.  One CTA handles one
// tile's particles and stages phi, chi and B_i over the tile plus the stencil
// reach ([-1, 10)^3 relative to the tile origin) in shared memory, so every
// gather is a shared-memory read.  The drift moves the cell index and the FP64
// in-cell offset and assigns the particle its new bucket; a warp-aggregated
// counter gives it a slot, and launch_rebin moves it into bucket order -- and
// inside each bucket into (cell, ID) order -- after an exclusive scan of the
// bucket counts (the re-binning that LATfield2's moveParticles does into its
// row buffers).
#include <algorithm>
#include "common.cuh"
#include "kernels.h"
#include "particles.cuh"

namespace gev {

constexpr int KD_NT = 256;
constexpr int KD_W = 11;   // staged extent per axis

template <class R>
__device__ __forceinline__ R SF(const R *s, int rx, int ry, int rz, int dx, int dy, int dz)
{
    return s[(rx + 1 + dx) + KD_W * ((ry + 1 + dy) + KD_W * (rz + 1 + dz))];
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// 1/x and 1/sqrt(x) in the field precision: the geodesic's divisions by e^2,
// sqrt(e^2) and the uniform coefficients become multiplications (FP32: the
// hardware reciprocal square root, within 2 ulp; FP64: correctly rounded
// division and square root)
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip(double x) { return 1.0 / x; }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return 1.0 / sqrt(x); }

// slot within bucket b, warp-aggregated (order inside a bucket is not significant)
__device__ __forceinline__ uint32_t bucket_slot(uint32_t b, uint32_t *counts)
{
    unsigned act = __activemask();
    unsigned peers = __match_any_sync(act, b);
    int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&counts[b], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + (uint32_t)__popc(peers & lanemask_lt());
}

template <class R>
__global__ void __launch_bounds__(KD_NT, sizeof(R) == 4 ? 4 : 2) k_kick_drift(PView<R> p, const uint32_t *__restrict__ bstart, int N, int nt,
                                                      const R *__restrict__ phi, const R *__restrict__ chi,
                                                      const R *__restrict__ Bi, int64_t n3, KickDriftParams kp,
                                                      uint32_t *counts, uint32_t *bucket, uint32_t *rank,
                                                      unsigned long long *vmax_bits, int *err, FastDiv fN)
{
    extern __shared__ __align__(16) unsigned char kd_smem[];
    R(*sf)[KD_W * KD_W * KD_W] = reinterpret_cast<R(*)[KD_W * KD_W * KD_W]>(kd_smem);
    __shared__ double wmax[KD_NT / 32];
    const int tile = blockIdx.x;
    const int tx = tile % nt, ty = (tile / nt) % nt, tz = tile / (nt * nt);
    const int x0 = tx * 8, y0 = ty * 8, z0 = tz * 8;

    const bool need_phi = kp.do_kick || (kp.do_drift && kp.nfield_d >= 1);
    const bool need_chi = (kp.do_kick && kp.nfield_k >= 2) || (kp.do_drift && kp.nfield_d >= 2);
    const bool need_B = (kp.do_kick && kp.nfield_k >= 3) || (kp.do_drift && kp.nfield_d >= 3);
    {
        // all loads of this thread's share first, then the shared-memory stores,
        // so that up to PER*5 global loads are in flight per thread
        constexpr int NS = KD_W * KD_W * KD_W;
        constexpr int PER = (NS + KD_NT - 1) / KD_NT;
        int64_t gi[PER];
        R v[PER][5];
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const int i = threadIdx.x + k * KD_NT;
            const int ii = i < NS ? i : NS - 1;
            const int vx = ii % KD_W - 1, vy = (ii / KD_W) % KD_W - 1, vz = ii / (KD_W * KD_W) - 1;
            gi[k] = sidx(N, wrapi(x0 + vx, N), wrapi(y0 + vy, N), wrapi(z0 + vz, N));
        }
#pragma unroll
        for (int k = 0; k < PER; k++) {
            if (need_phi) v[k][0] = __ldg(phi + gi[k]);
            if (need_chi) v[k][1] = __ldg(chi + gi[k]);
            if (need_B) {
                v[k][2] = __ldg(Bi + gi[k]);
                v[k][3] = __ldg(Bi + n3 + gi[k]);
                v[k][4] = __ldg(Bi + 2 * n3 + gi[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const int i = threadIdx.x + k * KD_NT;
            if (i < NS) {
                if (need_phi) sf[0][i] = v[k][0];
                if (need_chi) sf[1][i] = v[k][1];
                if (need_B) { sf[2][i] = v[k][2]; sf[3][i] = v[k][3]; sf[4][i] = v[k][4]; }
            }
        }
    }
    __syncthreads();
    const R *P_ = sf[0], *X_ = sf[1], *B0 = sf[2], *B1 = sf[3], *B2 = sf[4];

    const uint32_t lo = bstart[8 * tile], hi = bstart[8 * tile + 8];
    R lmax = 0;   // max of q^2 / a^2 (converted to FP64 once, at the end)
    const R ib_k = (R)(1.0 / kp.b_k), ib_d = (R)(1.0 / kp.b_d);
    const R ia2_k = (R)(1.0 / (kp.a_k * kp.a_k));
    const double dtau_N = kp.dtau_d * (double)N;   // box units -> cell units
    for (uint32_t base = lo; base < hi; base += 2 * KD_NT) {
        // two particles per thread and pass: both loads are issued before either is used
        RawParticle<R> raw[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint32_t i = base + threadIdx.x + u * KD_NT;
            if (i < hi) raw[u] = load_particle(p, i);
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
        const uint32_t i = base + threadIdx.x + u * KD_NT;
        if (i >= hi) continue;
        const RawParticle<R> &pr = raw[u];
        int cx, cy, cz;
        decode_cell(pr.cell, fN, cx, cy, cz);
        int rx = cx - x0, ry = cy - y0, rz = cz - z0;
        // a particle outside this tile means the bucket order is stale: flag it, leave it
        // unmoved (never read outside the stage) and still give it a bucket slot
        const bool ok = !(rx < 0 || rx > 7 || ry < 0 || ry > 7 || rz < 0 || rz > 7);
        if (!ok) atomicOr(err, ERR_BAD_CELL);
        if (!ok) { rx = ry = rz = 0; cx = x0; cy = y0; cz = z0; }
        // FP64 offsets for the position update; the interpolation weights and the
        // geodesic arithmetic run in the field precision R
        const double dd[3] = {pr.off[0], pr.off[1], pr.off[2]};
        const R d[3] = {(R)dd[0], (R)dd[1], (R)dd[2]};
        R v[3] = {pr.q[0], pr.q[1], pr.q[2]};
        R w8[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            w8[k] = (((k >> 2) & 1) ? d[0] : (R)1 - d[0]) * (((k >> 1) & 1) ? d[1] : (R)1 - d[1]) * ((k & 1) ? d[2] : (R)1 - d[2]);

        // The drift interpolates phi and B_i at the position the kick used
        // (the particle has not moved yet): when both run, the kick's sums are
        // kept for it -- phi(x) and the bilinear B_i interpolations in the
        // planes x_i = 0 of the cell.
        R phi_x = 0, B_x[3] = {0, 0, 0};
        bool kick_phi = false, kick_B = false;
        if (kp.do_kick && ok) {
            // update_q, gevolution.hpp:888-1011
            const R a = (R)kp.a_k;
            R gradphi[3];
            R v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            R e2 = v2 + a * a;
            R phiint = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) phiint += w8[k] * SF(P_, rx, ry, rz, (k >> 2) & 1, (k >> 1) & 1, k & 1);
            phi_x = phiint;
            kick_phi = true;
            const R ie2 = recip(e2);
            phiint *= ie2;
            phiint = (R)4 * phiint * v2 + ((R)1 + a * a * phiint) * (v2 + e2) * ie2;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int ex = c == 0, ey = c == 1, ez = c == 2;
                R g = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
                    g += (R)0.5 * w8[k] * (SF(P_, rx, ry, rz, bx + ex, by + ey, bz + ez) - SF(P_, rx, ry, rz, bx - ex, by - ey, bz - ez));
                }
                gradphi[c] = g * phiint;
            }
            if (kp.nfield_k >= 2) {
                gradphi[0] -= (1 - d[1]) * (1 - d[2]) * (SF(X_, rx, ry, rz, 1, 0, 0) - SF(X_, rx, ry, rz, 0, 0, 0));
                gradphi[1] -= (1 - d[0]) * (1 - d[2]) * (SF(X_, rx, ry, rz, 0, 1, 0) - SF(X_, rx, ry, rz, 0, 0, 0));
                gradphi[2] -= (1 - d[0]) * (1 - d[1]) * (SF(X_, rx, ry, rz, 0, 0, 1) - SF(X_, rx, ry, rz, 0, 0, 0));
                gradphi[0] -= d[1] * (1 - d[2]) * (SF(X_, rx, ry, rz, 1, 1, 0) - SF(X_, rx, ry, rz, 0, 1, 0));
                gradphi[1] -= d[0] * (1 - d[2]) * (SF(X_, rx, ry, rz, 1, 1, 0) - SF(X_, rx, ry, rz, 1, 0, 0));
                gradphi[2] -= d[0] * (1 - d[1]) * (SF(X_, rx, ry, rz, 1, 0, 1) - SF(X_, rx, ry, rz, 1, 0, 0));
                gradphi[0] -= (1 - d[1]) * d[2] * (SF(X_, rx, ry, rz, 1, 0, 1) - SF(X_, rx, ry, rz, 0, 0, 1));
                gradphi[1] -= (1 - d[0]) * d[2] * (SF(X_, rx, ry, rz, 0, 1, 1) - SF(X_, rx, ry, rz, 0, 0, 1));
                gradphi[2] -= (1 - d[0]) * d[1] * (SF(X_, rx, ry, rz, 0, 1, 1) - SF(X_, rx, ry, rz, 0, 1, 0));
                gradphi[0] -= d[1] * d[2] * (SF(X_, rx, ry, rz, 1, 1, 1) - SF(X_, rx, ry, rz, 0, 1, 1));
                gradphi[1] -= d[0] * d[2] * (SF(X_, rx, ry, rz, 1, 1, 1) - SF(X_, rx, ry, rz, 1, 0, 1));
                gradphi[2] -= d[0] * d[1] * (SF(X_, rx, ry, rz, 1, 1, 1) - SF(X_, rx, ry, rz, 1, 1, 0));
            }
            const R ie = rsqrt_r(e2);
            e2 *= ie;   // sqrt(q^2 + a^2)
            if (kp.nfield_k >= 3) {
                // gevolution.hpp:970-993.  The (d-1) B(-1) + (1-2d) B(0) + d B(1)
                // terms, weighted over the other two axes, are evaluated as that
                // combination of the bilinear interpolations I(-1), I(0), I(1)
                // of the three planes (the same quantity, fewer operations).
                const R wyz[4] = {(1 - d[1]) * (1 - d[2]), d[1] * (1 - d[2]), (1 - d[1]) * d[2], d[1] * d[2]};
                const R wxz[4] = {(1 - d[0]) * (1 - d[2]), d[0] * (1 - d[2]), (1 - d[0]) * d[2], d[0] * d[2]};
                const R wxy[4] = {(1 - d[0]) * (1 - d[1]), d[0] * (1 - d[1]), (1 - d[0]) * d[1], d[0] * d[1]};
                auto I0 = [&](int x) {
                    return wyz[0] * SF(B0, rx, ry, rz, x, 0, 0) + wyz[1] * SF(B0, rx, ry, rz, x, 1, 0) +
                           wyz[2] * SF(B0, rx, ry, rz, x, 0, 1) + wyz[3] * SF(B0, rx, ry, rz, x, 1, 1);
                };
                auto I1 = [&](int y) {
                    return wxz[0] * SF(B1, rx, ry, rz, 0, y, 0) + wxz[1] * SF(B1, rx, ry, rz, 1, y, 0) +
                           wxz[2] * SF(B1, rx, ry, rz, 0, y, 1) + wxz[3] * SF(B1, rx, ry, rz, 1, y, 1);
                };
                auto I2 = [&](int z) {
                    return wxy[0] * SF(B2, rx, ry, rz, 0, 0, z) + wxy[1] * SF(B2, rx, ry, rz, 1, 0, z) +
                           wxy[2] * SF(B2, rx, ry, rz, 0, 1, z) + wxy[3] * SF(B2, rx, ry, rz, 1, 1, z);
                };
                B_x[0] = I0(0);
                B_x[1] = I1(0);
                B_x[2] = I2(0);
                kick_B = true;
                R pg[3];
                pg[0] = ((1 - d[2]) * (SF(B1, rx, ry, rz, 1, 0, 0) - SF(B1, rx, ry, rz, 0, 0, 0)) + d[2] * (SF(B1, rx, ry, rz, 1, 0, 1) - SF(B1, rx, ry, rz, 0, 0, 1))) * v[1];
                pg[0] += ((1 - d[1]) * (SF(B2, rx, ry, rz, 1, 0, 0) - SF(B2, rx, ry, rz, 0, 0, 0)) + d[1] * (SF(B2, rx, ry, rz, 1, 1, 0) - SF(B2, rx, ry, rz, 0, 1, 0))) * v[2];
                pg[0] += ((d[0] - 1) * I0(-1) + (1 - 2 * d[0]) * B_x[0] + d[0] * I0(1)) * v[0];

                pg[1] = ((1 - d[0]) * (SF(B2, rx, ry, rz, 0, 1, 0) - SF(B2, rx, ry, rz, 0, 0, 0)) + d[0] * (SF(B2, rx, ry, rz, 1, 1, 0) - SF(B2, rx, ry, rz, 1, 0, 0))) * v[2];
                pg[1] += ((1 - d[2]) * (SF(B0, rx, ry, rz, 0, 1, 0) - SF(B0, rx, ry, rz, 0, 0, 0)) + d[2] * (SF(B0, rx, ry, rz, 0, 1, 1) - SF(B0, rx, ry, rz, 0, 0, 1))) * v[0];
                pg[1] += ((d[1] - 1) * I1(-1) + (1 - 2 * d[1]) * B_x[1] + d[1] * I1(1)) * v[1];

                pg[2] = ((1 - d[1]) * (SF(B0, rx, ry, rz, 0, 0, 1) - SF(B0, rx, ry, rz, 0, 0, 0)) + d[1] * (SF(B0, rx, ry, rz, 0, 1, 1) - SF(B0, rx, ry, rz, 0, 1, 0))) * v[0];
                pg[2] += ((1 - d[0]) * (SF(B1, rx, ry, rz, 0, 0, 1) - SF(B1, rx, ry, rz, 0, 0, 0)) + d[0] * (SF(B1, rx, ry, rz, 1, 0, 1) - SF(B1, rx, ry, rz, 1, 0, 0))) * v[1];
                pg[2] += ((d[2] - 1) * I2(-1) + (1 - 2 * d[2]) * B_x[2] + d[2] * I2(1)) * v[2];
#pragma unroll
                for (int c = 0; c < 3; c++) gradphi[c] += pg[c] * (ib_k * ie);
            }
            v2 = 0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                v[c] -= (R)kp.dtau_k * e2 * gradphi[c] * (R)N;
                v2 += v[c] * v[c];
            }
            lmax = fmax(lmax, v2 * ia2_k);
#pragma unroll
            for (int c = 0; c < 3; c++) p.q[c * p.cap + i] = v[c];
        }

        if (kp.do_drift && ok) {
            // update_pos, gevolution.hpp:1162-1232: the drift uses the kicked
            // momentum as stored (v holds it: the storage precision is R)
            const R a = (R)kp.a_d;
            R v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            R e2 = v2 + a * a;
            R ph = 0, ch = 0;
            if (kp.nfield_d >= 1) {
                if (kick_phi) {
                    ph = phi_x;
                } else {
#pragma unroll
                    for (int k = 0; k < 8; k++) ph += w8[k] * SF(P_, rx, ry, rz, (k >> 2) & 1, (k >> 1) & 1, k & 1);
                }
            }
            if (kp.nfield_d >= 2) {
#pragma unroll
                for (int k = 0; k < 8; k++) ch += w8[k] * SF(X_, rx, ry, rz, (k >> 2) & 1, (k >> 1) & 1, k & 1);
            }
            v2 = ((R)1 + ((R)3 - v2 * recip(e2)) * ph - ch) * rsqrt_r(e2);
            R dp[3] = {v[0] * v2, v[1] * v2, v[2] * v2};
            if (kp.nfield_d >= 3) {
                if (!kick_B) {
                    // the kick's bilinear interpolations, in the same form
                    const R wyz[4] = {(1 - d[1]) * (1 - d[2]), d[1] * (1 - d[2]), (1 - d[1]) * d[2], d[1] * d[2]};
                    const R wxz[4] = {(1 - d[0]) * (1 - d[2]), d[0] * (1 - d[2]), (1 - d[0]) * d[2], d[0] * d[2]};
                    const R wxy[4] = {(1 - d[0]) * (1 - d[1]), d[0] * (1 - d[1]), (1 - d[0]) * d[1], d[0] * d[1]};
                    B_x[0] = wyz[0] * SF(B0, rx, ry, rz, 0, 0, 0) + wyz[1] * SF(B0, rx, ry, rz, 0, 1, 0) +
                             wyz[2] * SF(B0, rx, ry, rz, 0, 0, 1) + wyz[3] * SF(B0, rx, ry, rz, 0, 1, 1);
                    B_x[1] = wxz[0] * SF(B1, rx, ry, rz, 0, 0, 0) + wxz[1] * SF(B1, rx, ry, rz, 1, 0, 0) +
                             wxz[2] * SF(B1, rx, ry, rz, 0, 0, 1) + wxz[3] * SF(B1, rx, ry, rz, 1, 0, 1);
                    B_x[2] = wxy[0] * SF(B2, rx, ry, rz, 0, 0, 0) + wxy[1] * SF(B2, rx, ry, rz, 1, 0, 0) +
                             wxy[2] * SF(B2, rx, ry, rz, 0, 1, 0) + wxy[3] * SF(B2, rx, ry, rz, 1, 1, 0);
                }
                dp[0] += B_x[0] * ib_d;
                dp[1] += B_x[1] * ib_d;
                dp[2] += B_x[2] * ib_d;
            }
            int cc[3] = {cx, cy, cz};
#pragma unroll
            for (int c = 0; c < 3; c++) {
                double o = dd[c] + dtau_N * (double)dp[c];
                if (!isfinite(o)) { atomicOr(err, ERR_NONFINITE); o = dd[c]; }
                double s = floor(o);
                o -= s;
                if (o >= 1.0) { o = 0.0; s += 1.0; }
                long long sh = (long long)s;
                long long nc = (long long)cc[c] + sh;
                if (nc < 0 || nc >= N) {   // crossed the periodic boundary (or moved far)
                    nc %= N;
                    if (nc < 0) nc += N;
                }
                cc[c] = (int)nc;
                p.off[c * p.cap + i] = o;
            }
            cx = cc[0]; cy = cc[1]; cz = cc[2];
            p.cell[i] = (uint32_t)sidx(N, cx, cy, cz);
        }
        if (kp.do_bin) {
            uint32_t b = bucket_of_cell(N, nt, cx, cy, cz);
            bucket[i] = b;
            rank[i] = bucket_slot(b, counts);
        }
        }
    }

    for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = (double)lmax;
    __syncthreads();
    if (threadIdx.x == 0 && kp.do_kick) {
        double m = 0.0;
        for (int w = 0; w < KD_NT / 32; w++) m = fmax(m, wmax[w]);
        atomicMax(vmax_bits, (unsigned long long)__double_as_longlong(m));
    }
}

template <class R>
void launch_kick_drift(const PView<R> &p, const uint32_t *bstart, int N, const R *phi, const R *chi, const R *Bi,
                       int64_t n3, const KickDriftParams &kp, uint32_t *counts, uint32_t *bucket, uint32_t *rank,
                       unsigned long long *vmax_bits, int *err, cudaStream_t st)
{
    int nt = N / 8;
    const size_t smem = 5 * KD_W * KD_W * KD_W * sizeof(R);
    static bool attr_set[SMEM_ATTR_DEVICES] = {};
    raise_smem_limit(k_kick_drift<R>, smem, attr_set);
    k_kick_drift<R><<<(unsigned)nt * nt * nt, KD_NT, smem, st>>>(p, bstart, N, nt, phi, chi, Bi, n3, kp, counts,
                                                                bucket, rank, vmax_bits, err, FastDiv((uint32_t)N));
}

// ---- particle I/O: host layout (box-unit positions, AoS triples) <-> cell + offset ----
template <class R>
__global__ void k_load_particles(PView<R> p, const double *pos, const double *q, const int64_t *id, int64_t n, int N,
                                 int *err)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double x = pos[3 * i + k];
        if (!isfinite(x)) { atomicOr(err, ERR_NONFINITE); x = 0.0; }
        x -= floor(x);
        double s = x * N;
        double f = floor(s);
        double o = s - f;
        int ci = (int)f;
        if (ci >= N) { ci = N - 1; o = 1.0 - 1e-16; }
        if (ci < 0) { ci = 0; o = 0.0; }
        c[k] = ci;
        p.off[k * p.cap + i] = o;
        p.q[k * p.cap + i] = (R)q[3 * i + k];
    }
    p.cell[i] = (uint32_t)sidx(N, c[0], c[1], c[2]);
    p.id[i] = id ? id[i] : i;
}

template <class R>
__global__ void k_store_particles(PView<R> p, double *pos, double *q, int64_t *id, int64_t n, int N)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t cell = p.cell[i];
    int c[3] = {(int)(cell % (uint32_t)N), (int)((cell / (uint32_t)N) % (uint32_t)N), (int)(cell / ((uint32_t)N * (uint32_t)N))};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (pos) pos[3 * i + k] = ((double)c[k] + p.off[k * p.cap + i]) / (double)N;
        if (q) q[3 * i + k] = (double)p.q[k * p.cap + i];
    }
    if (id) id[i] = p.id[i];
}

template <class R>
void launch_load_particles(PView<R> p, const double *pos, const double *q, const int64_t *id, int64_t n, int N,
                           int *err, cudaStream_t st)
{
    if (n > 0) k_load_particles<R><<<cdiv(n, 256), 256, 0, st>>>(p, pos, q, id, n, N, err);
}

template <class R>
void launch_store_particles(const PView<R> &p, double *pos, double *q, int64_t *id, int64_t n, int N,
                            cudaStream_t st)
{
    if (n > 0) k_store_particles<R><<<cdiv(n, 256), 256, 0, st>>>(p, pos, q, id, n, N);
}

template <class R>
__global__ void k_bin_count(PView<R> p, int N, int nt, uint32_t *counts, uint32_t *bucket, uint32_t *rank)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    uint32_t cell = p.cell[i];
    if ((int64_t)cell >= (int64_t)N * N * N) cell = 0;   // loaded cells are always in range; never index past the counts
    int cx = (int)(cell % (uint32_t)N), cy = (int)((cell / (uint32_t)N) % (uint32_t)N), cz = (int)(cell / ((uint32_t)N * (uint32_t)N));
    uint32_t b = bucket_of_cell(N, nt, cx, cy, cz);
    bucket[i] = b;
    rank[i] = bucket_slot(b, counts);
}

template <class R>
void launch_bin_count(const PView<R> &p, int N, uint32_t *counts, uint32_t *bucket, uint32_t *rank, cudaStream_t st)
{
    if (p.n > 0) k_bin_count<R><<<cdiv(p.n, 256), 256, 0, st>>>(p, N, N / 8, counts, bucket, rank);
}

// ---- exclusive scan of bucket counts: start[0..nb] ----
constexpr int SCAN_NT = 1024;

__global__ void k_scan_blocks(const uint32_t *counts, uint32_t *start, int64_t nb, uint32_t *block_sums)
{
    __shared__ uint32_t s[SCAN_NT];
    int64_t i = blockIdx.x * (int64_t)SCAN_NT + threadIdx.x;
    uint32_t v = (i < nb) ? counts[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < SCAN_NT; o <<= 1) {
        uint32_t t = (threadIdx.x >= (unsigned)o) ? s[threadIdx.x - o] : 0u;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < nb) start[i] = s[threadIdx.x] - v;
    if (threadIdx.x == SCAN_NT - 1) block_sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void k_scan_sums(uint32_t *block_sums, int64_t nblk, uint32_t *start, int64_t nb)
{
    __shared__ uint32_t s[SCAN_NT];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t b0 = 0; b0 < nblk; b0 += SCAN_NT) {
        int64_t i = b0 + threadIdx.x;
        uint32_t v = (i < nblk) ? block_sums[i] : 0u;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < SCAN_NT; o <<= 1) {
            uint32_t t = (threadIdx.x >= (unsigned)o) ? s[threadIdx.x - o] : 0u;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nblk) block_sums[i] = carry + s[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == SCAN_NT - 1) carry += s[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) start[nb] = carry;
}

__global__ void k_scan_add(uint32_t *start, int64_t nb, const uint32_t *block_sums)
{
    int64_t i = blockIdx.x * (int64_t)SCAN_NT + threadIdx.x;
    if (i < nb) start[i] += block_sums[blockIdx.x];
}

void launch_scan(const uint32_t *counts, uint32_t *start, int64_t nb, uint32_t *block_sums, cudaStream_t st)
{
    int64_t nblk = (nb + SCAN_NT - 1) / SCAN_NT;
    k_scan_blocks<<<(unsigned)nblk, SCAN_NT, 0, st>>>(counts, start, nb, block_sums);
    k_scan_sums<<<1, SCAN_NT, 0, st>>>(block_sums, nblk, start, nb);
    k_scan_add<<<(unsigned)nblk, SCAN_NT, 0, st>>>(start, nb, block_sums);
}

// ---- re-binning into bucket order, each bucket in (cell, ID) order ----
// Step 1: every particle's destination j = start[bucket] + slot; inv[j] = i.
__global__ void k_scatter_index(const uint32_t *__restrict__ bstart, const uint32_t *__restrict__ bucket,
                                const uint32_t *__restrict__ rank, int64_t n, uint32_t *inv)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t j = bstart[bucket[i]] + rank[i];
    if ((int64_t)j < n) inv[j] = (uint32_t)i;   // inconsistent counts: never write out of range
}

constexpr int RB_NT = 512;   // one thread per tile cell in the counting sort

template <class R> constexpr size_t rb_smem_bytes()
{
    // per particle: id, off[3], q[3], cell, source index, cell rank, slot, sorted index
    return (size_t)REBIN_SORT_MAX * (sizeof(int64_t) + 3 * sizeof(double) + 3 * sizeof(R) + sizeof(uint32_t) + 3 * sizeof(uint16_t));
}

// Step 2: one CTA per destination tile.  The tile's particles (or, for a tile
// of more than REBIN_SORT_MAX, each of its buckets that small) are loaded once
// from their source positions into shared memory, sorted there -- counting
// sort by class_ord of the cell, then insertion sort by ID inside each cell --
// and written to the sorted destination positions (coalesced writes).  A
// bucket larger than REBIN_SORT_MAX is copied in slot order.
template <class R>
__global__ void __launch_bounds__(RB_NT) k_rebin_tile(PView<R> src, PView<R> dst, const uint32_t *__restrict__ bstart,
                                                      const uint32_t *__restrict__ inv, int nt, int *err, FastDiv fN)
{
    constexpr int M = REBIN_SORT_MAX;
    extern __shared__ __align__(16) unsigned char rb_smem[];
    int64_t *s_id = reinterpret_cast<int64_t *>(rb_smem);
    double *s_off = reinterpret_cast<double *>(s_id + M);          // 3 planes of M
    R *s_q = reinterpret_cast<R *>(s_off + 3 * M);                 // 3 planes of M
    uint32_t *s_cell = reinterpret_cast<uint32_t *>(s_q + 3 * M);
    uint16_t *s_ord = reinterpret_cast<uint16_t *>(s_cell + M);
    uint16_t *s_slot = s_ord + M;
    uint16_t *s_order = s_slot + M;
    __shared__ int s_cnt[512], s_start[512], s_wsum[RB_NT / 32];

    const int t = threadIdx.x, tile = blockIdx.x;
    const int x0 = 8 * (tile % nt), y0 = 8 * ((tile / nt) % nt), z0 = 8 * (tile / (nt * nt));

    // source index of destination position pos (never past the particle count)
    auto source = [&](uint32_t pos) -> uint32_t {
        uint32_t s = inv[pos];
        if ((int64_t)s >= src.n) { atomicOr(err, ERR_BAD_CELL); s = 0; }
        return s;
    };

    auto sort_range = [&](uint32_t lo, int m) {
        for (int c = t; c < 512; c += RB_NT) s_cnt[c] = 0;
        __syncthreads();
        for (int j = t; j < m; j += RB_NT) {
            const uint32_t s = source(lo + (uint32_t)j);
            const uint32_t cell = src.cell[s];
            const int64_t id = src.id[s];
            double o[3];
            R q[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                o[k] = src.off[k * src.cap + s];
                q[k] = src.q[k * src.cap + s];
            }
            int cx, cy, cz;
            decode_cell(cell, fN, cx, cy, cz);
            int lx = cx - x0, ly = cy - y0, lz = cz - z0;
            if (lx < 0 || lx > 7 || ly < 0 || ly > 7 || lz < 0 || lz > 7) { atomicOr(err, ERR_BAD_CELL); lx = ly = lz = 0; }
            const int c = class_ord(lx, ly, lz);
            s_cell[j] = cell;
            s_id[j] = id;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                s_off[k * M + j] = o[k];
                s_q[k * M + j] = q[k];
            }
            s_ord[j] = (uint16_t)c;
            s_slot[j] = (uint16_t)atomicAdd(&s_cnt[c], 1);
        }
        __syncthreads();
        {   // exclusive scan of the 512 cell counts, one per thread
            const int v = s_cnt[t];
            int incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl, o);
                if ((t & 31) >= o) incl += u;
            }
            if ((t & 31) == 31) s_wsum[t >> 5] = incl;
            __syncthreads();
            if (t < 32) {
                const int w = t < RB_NT / 32 ? s_wsum[t] : 0;
                int wi = w;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, wi, o);
                    if (t >= o) wi += u;
                }
                if (t < RB_NT / 32) s_wsum[t] = wi - w;
            }
            __syncthreads();
            s_start[t] = incl - v + s_wsum[t >> 5];
        }
        __syncthreads();
        for (int j = t; j < m; j += RB_NT) s_order[s_start[s_ord[j]] + s_slot[j]] = (uint16_t)j;
        __syncthreads();
        {   // insertion sort by ID inside the cell (cells hold a few particles)
            const int k0 = s_start[t], mc = s_cnt[t];
            for (int a1 = 1; a1 < mc; a1++) {
                const uint16_t key = s_order[k0 + a1];
                const int64_t kid = s_id[key];
                int b1 = a1 - 1;
                while (b1 >= 0 && s_id[s_order[k0 + b1]] > kid) {
                    s_order[k0 + b1 + 1] = s_order[k0 + b1];
                    b1--;
                }
                s_order[k0 + b1 + 1] = key;
            }
        }
        __syncthreads();
        for (int k = t; k < m; k += RB_NT) {
            const int j = s_order[k];
            const uint32_t i = lo + (uint32_t)k;
            dst.cell[i] = s_cell[j];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                dst.off[c * dst.cap + i] = s_off[c * M + j];
                dst.q[c * dst.cap + i] = s_q[c * M + j];
            }
            dst.id[i] = s_id[j];
        }
        __syncthreads();
    };

    const uint32_t b0 = bstart[8 * tile], b8 = bstart[8 * tile + 8];
    if (b8 - b0 <= (uint32_t)M) {
        if (b8 > b0) sort_range(b0, (int)(b8 - b0));
        return;
    }
    for (int c = 0; c < 8; c++) {
        const uint32_t lo = bstart[8 * tile + c], hi = bstart[8 * tile + c + 1];
        if (hi - lo <= (uint32_t)M) {
            if (hi > lo) sort_range(lo, (int)(hi - lo));
        } else {
            for (uint32_t i = lo + (uint32_t)t; i < hi; i += RB_NT) {
                const uint32_t s = source(i);
                dst.cell[i] = src.cell[s];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    dst.off[k * dst.cap + i] = src.off[k * src.cap + s];
                    dst.q[k * dst.cap + i] = src.q[k * src.cap + s];
                }
                dst.id[i] = src.id[s];
            }
        }
    }
}

template <class R>
void launch_rebin(const PView<R> &src, PView<R> dst, const uint32_t *bstart, const uint32_t *bucket,
                  const uint32_t *rank, uint32_t *inv, int N, int *err, cudaStream_t st)
{
    if (src.n <= 0) return;
    k_scatter_index<<<cdiv(src.n, 256), 256, 0, st>>>(bstart, bucket, rank, src.n, inv);
    static bool attr_set[SMEM_ATTR_DEVICES] = {};
    raise_smem_limit(k_rebin_tile<R>, rb_smem_bytes<R>(), attr_set);
    const int nt = N / 8;
    k_rebin_tile<R><<<(unsigned)nt * nt * nt, RB_NT, rb_smem_bytes<R>(), st>>>(src, dst, bstart, inv, nt, err,
                                                                    FastDiv((uint32_t)N));
}

// CIC mass density in FP64 (scalarProjectionCIC_project, gevolution.hpp:1902,
// with LATfield2's meshprojection weights) from the FP64 positions, by
// atomic adds: the density a mixed-precision context measures its power
// spectrum on.  m = particle mass / dx^3.
template <class R>
__global__ void k_cic_f64(PView<R> p, int N, FastDiv fN, double m, double *__restrict__ rho)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < p.n; i += (int64_t)gridDim.x * blockDim.x) {
        int cx, cy, cz;
        decode_cell(p.cell[i], fN, cx, cy, cz);
        const double d[3] = {p.off[i], p.off[p.cap + i], p.off[2 * p.cap + i]};
        const int x1 = cx + 1 == N ? 0 : cx + 1, y1 = cy + 1 == N ? 0 : cy + 1, z1 = cz + 1 == N ? 0 : cz + 1;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const double w = ((k & 1) ? d[0] : 1.0 - d[0]) * ((k & 2) ? d[1] : 1.0 - d[1]) * ((k & 4) ? d[2] : 1.0 - d[2]);
            atomicAdd(rho + sidx(N, (k & 1) ? x1 : cx, (k & 2) ? y1 : cy, (k & 4) ? z1 : cz), m * w);
        }
    }
}

template <class R> void launch_cic_f64(const PView<R> &p, int N, double m, double *rho, cudaStream_t st)
{
    if (p.n <= 0) return;
    k_cic_f64<R><<<(unsigned)std::min<int64_t>(cdiv(p.n, 256), 148 * 16), 256, 0, st>>>(p, N, FastDiv((uint32_t)N), m, rho);
}

__global__ void k_f64_to_f32(const double *__restrict__ in, int64_t n, float *__restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

void launch_f64_to_f32(const double *in, int64_t n, float *out, cudaStream_t st)
{
    if (n > 0) k_f64_to_f32<<<(unsigned)std::min<int64_t>(cdiv(n, 256), 148 * 16), 256, 0, st>>>(in, n, out);
}

// deterministic sum of per-block partials (fixed order)
__global__ void k_reduce_sum(const double *partial, int64_t n, double *out)
{
    __shared__ double s[1024];
    double v = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += 1024) v += partial[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (threadIdx.x < (unsigned)o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

void launch_reduce_sum(const double *partial, int64_t n, double *out, cudaStream_t st)
{
    k_reduce_sum<<<1, 1024, 0, st>>>(partial, n, out);
}

#define GEV_INST(R)                                                                                                   \
    template void launch_kick_drift<R>(const PView<R> &, const uint32_t *, int, const R *, const R *, const R *,     \
                                       int64_t, const KickDriftParams &, uint32_t *, uint32_t *, uint32_t *,          \
                                       unsigned long long *, int *, cudaStream_t);                                    \
    template void launch_load_particles<R>(PView<R>, const double *, const double *, const int64_t *, int64_t, int,  \
                                           int *, cudaStream_t);                                                      \
    template void launch_store_particles<R>(const PView<R> &, double *, double *, int64_t *, int64_t, int,           \
                                            cudaStream_t);                                                            \
    template void launch_bin_count<R>(const PView<R> &, int, uint32_t *, uint32_t *, uint32_t *, cudaStream_t);       \
    template void launch_rebin<R>(const PView<R> &, PView<R>, const uint32_t *, const uint32_t *, const uint32_t *,   \
                                  uint32_t *, int, int *, cudaStream_t);                                              \
    template void launch_cic_f64<R>(const PView<R> &, int, double, double *, cudaStream_t);
GEV_INST(float)
GEV_INST(double)
#undef GEV_INST

}  // namespace gev
