// deposit.cu -- deterministic tile deposits of T00, Tij and T0i.
//
// One CTA owns the 8^3 vertices of a tile and gathers every particle whose CIC
// stencil touches them: its own 8 class buckets plus the face-class buckets of
// the 7 lower neighbour tiles (tile_segments).  Contributions are accumulated
// in shared memory as 64-bit fixed point with a per-CTA, per-component scale
// chosen from the exact maximum contribution (first pass) and the particle
// count, so the sum is exact integer arithmetic: the result does not depend on
// particle order or thread scheduling (bitwise reproducible), and each output
// vertex is written exactly once with plain stores -- no global atomics and no
// halo fold (projection_comm1, gevolution.hpp:1543, is not needed on one GPU).
//
// Arithmetic follows the reference functors term by term, in FP64:
//   particle_T00_project  gevolution.hpp:1729-1854
//   particle_Tij_project  gevolution.hpp:2582-2965 (non-CIC_PROJECT_TIJ)
//   particle_T0i_project  gevolution.hpp:2031-2201
#include "common.cuh"
#include "particles.cuh"
#include "kernels.h"

namespace gev {

constexpr int DEP_NT = 256;

// φ staged over the vertex region [-1, 8] of the tile (10^3)
template <class R>
__device__ __forceinline__ double phs(const R *s, int vx, int vy, int vz)
{
    return (double)s[(vx + 1) + 10 * ((vy + 1) + 10 * (vz + 1))];
}

// Visit every contribution of one particle: f(component, vx, vy, vz, value),
// vertex coordinates relative to the tile origin.
template <class R, int KIND, bool USE_PHI, class F>
__device__ __forceinline__ void particle_contribs(const PView<R> &p, uint32_t i, int N, int x0, int y0, int z0,
                                                  const R *phis, double a, double m00, double mij, F &&f)
{
    uint32_t cell = p.cell[i];
    int cx = (int)(cell % (uint32_t)N), cy = (int)((cell / (uint32_t)N) % (uint32_t)N), cz = (int)(cell / ((uint32_t)N * (uint32_t)N));
    int rx = rel_coord(cx, x0, N), ry = rel_coord(cy, y0, N), rz = rel_coord(cz, z0, N);
    // a particle outside the tile's reach means the bucket order is stale: skip it
    // (the staged phi region covers vertices -1..8 only)
    if (rx < -1 || rx > 7 || ry < -1 || ry > 7 || rz < -1 || rz > 7) return;
    double d[3] = {p.off[i], p.off[p.cap + i], p.off[2 * p.cap + i]};
    double q[3] = {(double)p.q[i], (double)p.q[p.cap + i], (double)p.q[2 * p.cap + i]};
    double ph[8];
    if (USE_PHI) {
#pragma unroll
        for (int k = 0; k < 8; k++) ph[k] = phs(phis, rx + ((k >> 2) & 1), ry + ((k >> 1) & 1), rz + (k & 1));
    }
    double w8[8];
#pragma unroll
    for (int k = 0; k < 8; k++)
        w8[k] = (((k >> 2) & 1) ? d[0] : 1.0 - d[0]) * (((k >> 1) & 1) ? d[1] : 1.0 - d[1]) * ((k & 1) ? d[2] : 1.0 - d[2]);

    if constexpr (KIND == DEP_T00 || KIND == DEP_T00_TIJ) {
        // T00 -> component 0
        if (USE_PHI) {
            double f2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
            double e = sqrt(f2 + a * a);
            double fc = 3.0 * e + f2 / e;
            f2 = (0.5 * fc * fc + f2 / (1.0 + f2 / a / a)) / e;
#pragma unroll
            for (int k = 0; k < 8; k++)
                f(0, rx + ((k >> 2) & 1), ry + ((k >> 1) & 1), rz + (k & 1), w8[k] * (e + fc * ph[k] + f2 * ph[k] * ph[k]) * m00);
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++) f(0, rx + ((k >> 2) & 1), ry + ((k >> 1) & 1), rz + (k & 1), w8[k] * m00);
        }
    }
    if constexpr (KIND == DEP_TIJ || KIND == DEP_T00_TIJ) {
        constexpr int C0 = (KIND == DEP_T00_TIJ) ? 1 : 0;   // first Tij component slot
        double qq = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        double e = sqrt(qq + a * a);
        double fac = 1.0;
        if (USE_PHI) {
            double pint = 0.0;
#pragma unroll
            for (int k = 0; k < 8; k++) pint += w8[k] * ph[k];
            fac = 1.0 + (4.0 + a * a / (qq + a * a)) * pint;
        }
        const int dslot[3] = {0, 3, 5};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double W = fac * mij * q[c] * q[c] / e;
#pragma unroll
            for (int k = 0; k < 8; k++) f(C0 + dslot[c], rx + ((k >> 2) & 1), ry + ((k >> 1) & 1), rz + (k & 1), W * w8[k]);
        }
        double W;
        W = fac * mij * q[0] * q[1] / e;   // (0,1): x and x+e2
        f(C0 + 1, rx, ry, rz, W * (1.0 - d[2]));
        f(C0 + 1, rx, ry, rz + 1, W * d[2]);
        W = fac * mij * q[0] * q[2] / e;   // (0,2): x and x+e1
        f(C0 + 2, rx, ry, rz, W * (1.0 - d[1]));
        f(C0 + 2, rx, ry + 1, rz, W * d[1]);
        W = fac * mij * q[1] * q[2] / e;   // (1,2): x and x+e0
        f(C0 + 4, rx, ry, rz, W * (1.0 - d[0]));
        f(C0 + 4, rx + 1, ry, rz, W * d[0]);
    }
    if constexpr (KIND == DEP_T0I) {
        double p_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (USE_PHI) {
#pragma unroll
            for (int k = 0; k < 8; k++) p_[k] = ph[k];
        }
        const double m = m00;
        f(0, rx, ry, rz, (1 - d[1]) * (1 - d[2]) * (1 + p_[0] + p_[4]) * m * q[0]);
        f(1, rx, ry, rz, (1 - d[0]) * (1 - d[2]) * (1 + p_[0] + p_[2]) * m * q[1]);
        f(2, rx, ry, rz, (1 - d[0]) * (1 - d[1]) * (1 + p_[0] + p_[1]) * m * q[2]);
        f(1, rx + 1, ry, rz, d[0] * (1 - d[2]) * (1 + p_[4] + p_[6]) * m * q[1]);
        f(2, rx + 1, ry, rz, d[0] * (1 - d[1]) * (1 + p_[4] + p_[5]) * m * q[2]);
        f(0, rx, ry + 1, rz, d[1] * (1 - d[2]) * (1 + p_[2] + p_[6]) * m * q[0]);
        f(2, rx, ry + 1, rz, d[1] * (1 - d[0]) * (1 + p_[2] + p_[3]) * m * q[2]);
        f(0, rx, ry, rz + 1, d[2] * (1 - d[1]) * (1 + p_[1] + p_[5]) * m * q[0]);
        f(1, rx, ry, rz + 1, d[2] * (1 - d[0]) * (1 + p_[1] + p_[3]) * m * q[1]);
        f(0, rx, ry + 1, rz + 1, d[1] * d[2] * (1 + p_[3] + p_[7]) * m * q[0]);
        f(1, rx + 1, ry, rz + 1, d[0] * d[2] * (1 + p_[5] + p_[7]) * m * q[1]);
        f(2, rx + 1, ry + 1, rz, d[0] * d[1] * (1 + p_[6] + p_[7]) * m * q[2]);
    }
}

template <int KIND> struct DepShape {
    static constexpr int NC = (KIND == DEP_T00) ? 1 : (KIND == DEP_TIJ ? 6 : (KIND == DEP_T00_TIJ ? 7 : 3));
};

// outputs: component c is written to out[c] (N^3 plane each)
template <class R, int KIND, bool USE_PHI>
__global__ void __launch_bounds__(DEP_NT) k_deposit(PView<R> p, const uint32_t *__restrict__ bstart, int N, int nt,
                                                    const R *__restrict__ phi, DepOut<R> out, double a, double m00,
                                                    double mij, int accumulate)
{
    constexpr int NC = DepShape<KIND>::NC;
    __shared__ unsigned long long acc[NC][512];
    __shared__ R phis[USE_PHI ? 1000 : 1];
    __shared__ uint32_t seg_lo[20], seg_hi[20], seg_pre[21];
    __shared__ int nseg;
    __shared__ unsigned long long vmax[NC];
    __shared__ double scl[NC], iscl[NC];

    const int tile = blockIdx.x;
    const int tx = tile % nt, ty = (tile / nt) % nt, tz = tile / (nt * nt);
    const int x0 = tx * 8, y0 = ty * 8, z0 = tz * 8;

    if (threadIdx.x == 0) {
        int ns = tile_segments(bstart, nt, tx, ty, tz, seg_lo, seg_hi);
        seg_pre[0] = 0;
        for (int s = 0; s < ns; s++) seg_pre[s + 1] = seg_pre[s] + (seg_hi[s] - seg_lo[s]);
        nseg = ns;
    }
    for (int i = threadIdx.x; i < NC * 512; i += DEP_NT) (&acc[0][0])[i] = 0ull;
    if (threadIdx.x < NC) vmax[threadIdx.x] = 0ull;
    if (USE_PHI) {
        for (int i = threadIdx.x; i < 1000; i += DEP_NT) {
            int vx = i % 10 - 1, vy = (i / 10) % 10 - 1, vz = i / 100 - 1;
            phis[i] = phi[sidx(N, wrapi(x0 + vx, N), wrapi(y0 + vy, N), wrapi(z0 + vz, N))];
        }
    }
    __syncthreads();
    const int ns = nseg;
    const uint32_t total = seg_pre[ns];

    // pass 1: exact maximum |contribution| per component
    {
        double lm[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) lm[c] = 0.0;
        for (uint32_t j = threadIdx.x; j < total; j += DEP_NT) {
            uint32_t i = seg_map(ns, seg_lo, seg_pre, j);
            particle_contribs<R, KIND, USE_PHI>(p, i, N, x0, y0, z0, phis, a, m00, mij,
                                                [&](int c, int vx, int vy, int vz, double v) {
                                                    if ((unsigned)vx < 8u && (unsigned)vy < 8u && (unsigned)vz < 8u) lm[c] = fmax(lm[c], fabs(v));
                                                });
        }
#pragma unroll
        for (int c = 0; c < NC; c++) {
            double m = lm[c];
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(&vmax[c], (unsigned long long)__double_as_longlong(m));
        }
    }
    __syncthreads();
    if (threadIdx.x < NC) {
        double m = __longlong_as_double((long long)vmax[threadIdx.x]);
        int e = 0;
        if (m > 0.0 && total > 0) {
            int ex;
            frexp(m * (double)total, &ex);
            e = 61 - ex;
            e = e > 1000 ? 1000 : (e < -1000 ? -1000 : e);
        }
        scl[threadIdx.x] = ldexp(1.0, e);
        iscl[threadIdx.x] = ldexp(1.0, -e);
    }
    __syncthreads();

    // pass 2: fixed-point accumulation
    for (uint32_t j = threadIdx.x; j < total; j += DEP_NT) {
        uint32_t i = seg_map(ns, seg_lo, seg_pre, j);
        particle_contribs<R, KIND, USE_PHI>(p, i, N, x0, y0, z0, phis, a, m00, mij,
                                            [&](int c, int vx, int vy, int vz, double v) {
                                                if ((unsigned)vx < 8u && (unsigned)vy < 8u && (unsigned)vz < 8u) {
                                                    long long fx = __double2ll_rn(v * scl[c]);
                                                    atomicAdd(&acc[c][vx + 8 * (vy + 8 * vz)], (unsigned long long)fx);
                                                }
                                            });
    }
    __syncthreads();

    for (int i = threadIdx.x; i < NC * 512; i += DEP_NT) {
        int c = i >> 9, v = i & 511;
        int vx = v & 7, vy = (v >> 3) & 7, vz = v >> 6;
        double val = (double)(long long)acc[c][v] * iscl[c];
        int64_t gi = sidx(N, x0 + vx, y0 + vy, z0 + vz);
        R *o = out.p[c];
        if (accumulate) o[gi] = (R)((double)o[gi] + val);
        else o[gi] = (R)val;
    }
}

template <class R>
void launch_deposit(int kind, bool use_phi, const PView<R> &p, const uint32_t *bstart, int N, const R *phi,
                    const DepOut<R> &out, double a, double m00, double mij, int accumulate, cudaStream_t st)
{
    int nt = N / 8;
    unsigned grid = (unsigned)nt * nt * nt;
#define GEV_DEP(K)                                                                                               \
    if (kind == K) {                                                                                             \
        if (use_phi) k_deposit<R, K, true><<<grid, DEP_NT, 0, st>>>(p, bstart, N, nt, phi, out, a, m00, mij, accumulate); \
        else k_deposit<R, K, false><<<grid, DEP_NT, 0, st>>>(p, bstart, N, nt, phi, out, a, m00, mij, accumulate); \
        return;                                                                                                  \
    }
    GEV_DEP(DEP_T00)
    GEV_DEP(DEP_TIJ)
    GEV_DEP(DEP_T00_TIJ)
    GEV_DEP(DEP_T0I)
#undef GEV_DEP
}

template void launch_deposit<float>(int, bool, const PView<float> &, const uint32_t *, int, const float *,
                                    const DepOut<float> &, double, double, double, int, cudaStream_t);
template void launch_deposit<double>(int, bool, const PView<double> &, const uint32_t *, int, const double *,
                                     const DepOut<double> &, double, double, double, int, cudaStream_t);

}  // namespace gev
