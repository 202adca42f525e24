// ics.cu -- kernels of the Zel'dovich initial-condition generator
// (gev_ics_zeldovich): the Gaussian white-noise field, the displaced lattice,
// and the linear-theory momenta.
//
// The white noise is a counter-based stream: cell i draws Philox4x32-10
// (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011) with counter (i, 0, 0, 0) and key (seed_lo, seed_hi), and turns
// the first two words into one standard normal by the Box-Muller transform.
// The field therefore depends on the seed and the grid only, not on the launch
// shape.  (The reference draws from the sitmo engine, ic_basic.hpp:1175,
// whose stream is not reproduced here: the statistics are the same, the
// realisation differs.)
#include "common.cuh"
#include "kernels.h"
#include "particles.cuh"

namespace gev {

__host__ __device__ inline void philox4x32_10(uint32_t ctr[4], uint32_t key0, uint32_t key1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++) {
        if (r > 0) { key0 += W0; key1 += W1; }
        const uint64_t p0 = (uint64_t)M0 * ctr[0], p1 = (uint64_t)M1 * ctr[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t c0 = hi1 ^ ctr[1] ^ key0, c2 = hi0 ^ ctr[3] ^ key1;
        ctr[0] = c0; ctr[1] = lo1; ctr[2] = c2; ctr[3] = lo0;
    }
}

template <class R>
__global__ void k_ics_noise(R *out, int64_t n3, uint64_t seed)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n3) return;
    uint32_t c[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u1 = ((double)c[0] + 0.5) * (1.0 / 4294967296.0);   // (0, 1)
    const double u2 = (double)c[1] * (1.0 / 4294967296.0);           // [0, 1)
    out[i] = (R)(sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
}

// One particle per cell at the cell centre (i + 1/2)/N displaced by the
// displacement field at vertex i (box units), momentum zero, ID = cell index.
template <class R>
__global__ void k_ics_lattice(PView<R> p, const R *__restrict__ psi, int N)
{
    const int64_t n3 = (int64_t)N * N * N;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const int c0[3] = {(int)(i % N), (int)((i / N) % N), (int)(i / ((int64_t)N * N))};
    int c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double x = ((double)c0[k] + 0.5) / N + (double)psi[k * n3 + i];
        x -= floor(x);
        const double s = x * N, f = floor(s);
        double o = s - f;
        int ci = (int)f;
        if (ci >= N) { ci = N - 1; o = 1.0 - 1e-16; }
        if (ci < 0) { ci = 0; o = 0.0; }
        c[k] = ci;
        p.off[k * p.cap + i] = o;
        p.q[k * p.cap + i] = (R)0;
    }
    p.cell[i] = (uint32_t)sidx(N, c[0], c[1], c[2]);
    p.id[i] = i;
}

template <class R>
__device__ __forceinline__ double ics_phi(const R *phi, int N, int x, int y, int z)
{
    return (double)phi[sidx(N, wrapi(x, N), wrapi(y, N), wrapi(z, N))];
}

// initialize_q_ic_basic (ic_basic.hpp:133-166) with one field: q = -coeff grad phi,
// the gradient from the cell's edge differences with bilinear weights, / dx
template <class R>
__global__ void k_ics_velocity(PView<R> p, const R *__restrict__ phi, int N, double coeff, FastDiv fN)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    int cx, cy, cz;
    decode_cell(p.cell[i], fN, cx, cy, cz);
    const double d[3] = {p.off[i], p.off[p.cap + i], p.off[2 * p.cap + i]};
    auto F = [&](int dx, int dy, int dz) { return ics_phi(phi, N, cx + dx, cy + dy, cz + dz); };
    double g[3];
    g[0] = (1. - d[1]) * (1. - d[2]) * (F(1, 0, 0) - F(0, 0, 0));
    g[1] = (1. - d[0]) * (1. - d[2]) * (F(0, 1, 0) - F(0, 0, 0));
    g[2] = (1. - d[0]) * (1. - d[1]) * (F(0, 0, 1) - F(0, 0, 0));
    g[0] += d[1] * (1. - d[2]) * (F(1, 1, 0) - F(0, 1, 0));
    g[1] += d[0] * (1. - d[2]) * (F(1, 1, 0) - F(1, 0, 0));
    g[2] += d[0] * (1. - d[1]) * (F(1, 0, 1) - F(1, 0, 0));
    g[0] += (1. - d[1]) * d[2] * (F(1, 0, 1) - F(0, 0, 1));
    g[1] += (1. - d[0]) * d[2] * (F(0, 1, 1) - F(0, 0, 1));
    g[2] += (1. - d[0]) * d[1] * (F(0, 1, 1) - F(0, 1, 0));
    g[0] += d[1] * d[2] * (F(1, 1, 1) - F(0, 1, 1));
    g[1] += d[0] * d[2] * (F(1, 1, 1) - F(1, 0, 1));
    g[2] += d[0] * d[1] * (F(1, 1, 1) - F(1, 1, 0));
#pragma unroll
    for (int k = 0; k < 3; k++) p.q[k * p.cap + i] = (R)(-g[k] * (double)N * coeff);
}

template <class R> void launch_ics_noise(R *out, int64_t n3, uint64_t seed, cudaStream_t st)
{
    k_ics_noise<R><<<cdiv(n3, 256), 256, 0, st>>>(out, n3, seed);
}
template <class R> void launch_ics_lattice(PView<R> p, const R *psi, int N, cudaStream_t st)
{
    k_ics_lattice<R><<<cdiv((int64_t)N * N * N, 256), 256, 0, st>>>(p, psi, N);
}
template <class R> void launch_ics_velocity(const PView<R> &p, const R *phi, int N, double coeff, cudaStream_t st)
{
    if (p.n > 0) k_ics_velocity<R><<<cdiv(p.n, 256), 256, 0, st>>>(p, phi, N, coeff, FastDiv((uint32_t)N));
}

#define GEV_ICS_INST(R)                                                                              \
    template void launch_ics_noise<R>(R *, int64_t, uint64_t, cudaStream_t);                         \
    template void launch_ics_lattice<R>(PView<R>, const R *, int, cudaStream_t);                     \
    template void launch_ics_velocity<R>(const PView<R> &, const R *, int, double, cudaStream_t);
GEV_ICS_INST(float)
GEV_ICS_INST(double)
#undef GEV_ICS_INST

}  // namespace gev
