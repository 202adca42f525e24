// lightcone.cuh -- per-particle lightcone crossing shared by the lightcone
// kernel and the kick/drift kernel that runs it before the kick: the shell and
// cone test of count_tracer_particles / buffer_tracer_particles
// (Particles_gevolution.hpp:1271-1345, :1381-1466), the ID-backlog
// de-duplication of the check zone (count_lightcone_duplicate_ids /
// mark_lightcone_kept_particles, :1468-1510), the interpolation to the
// crossing time (bufferTracerParticle with EXACT_OUTPUT_REDSHIFTS, :500-560)
// and the logging of IDs near the inner edge for the next cycle.
//
// The ID logs are open-addressing hash sets in device memory (keys are particle
// IDs, EMPTY marks a free slot): membership is a set property, so the result
// does not depend on insertion order.
#pragma once

#include "common.cuh"
#include "kernels.h"
#include "particles.cuh"

namespace gev {

constexpr double LC_IDCHECK_ZONE = 0.05;            // metadata.hpp:38-40
constexpr double LC_GADGET_VEL = 3.335640952e-6;    // GADGET_VELOCITY_CONVERSION, metadata.hpp

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    // splitmix64 finaliser
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27; x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

__device__ __forceinline__ bool idset_contains(const unsigned long long *tab, int64_t cap, int64_t id)
{
    if (cap <= 0) return false;
    uint64_t h = mix64((uint64_t)id) & (uint64_t)(cap - 1);
    const int64_t maxp = cap < LC_MAX_PROBES ? cap : LC_MAX_PROBES;
    for (int64_t probe = 0; probe < maxp; probe++) {
        unsigned long long k = tab[h];
        if (k == (unsigned long long)id) return true;
        if (k == LC_EMPTY) return false;
        h = (h + 1) & (uint64_t)(cap - 1);
    }
    return false;
}

// returns false when the table is full
__device__ __forceinline__ bool idset_insert(unsigned long long *tab, int64_t cap, int64_t id)
{
    uint64_t h = mix64((uint64_t)id) & (uint64_t)(cap - 1);
    const int64_t maxp = cap < LC_MAX_PROBES ? cap : LC_MAX_PROBES;
    for (int64_t probe = 0; probe < maxp; probe++) {
        unsigned long long prev = atomicCAS(&tab[h], LC_EMPTY, (unsigned long long)id);
        if (prev == LC_EMPTY || prev == (unsigned long long)id) return true;
        h = (h + 1) & (uint64_t)(cap - 1);
    }
    return false;
}

template <class R>
__device__ __forceinline__ double gphi(const R *phi, int N, int x, int y, int z)
{
    return (double)phi[sidx(N, wrapi(x, N), wrapi(y, N), wrapi(z, N))];
}

// the reference's exact test and output for one particle, starting at kept image kv
template <class R>
__device__ __forceinline__ void lc_particle(const PView<R> &p, int64_t i, int N, const int c[3], const double fr[3],
                                            const R *__restrict__ phi, const LcKernelArgs &la, const int *vlist,
                                            int kv, int nkeep, float *opos, float *ovel, int64_t *oid,
                                            unsigned long long *count, unsigned long long *newlog,
                                            int64_t newlog_cap, int *err)
{
    const int64_t id = p.id[i];
    const double x[3] = {(c[0] + fr[0]) / N, (c[1] + fr[1]) / N, (c[2] + fr[2]) / N};
    const double q[3] = {(double)p.q[i], (double)p.q[p.cap + i], (double)p.q[2 * p.cap + i]};

    for (; kv < nkeep; kv++) {
        const double *V = la.vtx[vlist[kv]];
        double r[3] = {x[0] - V[0], x[1] - V[1], x[2] - V[2]};
        double d = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        if (!(d >= la.inner && d < la.outer)) continue;
        if (!(la.opening == -1. || (r[0] * la.direction[0] + r[1] * la.direction[1] + r[2] * la.direction[2]) / d > la.opening)) continue;

        // check zone near the outer edge: drop IDs written in the previous cycle
        if (la.outer - d <= 2. * LC_IDCHECK_ZONE * la.dtau_old && idset_contains(la.backlog, la.backlog_cap, id)) return;

        double vlos = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + la.a * (la.a + la.dtau_old * la.dadtau));
        vlos = (q[0] * r[0] + q[1] * r[1] + q[2] * r[2]) / d / vlos;
        const double dtau_pos = (la.dist - d) / (1. + vlos);
        const double dtau_vel = dtau_pos + 0.5 * la.dtau_old;
        const double at = la.a + dtau_pos * la.dadtau;

        // bufferTracerParticle (EXACT_OUTPUT_REDSHIFTS)
        double phip = 0., g[3] = {0., 0., 0.};
        if (phi) {
            double w[8], P[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                w[k] = (((k >> 2) & 1) ? fr[0] : 1. - fr[0]) * (((k >> 1) & 1) ? fr[1] : 1. - fr[1]) * ((k & 1) ? fr[2] : 1. - fr[2]);
                P[k] = gphi(phi, N, c[0] + ((k >> 2) & 1), c[1] + ((k >> 1) & 1), c[2] + (k & 1));   // P[4bx+2by+bz]
                phip += w[k] * P[k];
            }
            g[0] = (1 - fr[1]) * (1 - fr[2]) * (P[4] - P[0]) + fr[1] * (1 - fr[2]) * (P[6] - P[2]) + (1 - fr[1]) * fr[2] * (P[5] - P[1]) + fr[1] * fr[2] * (P[7] - P[3]);
            g[1] = (1 - fr[0]) * (1 - fr[2]) * (P[2] - P[0]) + fr[0] * (1 - fr[2]) * (P[6] - P[4]) + (1 - fr[0]) * fr[2] * (P[3] - P[1]) + fr[0] * fr[2] * (P[7] - P[5]);
            g[2] = (1 - fr[0]) * (1 - fr[1]) * (P[1] - P[0]) + fr[0] * (1 - fr[1]) * (P[5] - P[4]) + (1 - fr[0]) * fr[1] * (P[3] - P[2]) + fr[0] * fr[1] * (P[7] - P[6]);
        }
        double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        double f1 = q2 + at * at, f2 = sqrt(f1), f0 = q2 + f1;
        f1 = 1. + (4. - f0 / f1) * phip;
        const double rescale_vel = 1. / sqrt(at) / LC_GADGET_VEL;

        unsigned long long slot = atomicAdd(count, 1ull);
        if (slot < (unsigned long long)la.capacity) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                float pos_offset = (float)(la.lc_vertex[k] - V[k]);
                opos[3 * slot + k] = ((float)(x[k] + dtau_pos * q[k] * f1 / f2) + pos_offset) * (float)la.boxsize;
                ovel[3 * slot + k] = (float)((q[k] - dtau_vel * f0 * g[k] * (double)N / f2) * rescale_vel) / (float)at;
            }
            oid[slot] = id;
        }
        if (d - la.inner < 2. * LC_IDCHECK_ZONE * la.dtau) {
            if (!idset_insert(newlog, newlog_cap, id)) atomicOr(err, ERR_LC_OVERFLOW);
        }
        return;
    }
}

// Block-cooperative: the periodic images of the vertex whose shell [inner,
// outer) can reach the bounding box of tile (tx, ty, tz), in vertex order (so
// the first image a particle matches is the same as in a test against all of
// them).  Threads 0..63 test one image each and write the ballots to vmask[2];
// after the caller's barrier, lc_compact_images lists the kept ones.
__device__ __forceinline__ void lc_cull_images(const LcKernelArgs &la, int N, int tx, int ty, int tz, unsigned int *vmask)
{
    if (threadIdx.x < 64) {
        bool hit = false;
        const int v = threadIdx.x;
        if (v < la.nvtx) {
            const double lo[3] = {tx * 8.0 / N, ty * 8.0 / N, tz * 8.0 / N};
            double dmin2 = 0.0, dmax2 = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double V = la.vtx[v][k], h = lo[k] + 8.0 / N;
                const double c = V < lo[k] ? lo[k] : (V > h ? h : V);
                dmin2 += (c - V) * (c - V);
                const double f = fmax(fabs(V - lo[k]), fabs(V - h));
                dmax2 += f * f;
            }
            hit = sqrt(dmax2) + 1e-9 >= la.inner && sqrt(dmin2) - 1e-9 < la.outer;
        }
        const unsigned int m = __ballot_sync(0xffffffffu, hit);
        if ((threadIdx.x & 31) == 0) vmask[threadIdx.x >> 5] = m;
    }
}

// the kept images' indexes into vlist (threads 0..63; vmask visible to all)
__device__ __forceinline__ int lc_compact_images(const unsigned int *vmask, int *vlist)
{
    const unsigned int m0 = vmask[0], m1 = vmask[1];
    if (threadIdx.x < 64) {
        const int v = threadIdx.x;
        const unsigned int mine = v < 32 ? m0 : m1;
        if ((mine >> (v & 31)) & 1u) {
            const unsigned int below = (v & 31) ? (mine & ((1u << (v & 31)) - 1u)) : 0u;
            vlist[(v < 32 ? 0 : __popc(m0)) + __popc(below)] = v;
        }
    }
    return __popc(m0) + __popc(m1);
}

// FP32 radius pre-test against the kept images (margins far above the FP32
// rounding of |x - V|^2 for |x - V| < 4 box lengths); the exact FP64 test and
// the output only for a particle near the shell.  c, fr: the particle's cell
// and FP64 in-cell offset before this cycle's kick.
struct LcShell {
    float invN, in2, out2;
    __device__ __forceinline__ LcShell(const LcKernelArgs &la, int N)
    {
        invN = 1.0f / (float)N;
        in2 = (float)(la.inner * la.inner) * (1.0f - 1e-4f) - 1e-5f;
        out2 = (float)(la.outer * la.outer) * (1.0f + 1e-4f) + 1e-5f;
    }
};

template <class R>
__device__ __forceinline__ void lc_visit(const PView<R> &p, int64_t i, int N, const int c[3], const double fr[3],
                                         const R *__restrict__ phi, const LcKernelArgs &la, const LcShell &sh,
                                         const int *vlist, int nkeep, float *opos, float *ovel, int64_t *oid,
                                         unsigned long long *count, unsigned long long *newlog, int64_t newlog_cap,
                                         int *err)
{
    const float xf[3] = {((float)c[0] + (float)fr[0]) * sh.invN, ((float)c[1] + (float)fr[1]) * sh.invN,
                         ((float)c[2] + (float)fr[2]) * sh.invN};
    int kv = 0;
    for (; kv < nkeep; kv++) {
        const int v = vlist[kv];
        const float r0 = xf[0] - (float)la.vtx[v][0], r1 = xf[1] - (float)la.vtx[v][1], r2 = xf[2] - (float)la.vtx[v][2];
        const float d2 = r0 * r0 + r1 * r1 + r2 * r2;
        if (d2 >= sh.in2 && d2 < sh.out2) break;
    }
    if (kv == nkeep) return;
    if (la.tracer_factor > 1 && p.id[i] % la.tracer_factor != 0) return;
    lc_particle(p, i, N, c, fr, phi, la, vlist, kv, nkeep, opos, ovel, oid, count, newlog, newlog_cap, err);
}

}  // namespace gev
