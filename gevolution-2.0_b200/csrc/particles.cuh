// particles.cuh -- particle storage and tile bucketing shared by the deposit,
// kick/drift and lightcone kernels.
//
// Particles are structure-of-arrays, ordered by bucket = 8*tile + class (tiles
// of 8^3 cells; the class bits mark the tile's upper faces x,y,z == 7).  Inside
// every bucket of at most REBIN_SORT_MAX particles the order is (cell, particle
// ID), so the records of one cell are contiguous and the deposits sum them in a
// fixed order; larger buckets keep an arbitrary order and are only ever read by
// the deposits' fixed-point path, whose sums do not depend on it.
//   cell  : uint32 linear cell index x + N*(y + N*z)
//   off   : 3 planes of FP64 offsets inside the cell, in cell units, [0,1)
//   q     : 3 planes of momenta per unit mass (R = float in mixed mode)
//   id    : int64
#pragma once

#include "common.cuh"

namespace gev {

template <class R> struct PView {
    uint32_t *cell;
    double *off;    // 3 planes, stride cap
    R *q;           // 3 planes, stride cap
    int64_t *id;
    int64_t cap;
    int64_t n;
};

// buckets up to this many particles are kept in (cell, ID) order; at least the
// largest single-chunk deposit (1024 records)
constexpr int REBIN_SORT_MAX = 1024;

// Rank of the tile-local cell (lx, ly, lz) in class-major order: the cells of
// class 0 (343 of them), then class 1 (49), ..., class 7 (1), each class in
// (z, y, x) lexicographic order -- so sorting a tile by this rank sorts it by
// bucket and, inside every bucket, by cell index.
__host__ __device__ __forceinline__ int class_ord(int lx, int ly, int lz)
{
    const bool fx = lx == 7, fy = ly == 7, fz = lz == 7;
    const int cls = (fx ? 1 : 0) | (fy ? 2 : 0) | (fz ? 4 : 0);
    // first rank of each class: 0, 343, 343+49, ... (class sizes 343, 49, 49, 7, 49, 7, 7, 1)
    const int first = cls == 0 ? 0 : cls == 1 ? 343 : cls == 2 ? 392 : cls == 3 ? 441 : cls == 4 ? 448 : cls == 5 ? 497 : cls == 6 ? 504 : 511;
    int r = 0, mul = 1;
    if (!fx) { r += lx * mul; mul *= 7; }
    if (!fy) { r += ly * mul; mul *= 7; }
    if (!fz) r += lz * mul;
    return first + r;
}

// Particle ranges a tile's deposit needs: its own 8 class buckets and, from
// each of the 7 lower neighbour tiles, the classes whose cells lie on the
// shared faces.  Block-cooperative: thread k < 64 reads candidate k =
// (neighbour offset m = k >> 3, class c = k & 7), the range of that class in
// the neighbour tile when the class lies on the faces shared with this tile
// (c & m == m) and an empty range otherwise; warp 0 then forms the exclusive
// prefix sums of the 64 range lengths.  seg_lo/seg_hi hold 64 entries and
// seg_pre 65; the particle at position i of the concatenation is found with
// seg_find.  Contains __syncthreads(); every thread of the block must call it.
__device__ __forceinline__ void tile_segments_block(const uint32_t *bstart, int nt, int tx, int ty, int tz,
                                                    uint32_t *seg_lo, uint32_t *seg_hi, uint32_t *seg_pre)
{
    const int t = threadIdx.x;
    if (t < 64) {
        const int m = t >> 3, c = t & 7;
        uint32_t lo = 0, hi = 0;
        if ((c & m) == m) {
            const int dx = m & 1, dy = (m >> 1) & 1, dz = (m >> 2) & 1;
            const int nx = tx - dx < 0 ? nt - 1 : tx - dx;
            const int ny = ty - dy < 0 ? nt - 1 : ty - dy;
            const int nz = tz - dz < 0 ? nt - 1 : tz - dz;
            const uint32_t nb = (uint32_t)nx + (uint32_t)nt * ((uint32_t)ny + (uint32_t)nt * (uint32_t)nz);
            lo = bstart[8 * nb + c];
            hi = bstart[8 * nb + c + 1];
        }
        seg_lo[t] = lo;
        seg_hi[t] = hi > lo ? hi : lo;
    }
    __syncthreads();
    if (t < 32) {
        const uint32_t n0 = seg_hi[2 * t] - seg_lo[2 * t], n1 = seg_hi[2 * t + 1] - seg_lo[2 * t + 1];
        uint32_t s = n0 + n1, incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (t >= o) incl += u;
        }
        seg_pre[2 * t] = incl - s;
        seg_pre[2 * t + 1] = incl - s + n0;
        if (t == 31) seg_pre[64] = incl;
    }
    __syncthreads();
}

// position i (< seg_pre[64]) of the concatenated candidate ranges -> particle index
__device__ __forceinline__ uint32_t seg_find(const uint32_t *seg_lo, const uint32_t *seg_pre, uint32_t i)
{
    int lo = 0;
#pragma unroll
    for (int step = 32; step > 0; step >>= 1)
        if (seg_pre[lo + step] <= i) lo += step;
    return seg_lo[lo] + (i - seg_pre[lo]);
}

// As seg_find, with the tile's own 8 class buckets (candidates 0..7, one
// contiguous range that holds most of the tile's reach) resolved without the
// search.
__device__ __forceinline__ uint32_t seg_index(const uint32_t *seg_lo, const uint32_t *seg_pre, uint32_t i)
{
    if (i < seg_pre[8]) return seg_lo[0] + i;
    return seg_find(seg_lo, seg_pre, i);
}

// The per-particle words a kernel reads, loaded together so that the loads of
// several particles can be in flight at once.
template <class R> struct RawParticle {
    uint32_t cell;
    double off[3];
    R q[3];
};

template <class R> __device__ __forceinline__ RawParticle<R> load_particle(const PView<R> &p, int64_t i)
{
    RawParticle<R> r;
    r.cell = p.cell[i];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        r.off[k] = p.off[k * p.cap + i];
        r.q[k] = p.q[k * p.cap + i];
    }
    return r;
}

// relative coordinate of cell coordinate c to a tile origin o, in [-1, N-2]
__device__ __forceinline__ int rel_coord(int c, int o, int N)
{
    int r = c - o;
    if (r < -1) r += N;
    else if (r >= N - 1) r -= N;
    return r;
}

}  // namespace gev
