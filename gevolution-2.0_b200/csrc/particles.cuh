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
// shared faces.  Candidate k = (neighbour offset m = k >> 3, class c = k & 7)
// is the range of that class in the neighbour tile when the class lies on the
// faces shared with this tile (c & m == m) and an empty range otherwise; pre
// holds the exclusive prefix sums of the 64 range lengths.  Formed by one
// warp in registers (lane l holds candidates l and l + 32) with no block
// barrier; tile_segments_store copies them to shared memory (seg_lo, seg_hi:
// 64 entries, seg_pre: 65) for seg_find and seg_index.
struct TileSegs {
    uint32_t lo[2], hi[2], pre[2];   // candidates l and l + 32 of lane l
    uint32_t total;                  // length of the concatenation
};

__device__ __forceinline__ TileSegs tile_segments_warp(const uint32_t *bstart, int nt, int tx, int ty, int tz)
{
    const int l = threadIdx.x & 31;
    TileSegs s;
    uint32_t len[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int k = l + 32 * h, m = k >> 3, c = k & 7;
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
        hi = hi > lo ? hi : lo;
        s.lo[h] = lo;
        s.hi[h] = hi;
        len[h] = hi - lo;
    }
    uint32_t inc0 = len[0], inc1 = len[1];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u0 = __shfl_up_sync(0xffffffffu, inc0, o);
        const uint32_t u1 = __shfl_up_sync(0xffffffffu, inc1, o);
        if (l >= o) { inc0 += u0; inc1 += u1; }
    }
    const uint32_t tot0 = __shfl_sync(0xffffffffu, inc0, 31);
    s.pre[0] = inc0 - len[0];
    s.pre[1] = tot0 + inc1 - len[1];
    s.total = __shfl_sync(0xffffffffu, tot0 + inc1, 31);
    return s;
}

// one warp's segments to shared memory (the caller's next __syncthreads()
// publishes them to the block)
__device__ __forceinline__ void tile_segments_store(const TileSegs &s, uint32_t *seg_lo, uint32_t *seg_hi,
                                                    uint32_t *seg_pre)
{
    const int l = threadIdx.x & 31;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        seg_lo[l + 32 * h] = s.lo[h];
        seg_hi[l + 32 * h] = s.hi[h];
        seg_pre[l + 32 * h] = s.pre[h];
    }
    if (l == 31) seg_pre[64] = s.total;
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
