// particles.cuh -- particle storage and tile bucketing shared by the deposit,
// kick/drift and lightcone kernels.
//
// Particles are structure-of-arrays, ordered by bucket = 8*tile + class (tiles
// of 8^3 cells; the class bits mark the tile's upper faces x,y,z == 7).  Order
// inside a bucket is not significant: every consumer is order-independent
// (fixed-point deposits, per-particle updates, max reductions).
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

struct Buckets {
    const uint32_t *start;   // nb + 1 entries (exclusive scan of counts)
};

// Gather the particle ranges a tile's deposit needs: its own 8 class buckets
// (one contiguous range) and, from each of the 7 lower neighbour tiles, the
// classes whose cells lie on the shared faces.  Ranges are written to
// seg_lo/seg_hi; returns their number (at most 20).
__device__ __forceinline__ int tile_segments(const uint32_t *bstart, int nt, int tx, int ty, int tz,
                                             uint32_t *seg_lo, uint32_t *seg_hi)
{
    int ns = 0;
    uint32_t tile = (uint32_t)tx + (uint32_t)nt * ((uint32_t)ty + (uint32_t)nt * (uint32_t)tz);
    seg_lo[ns] = bstart[8 * tile];
    seg_hi[ns] = bstart[8 * tile + 8];
    if (seg_hi[ns] > seg_lo[ns]) ns++;
    for (int m = 1; m < 8; m++) {
        int dx = m & 1, dy = (m >> 1) & 1, dz = (m >> 2) & 1;
        int nx = tx - dx < 0 ? nt - 1 : tx - dx;
        int ny = ty - dy < 0 ? nt - 1 : ty - dy;
        int nz = tz - dz < 0 ? nt - 1 : tz - dz;
        uint32_t nb = (uint32_t)nx + (uint32_t)nt * ((uint32_t)ny + (uint32_t)nt * (uint32_t)nz);
        for (int c = 0; c < 8; c++) {
            if ((c & m) != m) continue;
            uint32_t lo = bstart[8 * nb + c], hi = bstart[8 * nb + c + 1];
            if (hi <= lo) continue;
            if (ns > 0 && seg_hi[ns - 1] == lo) seg_hi[ns - 1] = hi;   // merge adjacent classes
            else { seg_lo[ns] = lo; seg_hi[ns] = hi; ns++; }
        }
    }
    return ns;
}

// Block-cooperative form of tile_segments: 64 threads read the 64 candidate
// (neighbour, class) bucket ranges in parallel, thread 0 merges the non-empty
// ones (in the same order) and builds the prefix sums.  Arrays hold 64 (+1)
// entries.  Contains a __syncthreads(); every thread of the block must call it.
__device__ __forceinline__ void tile_segments_block(const uint32_t *bstart, int nt, int tx, int ty, int tz,
                                                    uint32_t *cand_lo, uint32_t *cand_hi, uint32_t *seg_lo,
                                                    uint32_t *seg_hi, uint32_t *seg_pre, int *nseg)
{
    const int t = threadIdx.x;
    if (t < 64) {
        const int m = t >> 3, c = t & 7;   // neighbour offset bits, class
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
        cand_lo[t] = lo;
        cand_hi[t] = hi;
    }
    __syncthreads();
    if (t == 0) {
        int ns = 0;
        for (int k = 0; k < 64; k++) {
            const uint32_t lo = cand_lo[k], hi = cand_hi[k];
            if (hi <= lo) continue;
            if (ns > 0 && seg_hi[ns - 1] == lo) seg_hi[ns - 1] = hi;
            else { seg_lo[ns] = lo; seg_hi[ns] = hi; ns++; }
        }
        seg_pre[0] = 0;
        for (int s = 0; s < ns; s++) seg_pre[s + 1] = seg_pre[s] + (seg_hi[s] - seg_lo[s]);
        *nseg = ns;
    }
}

// map a position inside the concatenated segment list to a particle index
__device__ __forceinline__ uint32_t seg_map(int ns, const uint32_t *seg_lo, const uint32_t *seg_pre, uint32_t i)
{
    int s = 0;
    while (s + 1 < ns && seg_pre[s + 1] <= i) s++;
    return seg_lo[s] + (i - seg_pre[s]);
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
