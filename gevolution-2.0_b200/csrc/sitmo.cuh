// sitmo.cuh -- the random stream of the reference's initial-condition
// generator (generateDisplacementField, ic_basic.hpp:1165-1610), which draws
// from sitmo::prng_engine (prng_engine.hpp in the reference tree, by M.A. van
// den Berg, MIT licence, version 5).  That engine is the counter-based
// Threefry-4x64-20 block cipher of Salmon, Moraes, Dror and Shaw ("Parallel
// random numbers: as easy as 1, 2, 3", SC 2011) run in counter mode:
//
//   key     = (seed, 0, 0, 0)                       (seed(uint32_t))
//   block b = Threefry-4x64-20(key, counter = (b, 0, 0, 0))
//   word i of the stream = 32-bit half (i mod 8) of block floor(i / 8): even
//           halves are the low 32 bits of 64-bit lane (i mod 8) / 2, odd
//           halves the high ones
//
// and discard(z) from a freshly seeded engine moves to word z.  So every word
// of the stream is a pure function of (seed, index), which lets one GPU thread
// generate any line of modes without running the stream up to it.
//
// Threefry-4x64 as published: key schedule ks[4] = C240 ^ k0 ^ k1 ^ k2 ^ k3
// with C240 = 0x1BD11BDAA9FC1A22; 20 rounds of two MIX operations on word
// pairs (0,1),(2,3) in even rounds and (0,3),(2,1) in odd rounds (the
// Threefish-256 permutation), rotation constants R[r mod 8] =
// (14,16) (52,57) (23,40) (5,37) (25,33) (46,12) (58,22) (32,32); key injection
// s = 0..5 before round 4s (and after round 20): x_i += ks[(s + i) mod 5],
// x_3 += s.
#pragma once
#include <cstdint>

namespace gev {

__host__ __device__ inline uint64_t tf_rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

// Threefry-4x64-20 of counter c under key k into out
__host__ __device__ inline void threefry4x64_20(const uint64_t c[4], const uint64_t k[4], uint64_t out[4])
{
    const int R0[8] = {14, 52, 23, 5, 25, 46, 58, 32};
    const int R1[8] = {16, 57, 40, 37, 33, 12, 22, 32};
    uint64_t ks[5] = {k[0], k[1], k[2], k[3], 0x1BD11BDAA9FC1A22ull ^ k[0] ^ k[1] ^ k[2] ^ k[3]};
    uint64_t x0 = c[0] + ks[0], x1 = c[1] + ks[1], x2 = c[2] + ks[2], x3 = c[3] + ks[3];
#pragma unroll
    for (int r = 0; r < 20; r++) {
        if ((r & 1) == 0) {
            x0 += x1; x1 = tf_rotl(x1, R0[r & 7]) ^ x0;
            x2 += x3; x3 = tf_rotl(x3, R1[r & 7]) ^ x2;
        } else {
            x0 += x3; x3 = tf_rotl(x3, R0[r & 7]) ^ x0;
            x2 += x1; x1 = tf_rotl(x1, R1[r & 7]) ^ x2;
        }
        if ((r & 3) == 3) {
            const int s = (r + 1) >> 2;
            x0 += ks[s % 5];
            x1 += ks[(s + 1) % 5];
            x2 += ks[(s + 2) % 5];
            x3 += ks[(s + 3) % 5] + (uint64_t)s;
        }
    }
    out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

// Sequential reader of the stream of `seed` from word `pos` on; keeps the
// current block.
struct SitmoStream {
    uint64_t key[4];
    uint64_t pos;
    uint64_t block_id;
    uint64_t blk[4];
    bool have;
    __host__ __device__ SitmoStream(uint32_t seed, uint64_t start) : pos(start), block_id(0), have(false)
    {
        key[0] = seed; key[1] = 0; key[2] = 0; key[3] = 0;
        blk[0] = blk[1] = blk[2] = blk[3] = 0;
    }
    __host__ __device__ uint32_t next()
    {
        const uint64_t b = pos >> 3;
        if (!have || b != block_id) {
            const uint64_t c[4] = {b, 0, 0, 0};
            threefry4x64_20(c, key, blk);
            block_id = b;
            have = true;
        }
        const int w = (int)(pos & 7);
        ++pos;
        const uint64_t lane = blk[w >> 1];
        return (w & 1) ? (uint32_t)(lane >> 32) : (uint32_t)(lane & 0xFFFFFFFFull);
    }
};

}  // namespace gev
