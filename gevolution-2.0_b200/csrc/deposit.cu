// deposit.cu -- deterministic tile deposits of T00, Tij and T0i.
//
// One CTA owns the 8^3 vertices of a tile (one thread per vertex, or, in the
// FP32 tile launch, per pair of vertices of a z column) and gathers every
// particle whose CIC stencil touches them: its own 8 class buckets plus
// the face-class buckets of the 7 lower neighbour tiles (tile_segments_warp).
//
// The CTA
//   1. turns each particle into a short record of per-particle factors (in the
//      field precision R) and finds the one of the 9^3 cells of the tile's
//      reach (relative cell -1..7 per axis) that it lies in;
//   2. finds the records of each reach cell: when every candidate bucket
//      holds at most REBIN_SORT_MAX particles they already form one run of
//      the candidates' concatenation, because the re-binning keeps buckets
//      that small in (cell, particle ID) order -- the concatenation is taken
//      in chunks of records that fit shared memory (one chunk in the common
//      case); tiles that touch a larger bucket sort record indexes by cell
//      (counting sort) chunk by chunk;
//   3. lets every thread walk the cells whose stencil covers its vertex (8
//      cells) or its two vertices (12 cells, the 4 between them shared) and
//      accumulate the contributions in registers -- no shared-memory atomics
//      on the accumulation path, each output vertex written once with plain
//      stores, no global atomics and no halo fold (projection_comm1,
//      gevolution.hpp:1543, is not needed on one GPU).
// The result does not depend on the order in which the particles were given
// (bitwise reproducible, for unique particle IDs):
//   - sorted candidates: each vertex sums in R in a fixed order (source
//     cell, ID), chunk after chunk;
//   - tiles that touch a bucket above REBIN_SORT_MAX (kept in slot order)
//     accumulate 64-bit fixed point with a per-CTA, per-component scale from
//     an upper bound of the contributions and the particle count, so the sum
//     is exact integer arithmetic.
// Tiles whose reach fits one chunk are done by the tile launch; it lists the
// others for a second, dense-tile launch, so that the common case's kernel
// holds only the single-chunk path (fewer registers, no spills).
//
// Arithmetic follows the reference functors term by term:
//   particle_T00_project  gevolution.hpp:1729-1854
//   particle_Tij_project  gevolution.hpp:2582-2965 (non-CIC_PROJECT_TIJ)
//   particle_T0i_project  gevolution.hpp:2031-2201
#include "common.cuh"
#include "particles.cuh"
#include "kernels.h"

namespace gev {

constexpr int DEP_NT = 512;   // tile vertices; threads of the dense-tile launch (one per vertex)
// Threads of the tile launch: 256, each summing the two vertices (x, y, 2k)
// and (x, y, 2k + 1) of a z column, so that the records of the cell between
// them are read once for both.
#ifndef GEV_DEP_NT_TILE
#define GEV_DEP_NT_TILE 256
#endif
static_assert(GEV_DEP_NT_TILE == 256 || GEV_DEP_NT_TILE == 512, "one or two vertices per thread");
// FP64 records fill the shared memory of two CTAs per SM: the FP64 tile
// launch keeps one thread per vertex (512 threads) for the resident warps.
template <class R> __host__ __device__ constexpr int dep_tile_threads() { return sizeof(R) == 8 ? DEP_NT : GEV_DEP_NT_TILE; }
#ifndef GEV_DEP_MINB_F
#define GEV_DEP_MINB_F 3
#endif
#ifndef GEV_DEP_MINB_T0I_F
#define GEV_DEP_MINB_T0I_F 4
#endif
// the 16-value T00+Tij+S records: chunks of 768 records keep three CTAs per
// SM (1024 would leave two; measured over the full cycle at 512^3)
#ifndef GEV_DEP_MINB_S_F
#define GEV_DEP_MINB_S_F 3
#endif
#ifndef GEV_DEP_CH_S_F
#define GEV_DEP_CH_S_F 768
#endif

#ifndef GEV_DEP_CH_S_F_DENSE
#define GEV_DEP_CH_S_F_DENSE 768
#endif

// records per chunk (shared-memory budget) and the fixed-point exponent limit;
// DENSE: the chunks of the dense-tile launch
template <class R, int KIND = DEP_T00, bool DENSE = false> struct DepCh;
template <int KIND, bool DENSE> struct DepCh<float, KIND, DENSE> {
    static constexpr int v = KIND == DEP_T00_TIJ_S0I ? (DENSE ? GEV_DEP_CH_S_F_DENSE : GEV_DEP_CH_S_F) : 1024;
    static constexpr int EMAX = 120;
};
template <int KIND, bool DENSE> struct DepCh<double, KIND, DENSE> {
    static constexpr int v = 768;
    static constexpr int EMAX = 1000;
};
static_assert(DepCh<float>::v <= REBIN_SORT_MAX && DepCh<float, DEP_T00_TIJ_S0I>::v <= REBIN_SORT_MAX &&
                  DepCh<float, DEP_T00_TIJ_S0I, true>::v <= REBIN_SORT_MAX &&
                  DepCh<double>::v <= REBIN_SORT_MAX,
              "a single-chunk deposit must only see buckets that the re-binning keeps sorted");

// record layout: [d0 d1 d2 | T00: E F G | Tij: W00 W11 W22 W01 W02 W12 | T0i: Q0 Q1 Q2 | S: P0 P1 P2]
// (S: the T0i momenta m q_i without the potential factor, DEP_T00_TIJ_S0I)
template <int KIND> struct DepShape {
    static constexpr bool HAS00 = (KIND == DEP_T00 || KIND == DEP_T00_TIJ || KIND == DEP_T00_TIJ_S0I);
    static constexpr bool HASIJ = (KIND == DEP_TIJ || KIND == DEP_T00_TIJ || KIND == DEP_T00_TIJ_S0I);
    static constexpr bool HAS0I = (KIND == DEP_T0I);
    static constexpr bool HASS = (KIND == DEP_T00_TIJ_S0I);
    static constexpr int NC = (HAS00 ? 1 : 0) + (HASIJ ? 6 : 0) + (HAS0I ? 3 : 0) + (HASS ? 3 : 0);
    static constexpr int F00 = 3;
    static constexpr int FIJ = 3 + (HAS00 ? 3 : 0);
    static constexpr int F0I = 3;
    static constexpr int FS = FIJ + (HASIJ ? 6 : 0);
    static constexpr int NF = 3 + (HAS00 ? 3 : 0) + (HASIJ ? 6 : 0) + (HAS0I ? 3 : 0) + (HASS ? 3 : 0);
    static constexpr int NFP = (NF + 3) & ~3;   // padded for 16-byte record loads
    static constexpr int CIJ = HAS00 ? 1 : 0;   // first Tij output component
    static constexpr int CS = CIJ + (HASIJ ? 6 : 0);   // first S output component
    // Record slots of the Tij weights (k = 00, 11, 22, 01, 02, 12) and of the
    // S momenta.  The 16-value T00+Tij+S record is [d0 d1 d2 E | F G W00 W11 |
    // W22 P0 P1 P2 | W01 W02 W12 -]: the off-diagonal weights, which only the
    // vertices two or three of whose offsets are 0 receive, fill the last
    // 16-byte chunk, which the other half of the gather's corners never load.
    static constexpr bool SPLIT = HAS00 && HASIJ && HASS;
    __host__ __device__ static constexpr int fij(int k) { return SPLIT && k >= 3 ? 12 + (k - 3) : FIJ + k; }
    __host__ __device__ static constexpr int fs(int k) { return SPLIT ? FS - 3 + k : FS + k; }
};

constexpr int DEP_NCELL = 729;                  // 9^3 cells of a tile's reach
constexpr uint16_t DEP_SKIP = 0xFFFFu;
constexpr int DEP_RUN_NONE = 0x7fffffff;        // run start of a reach cell without records

template <class R> __device__ __forceinline__ long long to_fixed(R v);
template <> __device__ __forceinline__ long long to_fixed<float>(float v) { return __float2ll_rn(v); }
template <> __device__ __forceinline__ long long to_fixed<double>(double v) { return __double2ll_rn(v); }

__device__ __forceinline__ int phi_slot(int vx, int vy, int vz) { return (vx + 1) + 10 * ((vy + 1) + 10 * (vz + 1)); }

// Per-particle factors of one particle, in the field precision R (FP32 in
// mixed mode: the record is stored in R anyway).  Returns false when the
// particle lies outside the tile's reach (stale bucket order).  bnd[] receives
// an upper bound of |contribution| per output component.  The reference's
// divisions by e = sqrt(q^2 + a^2) are taken as one reciprocal, and
// f2 / (1 + f2/a^2) as f2 a^2 / e^2 (the same quantity).
template <class R, int KIND, bool USE_PHI>
__device__ __forceinline__ bool make_record(const RawParticle<R> &pr, int N, const FastDiv &fN, int x0, int y0, int z0,
                                            const R *phis, R a, R m00, R mij, R m0i, R (&v)[DepShape<KIND>::NF],
                                            int &lc, R (&bnd)[DepShape<KIND>::NC])
{
    using S = DepShape<KIND>;
    int cx, cy, cz;
    decode_cell(pr.cell, fN, cx, cy, cz);
    const int rx = rel_coord(cx, x0, N), ry = rel_coord(cy, y0, N), rz = rel_coord(cz, z0, N);
    if (rx < -1 || rx > 7 || ry < -1 || ry > 7 || rz < -1 || rz > 7) return false;
    lc = (rx + 1) + 9 * ((ry + 1) + 9 * (rz + 1));
    const R d[3] = {(R)pr.off[0], (R)pr.off[1], (R)pr.off[2]};
    const R q[3] = {pr.q[0], pr.q[1], pr.q[2]};
    v[0] = d[0]; v[1] = d[1]; v[2] = d[2];
    R pm = 0, pint = 0;
    if (USE_PHI) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
            const R ph = phis[phi_slot(rx + bx, ry + by, rz + bz)];
            const R w = (bx ? d[0] : (R)1 - d[0]) * (by ? d[1] : (R)1 - d[1]) * (bz ? d[2] : (R)1 - d[2]);
            pint += w * ph;
            pm = fmax(pm, fabs(ph));
        }
    }
    const R f2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    const R e2 = f2 + a * a;
    const R e = sqrt(e2);
    const R ie = (R)1 / e;
    if constexpr (S::HAS00) {
        if (USE_PHI) {
            const R fc = (R)3 * e + f2 * ie;
            const R g = ((R)0.5 * fc * fc + f2 * a * a * ie * ie) * ie;
            v[S::F00 + 0] = e * m00;
            v[S::F00 + 1] = fc * m00;
            v[S::F00 + 2] = g * m00;
            bnd[0] = fabs(e * m00) + fabs(fc * m00) * pm + fabs(g * m00) * pm * pm;
        } else {
            v[S::F00 + 0] = m00;
            v[S::F00 + 1] = 0;
            v[S::F00 + 2] = 0;
            bnd[0] = fabs(m00);
        }
    }
    if constexpr (S::HASIJ) {
        const R fac = USE_PHI ? (R)1 + ((R)4 + a * a * ie * ie) * pint : (R)1;
        const R s = fac * mij * ie;
        const R W[6] = {s * q[0] * q[0], s * q[1] * q[1], s * q[2] * q[2], s * q[0] * q[1], s * q[0] * q[2], s * q[1] * q[2]};
        // output order 00,01,02,11,12,22
        const int comp[6] = {0, 3, 5, 1, 2, 4};
#pragma unroll
        for (int k = 0; k < 6; k++) {
            v[S::fij(k)] = W[k];
            bnd[S::CIJ + comp[k]] = fabs(W[k]);
        }
    }
    if constexpr (S::HAS0I) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            v[S::F0I + k] = m00 * q[k];
            bnd[k] = fabs(m00 * q[k]) * ((R)1 + (R)2 * pm);
        }
    }
    if constexpr (S::HASS) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            v[S::fs(k)] = m0i * q[k];
            bnd[S::CS + k] = fabs(m0i * q[k]);
        }
    }
    return true;
}

// Multiply a record's value fields by the fixed-point scales of the
// components they feed (the CIC weights stay unscaled).
template <class R, int KIND> __device__ __forceinline__ void scale_record(R *r, const R *scl)
{
    using S = DepShape<KIND>;
    if constexpr (S::HAS00) {
#pragma unroll
        for (int k = 0; k < 3; k++) r[S::F00 + k] *= scl[0];
    }
    if constexpr (S::HASIJ) {
        const int comp[6] = {0, 3, 5, 1, 2, 4};
#pragma unroll
        for (int k = 0; k < 6; k++) r[S::fij(k)] *= scl[S::CIJ + comp[k]];
    }
    if constexpr (S::HAS0I) {
#pragma unroll
        for (int k = 0; k < 3; k++) r[S::F0I + k] *= scl[k];
    }
    if constexpr (S::HASS) {
#pragma unroll
        for (int k = 0; k < 3; k++) r[S::fs(k)] *= scl[S::CS + k];
    }
}

// add the contributions of one (scaled) record to the vertex at offset b from its cell
template <class R, int KIND, bool USE_PHI>
__device__ __forceinline__ void gather_one(const R *r, int bx, int by, int bz, R phv, R phx, R phy, R phz,
                                           long long (&acc)[DepShape<KIND>::NC])
{
    using S = DepShape<KIND>;
    const R wx = bx ? r[0] : (R)1 - r[0];
    const R wy = by ? r[1] : (R)1 - r[1];
    const R wz = bz ? r[2] : (R)1 - r[2];
    const R w = wx * wy * wz;
    if constexpr (S::HAS00) {
        const R val = USE_PHI ? w * (r[S::F00] + (r[S::F00 + 1] + r[S::F00 + 2] * phv) * phv) : w * r[S::F00];
        acc[0] += to_fixed<R>(val);
    }
    if constexpr (S::HASIJ) {
        constexpr int C = S::CIJ;
        acc[C + 0] += to_fixed<R>(w * r[S::fij(0)]);
        acc[C + 3] += to_fixed<R>(w * r[S::fij(1)]);
        acc[C + 5] += to_fixed<R>(w * r[S::fij(2)]);
        if (!bx && !by) acc[C + 1] += to_fixed<R>(wz * r[S::fij(3)]);   // (0,1): x and x+e2
        if (!bx && !bz) acc[C + 2] += to_fixed<R>(wy * r[S::fij(4)]);   // (0,2): x and x+e1
        if (!by && !bz) acc[C + 4] += to_fixed<R>(wx * r[S::fij(5)]);   // (1,2): x and x+e0
    }
    if constexpr (S::HAS0I) {
        // component i lands on the vertices with b_i = 0, weighted by the other two
        // axes and by 1 + phi(vertex) + phi(vertex + e_i)
        if (!bx) acc[0] += to_fixed<R>(wy * wz * r[S::F0I + 0] * ((R)1 + phv + phx));
        if (!by) acc[1] += to_fixed<R>(wx * wz * r[S::F0I + 1] * ((R)1 + phv + phy));
        if (!bz) acc[2] += to_fixed<R>(wx * wy * r[S::F0I + 2] * ((R)1 + phv + phz));
    }
    if constexpr (S::HASS) {
        constexpr int C = S::CS;
        if (!bx) acc[C + 0] += to_fixed<R>(wy * wz * r[S::fs(0)]);
        if (!by) acc[C + 1] += to_fixed<R>(wx * wz * r[S::fs(1)]);
        if (!bz) acc[C + 2] += to_fixed<R>(wx * wy * r[S::fs(2)]);
    }
}

// add the contributions of one (unscaled) record in the field precision
template <class R, int KIND, bool USE_PHI>
__device__ __forceinline__ void gather_sum(const R *r, int bx, int by, int bz, R phv, R phx, R phy, R phz,
                                           R (&acc)[DepShape<KIND>::NC])
{
    using S = DepShape<KIND>;
    const R wx = bx ? r[0] : (R)1 - r[0];
    const R wy = by ? r[1] : (R)1 - r[1];
    const R wz = bz ? r[2] : (R)1 - r[2];
    const R w = wx * wy * wz;
    if constexpr (S::HAS00) {
        acc[0] += USE_PHI ? w * (r[S::F00] + (r[S::F00 + 1] + r[S::F00 + 2] * phv) * phv) : w * r[S::F00];
    }
    if constexpr (S::HASIJ) {
        constexpr int C = S::CIJ;
        acc[C + 0] += w * r[S::fij(0)];
        acc[C + 3] += w * r[S::fij(1)];
        acc[C + 5] += w * r[S::fij(2)];
        if (!bx && !by) acc[C + 1] += wz * r[S::fij(3)];
        if (!bx && !bz) acc[C + 2] += wy * r[S::fij(4)];
        if (!by && !bz) acc[C + 4] += wx * r[S::fij(5)];
    }
    if constexpr (S::HAS0I) {
        if (!bx) acc[0] += wy * wz * r[S::F0I + 0] * ((R)1 + phv + phx);
        if (!by) acc[1] += wx * wz * r[S::F0I + 1] * ((R)1 + phv + phy);
        if (!bz) acc[2] += wx * wy * r[S::F0I + 2] * ((R)1 + phv + phz);
    }
    if constexpr (S::HASS) {
        constexpr int C = S::CS;
        if (!bx) acc[C + 0] += wy * wz * r[S::fs(0)];
        if (!by) acc[C + 1] += wx * wz * r[S::fs(1)];
        if (!bz) acc[C + 2] += wx * wy * r[S::fs(2)];
    }
}

// Records in shared memory: record k is C = NFP / L chunks of 16 bytes (L
// values of R each), stored whole with 16-byte accesses.  Chunk m of record k
// sits in 4-bank group (C k + m') mod 8; the chunk order m' is permuted by
// k so that the same chunk of any 8 consecutive records falls in 8 different
// groups (a quarter warp of 16-byte accesses without bank conflicts): an odd
// C spreads them by itself, C = 2 mod 4 swaps chunk pairs in records 4..7 mod
// 8, C = 4 mod 8 XORs the chunk index with (k / 2) mod 4, C = 0 mod 8 with
// k mod 8.
template <class R, int NFP> struct RecLayout {
    static constexpr int L = 16 / (int)sizeof(R);
    static constexpr int C = NFP / L;
    static_assert(NFP % L == 0, "records are whole 16-byte chunks");
    __device__ __forceinline__ static int chunk(int k, int m)
    {
        if constexpr (C % 8 == 0) return k * C + (m ^ (k & 7));
        else if constexpr (C % 4 == 0) return k * C + (m ^ ((k >> 1) & 3));
        else if constexpr (C % 2 == 0) return k * C + (m ^ ((k >> 2) & 1));
        else return k * C + m;
    }
};

template <class R, int NFP, int NF>
__device__ __forceinline__ void store_record(R *rec, int k, const R (&v)[NF])
{
    using Lay = RecLayout<R, NFP>;
#pragma unroll
    for (int m = 0; m < Lay::C; m++) {
        R *dst = rec + (size_t)Lay::chunk(k, m) * Lay::L;
        auto val = [&](int f) { return f < NF ? v[f] : (R)0; };
        if constexpr (sizeof(R) == 4) {
            *reinterpret_cast<float4 *>(dst) = make_float4(val(4 * m), val(4 * m + 1), val(4 * m + 2), val(4 * m + 3));
        } else {
            *reinterpret_cast<double2 *>(dst) = make_double2(val(2 * m), val(2 * m + 1));
        }
    }
}

template <class R, int NFP> __device__ __forceinline__ void load_record(const R *rec, int k, R (&dst)[NFP])
{
    using Lay = RecLayout<R, NFP>;
#pragma unroll
    for (int m = 0; m < Lay::C; m++) {
        const R *src = rec + (size_t)Lay::chunk(k, m) * Lay::L;
        if constexpr (sizeof(R) == 4) {
            const float4 t = *reinterpret_cast<const float4 *>(src);
            dst[4 * m] = t.x; dst[4 * m + 1] = t.y; dst[4 * m + 2] = t.z; dst[4 * m + 3] = t.w;
        } else {
            const double2 t = *reinterpret_cast<const double2 *>(src);
            dst[2 * m] = t.x; dst[2 * m + 1] = t.y;
        }
    }
}

template <class R, int KIND, bool DENSE = false>
__host__ __device__ constexpr size_t dep_smem_bytes()
{
    return (size_t)DepShape<KIND>::NFP * DepCh<R, KIND, DENSE>::v * sizeof(R) + (size_t)(2 * 730) * sizeof(int) +
           (size_t)3 * DepCh<R, KIND, DENSE>::v * sizeof(uint16_t);
}

// Resident CTAs per SM the register budget is sized for.  The kernel is bound
// by the latency of its dependent phases, so FP32 keeps as many CTAs as the
// shared memory allows: three for the T00/Tij records (their shared memory
// fits no fourth), four for the smaller T0i records.  FP64 records fill the
// shared memory of two CTAs.
template <class R, int KIND> struct DepMinBlocks { static constexpr int v = sizeof(R) == 4 ? GEV_DEP_MINB_F : 2; };
template <> struct DepMinBlocks<float, DEP_T0I> { static constexpr int v = GEV_DEP_MINB_T0I_F; };
template <> struct DepMinBlocks<float, DEP_T00_TIJ_S0I> { static constexpr int v = GEV_DEP_MINB_S_F; };

// The dense-tile launch holds only the paths for tiles whose reach takes
// several chunks, with a register budget of its own.
#ifndef GEV_DEP_MINB_DENSE
#define GEV_DEP_MINB_DENSE 3
#endif

// One tile's deposit; outputs: component c is written to out[c] (N^3 plane
// each).  The tile launch (DENSE = false) finishes every tile whose reach fits
// one chunk and appends the others to the work list work[2..] (count in
// work[0]); the dense-tile launch (DENSE = true) takes them from the list.
template <class R, int KIND, bool USE_PHI, bool DENSE>
__device__ __forceinline__ void deposit_tile(int tile, uint32_t *work, const PView<R> &p, const uint32_t *__restrict__ bstart,
                                             int N, int nt, const R *__restrict__ phi, const DepOut<R> &out, double a,
                                             double m00, double mij, double m0i, int accumulate, int *err, FastDiv fN)
{
    using S = DepShape<KIND>;
    constexpr int NC = S::NC, NF = S::NF, NFP = S::NFP;
    constexpr int CH = DepCh<R, KIND, DENSE>::v;
    constexpr int NT = DENSE ? DEP_NT : dep_tile_threads<R>();   // threads
    constexpr int VPT = DEP_NT / NT;                        // vertices per thread
    extern __shared__ __align__(16) unsigned char dsm[];
    R *rec = reinterpret_cast<R *>(dsm);                      // [CH][NFP]
    int *cstart = reinterpret_cast<int *>(rec + CH * NFP);    // 730
    int *ccount = cstart + 730;                               // 729 (+1 pad)
    uint16_t *order = reinterpret_cast<uint16_t *>(ccount + 730);
    uint16_t *rcell = order + CH;
    uint16_t *rslot = rcell + CH;

    __shared__ R phis[USE_PHI ? 1000 : 1];
    __shared__ uint32_t seg_lo[64], seg_hi[64], seg_pre[65];
    __shared__ unsigned long long vmax[NC];
    __shared__ R scl_s[NC];
    __shared__ double iscl_s[NC];
    __shared__ int wsum[DEP_NT / 32];

    const int t = threadIdx.x;
    const int tx = tile % nt, ty = (tile / nt) % nt, tz = tile / (nt * nt);
    const int x0 = tx * 8, y0 = ty * 8, z0 = tz * 8;

    const R ra = (R)a, rm00 = (R)m00, rmij = (R)mij, rm0i = (R)m0i;
    // the phi stencil loads go out first and stay in flight while the bucket
    // ranges are looked up
    constexpr int PER = (1000 + NT - 1) / NT;
    R pv[PER];
    if (USE_PHI) {
#pragma unroll
        for (int k = 0; k < PER; k++) {
            int s = t + k * NT;
            if (s < 1000) {
                int vx = s % 10 - 1, vy = (s / 10) % 10 - 1, vz = s / 100 - 1;
                pv[k] = __ldg(phi + sidx(N, wrapi(x0 + vx, N), wrapi(y0 + vy, N), wrapi(z0 + vz, N)));
            }
        }
    }
    // the tile's own particles (candidates 0..7: one contiguous range at the
    // head of the concatenation) are loaded as well, for the single-chunk path
    constexpr int PP = (CH + NT - 1) / NT;   // particles per thread (two or three)
    RawParticle<R> raw[PP];
    const uint32_t own_lo = bstart[8 * tile], own_n = bstart[8 * tile + 8] - own_lo;
#pragma unroll
    for (int u = 0; u < PP; u++) {
        const int j = t + u * NT;
        if ((uint32_t)j < own_n) raw[u] = load_particle(p, own_lo + (uint32_t)j);
    }
    // the candidate ranges, formed by warp 0 in registers and stored to shared
    // memory; the barrier below publishes them together with the phi stencil
    // and the per-cell run bounds (no barrier of their own)
    if (t < 32) {
        const TileSegs ts = tile_segments_warp(bstart, nt, tx, ty, tz);
        tile_segments_store(ts, seg_lo, seg_hi, seg_pre);
    }
    if (t < NC) vmax[t] = 0ull;
    for (int c = t; c < 730; c += NT) { cstart[c] = DEP_RUN_NONE; ccount[c] = 0; }
    if (USE_PHI) {
#pragma unroll
        for (int k = 0; k < PER; k++) {
            int s = t + k * NT;
            if (s < 1000) phis[s] = pv[k];
        }
    }
    __syncthreads();
    const uint32_t total = seg_pre[64];
    if (total == 0) {
        // nothing reaches this tile: the deposit is zero
        if (!accumulate) {
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int v = t + i * NT;
                const int64_t gi = sidx(N, x0 + (v & 7), y0 + ((v >> 3) & 7), z0 + (v >> 6));
#pragma unroll
                for (int c = 0; c < NC; c++) out.p[c][gi] = (R)0;
            }
        }
        return;
    }
    const bool multi = total > (uint32_t)CH;
    if constexpr (!DENSE) {
        if (multi) {
            // several chunks: the dense-tile launch takes this tile
            if (t == 0) work[2 + atomicAdd(&work[0], 1u)] = (uint32_t)tile;
            return;
        }
    }

    // exclusive scan of the 729 cell counts into cstart (two cells per thread;
    // the dense-tile launch's fixed-point path, 512 threads)
    auto scan_cells = [&]() {
        const int c0 = 2 * t, c1 = 2 * t + 1;
        const int n0 = c0 < DEP_NCELL ? ccount[c0] : 0;
        const int n1 = c1 < DEP_NCELL ? ccount[c1] : 0;
        int s = n0 + n1, incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, incl, o);
            if ((t & 31) >= o) incl += u;
        }
        if ((t & 31) == 31) wsum[t >> 5] = incl;
        __syncthreads();
        if (t < 32) {
            int w = t < NT / 32 ? wsum[t] : 0, wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int u = __shfl_up_sync(0xffffffffu, wi, o);
                if (t >= o) wi += u;
            }
            if (t < NT / 32) wsum[t] = wi - w;   // exclusive warp offsets
        }
        __syncthreads();
        const int excl = incl - s + wsum[t >> 5];
        if (c0 < DEP_NCELL) cstart[c0] = excl;
        if (c1 < DEP_NCELL) cstart[c1] = excl + n0;
    };

    // the phi values of vertex (vx, vy, vz): at the vertex and at its +x, +y, +z neighbours
    auto vertex_phi = [&](int vx, int vy, int vz, R &pv0, R &pvx, R &pvy, R &pvz) {
        pv0 = pvx = pvy = pvz = 0;
        if (USE_PHI) {
            pv0 = phis[phi_slot(vx, vy, vz)];
            pvx = phis[phi_slot(vx + 1, vy, vz)];
            pvy = phis[phi_slot(vx, vy + 1, vz)];
            pvz = phis[phi_slot(vx, vy, vz + 1)];
        }
    };
    auto write_vertex = [&](int vx, int vy, int vz, const R (&acc)[NC]) {
        const int64_t g = sidx(N, x0 + vx, y0 + vy, z0 + vz);
#pragma unroll
        for (int c = 0; c < NC; c++) {
            R *o = out.p[c];
            o[g] = accumulate ? (R)(o[g] + acc[c]) : acc[c];
        }
    };

    // One chunk of n <= CH candidates whose particles are in raw[]: records
    // stay at their load position; every vertex then adds their contributions
    // in the field precision, in a fixed order (source cell, then ID).
    auto build_chunk = [&](int n, RawParticle<R> (&raw)[PP]) {
        // 1. record j at position j, the reach cell it came from, and the
        //    bounds [cstart, cend) of that cell's run as the smallest and
        //    largest positions of its records (shared-memory atomic min / max:
        //    the bounds do not depend on the order of the updates; cend shares
        //    ccount's storage, cstart starts at DEP_RUN_NONE, cend at 0)
        int *cend = ccount;
#pragma unroll
        for (int u = 0; u < PP; u++) {
            const int j = t + u * NT;
            if (j >= n) continue;
            R v[NF], b[NC];
            int lc;
            if (make_record<R, KIND, USE_PHI>(raw[u], N, fN, x0, y0, z0, phis, ra, rm00, rmij, rm0i, v, lc, b)) {
                store_record<R, NFP>(rec, j, v);
                rcell[j] = (uint16_t)lc;
                atomicMin(&cstart[lc], j);
                atomicMax(&cend[lc], j + 1);
            } else {
                rcell[j] = DEP_SKIP;
            }
        }
        __syncthreads();
        // 2. every record is followed by the same cell up to its run's end:
        //    then each run holds exactly its cell's records (otherwise the
        //    bucket order was not sorted by cell)
        bool bad = false;
        for (int j = t; j < n; j += NT) {
            const uint16_t lc = rcell[j];
            if (lc == DEP_SKIP) continue;
            const int e = cend[lc];
            bad |= j + 1 < e && rcell[j + 1] != lc;
        }
        if (bad) atomicOr(err, ERR_BAD_ORDER);
    };
    // One vertex (VPT == 1): it receives from the cells v - b, b in {0,1}^3,
    // in the order b = 0..7 (a cell without records has cstart = DEP_RUN_NONE
    // > cend = 0).
    const int vx = t & 7, vy = (t >> 3) & 7, vz = t >> 6;
    auto gather_vertex = [&](R (&acc)[NC]) {
        R phv, phx, phy, phz;
        vertex_phi(vx, vy, vz, phv, phx, phy, phz);
        const int lc0 = (vx + 1) + 9 * ((vy + 1) + 9 * (vz + 1));
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int bx = b & 1, by = (b >> 1) & 1, bz = b >> 2;
            const int lc = lc0 - bx - 9 * by - 81 * bz;
            const int k1 = ccount[lc];
            for (int k = cstart[lc]; k < k1; k++) {
                R r[NFP];
                load_record<R, NFP>(rec, k, r);
                gather_sum<R, KIND, USE_PHI>(r, bx, by, bz, phv, phx, phy, phz, acc);
            }
        }
    };
    // Two vertices of a z column (VPT == 2): (vx, vy, vz2) and (vx, vy, vz2 + 1)
    // receive from the cells at z = vz2 - 1, vz2, vz2 + 1; the records of the
    // middle cell feed both (bz = 0 for the lower vertex, bz = 1 for the
    // upper).  Each vertex sums in a fixed order: cell z from low to high, then
    // (bx, by) = (0,0), (1,0), (0,1), (1,1), then ID.
    auto gather_pair = [&](int vz2, R (&acc0)[NC], R (&acc1)[NC]) {
        R p0v, p0x, p0y, p0z, p1v, p1x, p1y, p1z;
        vertex_phi(vx, vy, vz2, p0v, p0x, p0y, p0z);
        vertex_phi(vx, vy, vz2 + 1, p1v, p1x, p1y, p1z);
#pragma unroll
        for (int zc = 0; zc < 3; zc++) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int bx = q & 1, by = q >> 1;
                const int lc = (vx - bx + 1) + 9 * ((vy - by + 1) + 9 * (vz2 + zc));
                const int k1 = ccount[lc];
                for (int k = cstart[lc]; k < k1; k++) {
                    R r[NFP];
                    load_record<R, NFP>(rec, k, r);
                    if (zc <= 1) gather_sum<R, KIND, USE_PHI>(r, bx, by, 1 - zc, p0v, p0x, p0y, p0z, acc0);
                    if (zc >= 1) gather_sum<R, KIND, USE_PHI>(r, bx, by, 2 - zc, p1v, p1x, p1y, p1z, acc1);
                }
            }
        }
    };

    if constexpr (!DENSE) {
        // Single chunk (the common case).  The re-binning keeps every bucket
        // this small in (cell, particle ID) order, so in the concatenation of
        // the candidate buckets the records of each reach cell form one run,
        // already ordered by ID -- the sum is independent of the order in
        // which the particles were given.
        const int n = (int)total;
        // the neighbours' particles (the own ones are loaded already)
#pragma unroll
        for (int u = 0; u < PP; u++) {
            const int j = t + u * NT;
            if (j < n && (uint32_t)j >= own_n) raw[u] = load_particle(p, seg_find(seg_lo, seg_pre, (uint32_t)j));
        }
        build_chunk(n, raw);
        if constexpr (VPT == 2) {
            const int vz2 = 2 * (t >> 6);
            R acc0[NC], acc1[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) { acc0[c] = 0; acc1[c] = 0; }
            gather_pair(vz2, acc0, acc1);
            write_vertex(vx, vy, vz2, acc0);
            write_vertex(vx, vy, vz2 + 1, acc1);
        } else {
            R acc[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) acc[c] = 0;
            gather_vertex(acc);
            write_vertex(vx, vy, vz, acc);
        }
        return;
    } else {

    // Every candidate bucket holds at most REBIN_SORT_MAX particles: the
    // re-binning kept each in (cell, particle ID) order, so the concatenation
    // of the candidates is in a canonical order in which each reach cell's
    // records form one run.  It is taken in chunks of CH, each summed as the
    // single chunk above; a run that crosses a chunk boundary is summed in two
    // parts, at a position fixed by that canonical order -- still independent
    // of the order in which the particles were given.
    if (__syncthreads_and(t >= 64 || seg_hi[t] - seg_lo[t] <= (uint32_t)REBIN_SORT_MAX)) {
        R acc[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) acc[c] = 0;
        for (uint32_t base = 0; base < total; base += (uint32_t)CH) {
            const int n = (int)min((uint32_t)CH, total - base);
            if (base > 0) {
                // records and runs of the previous chunk are done with; the run
                // bounds start over before any record of this chunk updates them
                __syncthreads();
                for (int c = t; c < 730; c += NT) { cstart[c] = DEP_RUN_NONE; ccount[c] = 0; }
                __syncthreads();
            }
            // the chunk's particles (of the first chunk, the own ones are loaded already)
#pragma unroll
            for (int u = 0; u < PP; u++) {
                const uint32_t j = base + (uint32_t)(t + u * NT);
                if (t + u * NT < n && (base > 0 || j >= own_n)) raw[u] = load_particle(p, seg_index(seg_lo, seg_pre, j));
            }
            build_chunk(n, raw);
            gather_vertex(acc);
        }
        write_vertex(vx, vy, vz, acc);
        return;
    }

    auto reduce_bounds = [&](R (&lb)[NC]) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            R m = lb[c];
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if ((t & 31) == 0 && m > (R)0) atomicMax(&vmax[c], (unsigned long long)__double_as_longlong((double)m));
        }
    };
    auto set_scales = [&]() {
        if (t < NC) {
            double m = __longlong_as_double((long long)vmax[t]);
            int e = 0;
            if (m > 0.0) {
                int ex;
                frexp(m * (double)total, &ex);
                e = 61 - ex;
                e = e > DepCh<R>::EMAX ? DepCh<R>::EMAX : (e < -DepCh<R>::EMAX ? -DepCh<R>::EMAX : e);
            }
            scl_s[t] = (R)ldexp(1.0, e);
            iscl_s[t] = ldexp(1.0, -e);
        }
    };

    {
        // bounds over every particle first: the scale must be fixed before the first chunk
        R lb[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) lb[c] = 0;
        for (uint32_t j = t; j < total; j += NT) {
            const uint32_t i = seg_index(seg_lo, seg_pre, j);
            R v[NF], b[NC];
            int lc;
            if (make_record<R, KIND, USE_PHI>(load_particle(p, i), N, fN, x0, y0, z0, phis, ra, rm00, rmij, rm0i, v, lc, b)) {
#pragma unroll
                for (int c = 0; c < NC; c++) lb[c] = fmax(lb[c], b[c]);
            }
        }
        reduce_bounds(lb);
        __syncthreads();
        set_scales();
        __syncthreads();   // every record of the first chunk takes the scales
    }

    long long acc[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] = 0;
    R phv, phx, phy, phz;
    vertex_phi(vx, vy, vz, phv, phx, phy, phz);

    for (uint32_t base = 0; base < total; base += CH) {
        const int n = (int)min((uint32_t)CH, total - base);
        // 1. records and cell counts
        {
            for (int j = t; j < n; j += NT) {
                const uint32_t i = seg_index(seg_lo, seg_pre, base + (uint32_t)j);
                R v[NF], b[NC];
                int lc;
                if (make_record<R, KIND, USE_PHI>(load_particle(p, i), N, fN, x0, y0, z0, phis, ra, rm00, rmij, rm0i, v, lc, b)) {
                    scale_record<R, KIND>(v, scl_s);   // fixed-point scales of the components (weights unscaled)
                    store_record<R, NFP>(rec, j, v);
                    rcell[j] = (uint16_t)lc;
                    rslot[j] = (uint16_t)atomicAdd(&ccount[lc], 1);
                } else {
                    rcell[j] = DEP_SKIP;
                }
            }
        }
        __syncthreads();
        // 2. exclusive scan of the 729 cell counts
        scan_cells();
        __syncthreads();
        // 3. counting sort of record indexes by cell
        for (int j = t; j < n; j += NT) {
            const uint16_t lc = rcell[j];
            if (lc != DEP_SKIP) order[cstart[lc] + rslot[j]] = (uint16_t)j;
        }
        __syncthreads();
        // 4. gather: the vertex receives from the cells v - b, b in {0,1}^3
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int bx = b & 1, by = (b >> 1) & 1, bz = b >> 2;
            const int lc = (vx - bx + 1) + 9 * ((vy - by + 1) + 9 * (vz - bz + 1));
            const int k0 = cstart[lc], k1 = k0 + ccount[lc];
            for (int k = k0; k < k1; k++) {
                R r[NFP];
                load_record<R, NFP>(rec, order[k], r);
                gather_one<R, KIND, USE_PHI>(r, bx, by, bz, phv, phx, phy, phz, acc);
            }
        }
        __syncthreads();
        for (int c = t; c < DEP_NCELL; c += NT) ccount[c] = 0;
        __syncthreads();
    }

    const int64_t gi = sidx(N, x0 + vx, y0 + vy, z0 + vz);
#pragma unroll
    for (int c = 0; c < NC; c++) {
        double val = (double)acc[c] * iscl_s[c];
        R *o = out.p[c];
        if (accumulate) o[gi] = (R)((double)o[gi] + val);
        else o[gi] = (R)val;
    }
    }
}

template <class R, int KIND, bool USE_PHI>
__global__ void __launch_bounds__(dep_tile_threads<R>(), DepMinBlocks<R, KIND>::v)
    k_deposit(PView<R> p, const uint32_t *__restrict__ bstart, int N, int nt, const R *__restrict__ phi, DepOut<R> out,
              double a, double m00, double mij, double m0i, int accumulate, uint32_t *work, int *err, FastDiv fN)
{
    deposit_tile<R, KIND, USE_PHI, false>((int)blockIdx.x, work, p, bstart, N, nt, phi, out, a, m00, mij, m0i, accumulate,
                                          err, fN);
}

// The dense tiles, one at a time per CTA, each CTA claiming the next listed
// tile when it is done with one (their costs differ widely).
template <class R, int KIND, bool USE_PHI>
__global__ void __launch_bounds__(DEP_NT, GEV_DEP_MINB_DENSE)
    k_deposit_dense(PView<R> p, const uint32_t *__restrict__ bstart, int N, int nt, const R *__restrict__ phi,
                    DepOut<R> out, double a, double m00, double mij, double m0i, int accumulate, uint32_t *work, int *err,
                    FastDiv fN)
{
    __shared__ uint32_t next;
    const uint32_t count = work[0];
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(&work[1], 1u);
        __syncthreads();
        const uint32_t i = next;
        if (i >= count) break;
        deposit_tile<R, KIND, USE_PHI, true>((int)work[2 + i], work, p, bstart, N, nt, phi, out, a, m00, mij, m0i,
                                             accumulate, err, fN);
        __syncthreads();   // shared memory and `next` are reused for the next tile
    }
}

static int sm_count()
{
    static int count[SMEM_ATTR_DEVICES] = {};
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < SMEM_ATTR_DEVICES && count[dev] > 0) return count[dev];
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    if (dev >= 0 && dev < SMEM_ATTR_DEVICES) count[dev] = n;
    return n;
}

template <class R, int KIND, bool USE_PHI>
static void launch_k(const PView<R> &p, const uint32_t *bstart, int N, const R *phi, const DepOut<R> &out, double a,
                     double m00, double mij, double m0i, int accumulate, uint32_t *work, int *err, cudaStream_t st)
{
    constexpr size_t smem = dep_smem_bytes<R, KIND>(), smem_dense = dep_smem_bytes<R, KIND, true>();
    static bool attr_set[SMEM_ATTR_DEVICES] = {}, attr_set_dense[SMEM_ATTR_DEVICES] = {};
    raise_smem_limit(k_deposit<R, KIND, USE_PHI>, smem, attr_set);
    raise_smem_limit(k_deposit_dense<R, KIND, USE_PHI>, smem_dense, attr_set_dense);
    const int nt = N / 8;
    const unsigned tiles = (unsigned)nt * nt * nt;
    const FastDiv fN((uint32_t)N);
    k_deposit<R, KIND, USE_PHI><<<tiles, dep_tile_threads<R>(), smem, st>>>(p, bstart, N, nt, phi, out, a, m00, mij, m0i, accumulate,
                                                               work, err, fN);
    // one wave of resident CTAs; those that find the list empty return at once
    const unsigned grid = std::min(tiles, (unsigned)(sm_count() * GEV_DEP_MINB_DENSE));
    k_deposit_dense<R, KIND, USE_PHI><<<grid, DEP_NT, smem_dense, st>>>(p, bstart, N, nt, phi, out, a, m00, mij, m0i,
                                                                        accumulate, work, err, fN);
}

template <class R>
void launch_deposit(int kind, bool use_phi, const PView<R> &p, const uint32_t *bstart, int N, const R *phi,
                    const DepOut<R> &out, double a, double m00, double mij, double m0i, int accumulate, uint32_t *work,
                    int *err, cudaStream_t st)
{
#define GEV_DEP(K)                                                                                                \
    if (kind == K) {                                                                                              \
        if (use_phi) launch_k<R, K, true>(p, bstart, N, phi, out, a, m00, mij, m0i, accumulate, work, err, st);   \
        else launch_k<R, K, false>(p, bstart, N, phi, out, a, m00, mij, m0i, accumulate, work, err, st);          \
        return;                                                                                                   \
    }
    GEV_DEP(DEP_T00)
    GEV_DEP(DEP_TIJ)
    GEV_DEP(DEP_T00_TIJ)
    GEV_DEP(DEP_T0I)
    GEV_DEP(DEP_T00_TIJ_S0I)
#undef GEV_DEP
}

template void launch_deposit<float>(int, bool, const PView<float> &, const uint32_t *, int, const float *,
                                    const DepOut<float> &, double, double, double, double, int, uint32_t *, int *,
                                    cudaStream_t);
template void launch_deposit<double>(int, bool, const PView<double> &, const uint32_t *, int, const double *,
                                     const DepOut<double> &, double, double, double, double, int, uint32_t *, int *,
                                     cudaStream_t);

}  // namespace gev
