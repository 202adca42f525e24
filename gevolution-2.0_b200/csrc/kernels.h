// kernels.h -- host-side launchers of the sm_100a kernels (one translation
// unit per family: deposit.cu, particles_k.cu, solve.cu, lightcone.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>
#include <vector>

#include "common.cuh"
#include "particles.cuh"

namespace gev {

// DEP_T00_TIJ_S0I: T00 and Tij, plus the three T0i sums without their
// potential factor (completed by the B solve's x pass with the new phi)
enum { DEP_T00 = 0, DEP_TIJ = 1, DEP_T00_TIJ = 2, DEP_T0I = 3, DEP_T00_TIJ_S0I = 4 };

template <class R> struct DepOut { R *p[10]; };

// Two launches: every tile whose reach fits one chunk, then the denser tiles
// from the work list `work` (ntiles + 2 words; work[0] and work[1] must be
// zero on entry).
template <class R>
void launch_deposit(int kind, bool use_phi, const PView<R> &p, const uint32_t *bstart, int N, const R *phi,
                    const DepOut<R> &out, double a, double m00, double mij, double m0i, int accumulate, uint32_t *work,
                    int *err, cudaStream_t st);

// ---- particles ----
struct KickDriftParams {
    double dtau_k, a_k, b_k;  // kick: dtau, a, a^2 N
    int nfield_k;
    double dtau_d, a_d, b_d;  // drift
    int nfield_d;
    int do_kick, do_drift, do_bin;
};

template <class R>
void launch_kick_drift(const PView<R> &p, const uint32_t *bstart, int N, const R *phi, const R *chi, const R *Bi,
                       int64_t n3, const KickDriftParams &kp, uint32_t *counts, uint32_t *bucket, uint32_t *rank,
                       unsigned long long *vmax_bits, int *err, cudaStream_t st);

template <class R>
void launch_load_particles(PView<R> p, const double *pos, const double *q, const int64_t *id, int64_t n, int N,
                           int *err, cudaStream_t st);
template <class R>
void launch_store_particles(const PView<R> &p, double *pos, double *q, int64_t *id, int64_t n, int N,
                            cudaStream_t st);
template <class R>
void launch_bin_count(const PView<R> &p, int N, uint32_t *counts, uint32_t *bucket, uint32_t *rank, cudaStream_t st);
void launch_scan(const uint32_t *counts, uint32_t *start, int64_t nb, uint32_t *block_sums, cudaStream_t st);
template <class R>
void launch_rebin(const PView<R> &src, PView<R> dst, const uint32_t *bstart, const uint32_t *bucket,
                  const uint32_t *rank, uint32_t *inv, int N, int *err, cudaStream_t st);

void launch_reduce_sum(const double *partial, int64_t n, double *out, cudaStream_t st);

// FP64 CIC mass density of the particles (m = mass / dx^3) added into rho, and
// an FP64 -> FP32 copy: the power spectrum of a mixed-precision context is
// measured in FP64
template <class R> void launch_cic_f64(const PView<R> &p, int N, double m, double *rho, cudaStream_t st);
void launch_f64_to_f32(const double *in, int64_t n, float *out, cudaStream_t st);

// ---- Fourier passes ----
template <class R> struct FftTables {
    const typename CT<R>::C *tw_full;   // exp(-2 pi i k / N), k < N
    const typename CT<R>::C *tw_half;   // exp(-2 pi i k / (N/2)), k < N/2
    const double *k2;                   // gridk2
    const double2 *ks;                  // kshift
};

template <class R>
void fx_forward(int N, int mode, const R *in, int64_t in_stride, int ncomp, int comp0, const R *phi, const R *chi,
                double bg, double c, double c2, double c3, typename CT<R>::C *out, int64_t out_stride,
                double *partial, const FftTables<R> &tb, cudaStream_t st);
template <class R>
void fy_pass(int N, int sign, typename CT<R>::C *data, int64_t stride, int ncomp, int *err, const FftTables<R> &tb,
             cudaStream_t st);   // err: device error word for the transfer timeout (may be null)
template <class R>
void fx_inverse(int N, const typename CT<R>::C *in, int64_t in_stride, R *out, int64_t out_stride, int ncomp,
                const FftTables<R> &tb, cudaStream_t st);

struct FzParams {
    int op, extra;
    double p0, p1, p2, p3;
    double *phi_hom;
    double *bins;
    unsigned long long *occ;
    int *err;   // device error word for the transfer timeout (may be null)
    const double *tab = nullptr;   // OP_ZELD: ln k then ln P(k), device
    int ntab = 0;
    const double2 *modes = nullptr;   // OP_ICS: mode numerators, device (ics.cu)
};
template <class R>
void fz_pass(int N, const FzParams &fp, typename CT<R>::C *data, int64_t stride, typename CT<R>::C *hij,
             typename CT<R>::C *hijp, typename CT<R>::C *bstate, const FftTables<R> &tb, cudaStream_t st);
int fx_rows_per_block(int N, bool fp64);   // T of the x passes (partial-sum count = N*N/T)
// prepareFTsource in place: T00 form into source (partial[N*N]: sums of the
// source per (y, z) row), Tij form on the six Sij planes
template <class R>
void prep_t00_pass(int N, R *source, const R *phi, const R *chi, double bg, double c, double c2, double c3, double *partial,
                   cudaStream_t st);
template <class R> void prep_tij_pass(int N, R *Sij, const R *phi, double coeff, cudaStream_t st);

// ---- initial conditions ----
template <class R> void launch_ics_noise(R *out, int64_t n3, uint64_t seed, cudaStream_t st);
template <class R> void launch_ics_lattice(PView<R> p, const R *psi, int N, cudaStream_t st);
template <class R> void launch_ics_velocity(const PView<R> &p, const R *phi, int N, double coeff, cudaStream_t st);
// natural cubic spline on the device: knots x, values y, coefficients b, c, d
struct IcsSpline { const double *x, *y, *b, *c, *d; int n; };
void launch_ics_modes(double2 *modes, int N, uint32_t seed, int ksphere, float coeff, const IcsSpline &sp, int *err,
                      cudaStream_t st);
template <class R>
void launch_ics_template(PView<R> p, const R *chi, const float *tmpl, int64_t ntmpl, int numtile, int N, int64_t np,
                         cudaStream_t st);
// host side of the reference's generator (ics.cu)
void ics_natural_spline(const std::vector<double> &x, const std::vector<double> &y, std::vector<double> &b,
                        std::vector<double> &c, std::vector<double> &d);
template <class R>
void ics_cic_kernel(int N, int64_t numpcl, const float *pcl, int numtile, std::vector<std::pair<int64_t, R>> &sites);

// ---- lightcone ----
struct LcKernelArgs {
    double vtx[64][3];      // periodic images of the vertex that can intersect the shell
    double lc_vertex[3];    // the lightcone's own vertex (output positions are relative to it)
    int nvtx;
    double direction[3];
    double opening;
    double inner, outer, dist;
    double dtau, dtau_old, a, dadtau, boxsize;
    int tracer_factor;
    const unsigned long long *backlog;   // ID set of the previous cycle (hash table)
    int64_t backlog_cap;                 // power of two (0: empty)
    int64_t capacity;                    // output slots
};
// a shell's output buffers and ID log for one cycle
struct LcOut {
    float *pos, *vel;
    int64_t *ids;
    unsigned long long *count, *newlog;
    int64_t newlog_cap;
};
constexpr unsigned long long LC_EMPTY = ~0ull;   // free slot of an ID set (tables are filled with 0xff bytes)
constexpr int64_t LC_MAX_PROBES = 4096;          // bound on linear probing (load factor stays below 1/4)
template <class R>
void launch_lightcone(const PView<R> &p, const uint32_t *bstart, int N, const R *phi, const LcKernelArgs &la, float *pos, float *vel,
                      int64_t *ids, unsigned long long *count, unsigned long long *newlog, int64_t newlog_cap, int *err,
                      cudaStream_t st);

}  // namespace gev
