// ics.cu -- kernels of the Zel'dovich initial-condition generator
// (gev_ics_zeldovich): the Gaussian white-noise field, the displaced lattice,
// and the linear-theory momenta.
//
// The white noise is a counter-based stream: cell i draws Philox4x32-10
// (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011) with counter (i, 0, 0, 0) and key (seed_lo, seed_hi), and turns
// the first two words into one standard normal by the Box-Muller transform.
// The field therefore depends on the seed and the grid only, not on the launch
// shape.  This generator has the reference's statistics, not its realisation;
// the second generator below (gev_ics_basic) reproduces the reference's own
// realisation.
//
// The reference's generator (generateIC_basic, ic_basic.hpp:1834-2509, the
// tabulated-spectrum branch): k_ics_modes draws the Fourier modes of the
// displacement potential from the reference's sitmo stream (sitmo.cuh) line
// by line exactly as generateDisplacementField (:1165-1610) does, the z pass
// (OP_ICS) divides them by the transformed CIC kernel, and k_ics_template
// builds the particles from the tiled template (initializeParticlePositions,
// :1613-1668) displaced along the potential's gradient
// (displace_pcls_ic_basic, :65-96).
#include <map>
#include <utility>
#include <vector>
#include "gev.h"
#include "common.cuh"
#include "kernels.h"
#include "particles.cuh"
#include "sitmo.cuh"

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

// gsl_spline_eval of a natural cubic spline (GSL's cspline): the interval
// x[i] <= v < x[i+1] found by bisection (the last interval for v = x[n-1]),
// then y[i] + h (b[i] + h (c[i] + h d[i])) with h = v - x[i]
__device__ inline double ics_spline(const IcsSpline &s, double v, int *err)
{
    if (!(v >= s.x[0] && v <= s.x[s.n - 1])) {
        atomicOr(err, ERR_DOMAIN);
        return 0.0;
    }
    int lo = 0, hi = s.n - 1;
    while (hi > lo + 1) {
        const int mid = (lo + hi) >> 1;
        if (s.x[mid] > v) hi = mid; else lo = mid;
    }
    const double h = v - s.x[lo];
    return s.y[lo] + h * (s.b[lo] + h * (s.c[lo] + h * s.d[lo]));
}

// sinc deconvolution factor of generateDisplacementField (:1192-1197),
// evaluated in FP64 and stored in FP32 as the reference's table is
__device__ inline float ics_sinc(int i, int N)
{
    if (i == 0) return 1.0f;
    const double pi = 3.14159265358979323846;
    return (float)(sin(pi * (double)(float)i / (double)(float)N) * (double)(float)N / (pi * (double)(float)i));
}

// uniform (0, 1] draw of the reference: (float) word / (float) 0xFFFFFFFF,
// redrawn while zero; then the Box-Muller radius sqrt(-2 ln u) in FP32
// (boxMullerRadialAmplitude, :1122-1130; ln in FP64, rounded once)
__device__ inline float ics_radius(SitmoStream &rs)
{
    float u;
    do {
        u = (float)rs.next() / 4294967296.0f;
    } while (u == 0.0f);
    return sqrtf((float)(-2.0 * log((double)u)));
}
__device__ inline float ics_uniform(SitmoStream &rs) { return (float)rs.next() / 4294967296.0f; }

// One line (ky, kz) of generateDisplacementField: the four (ky, kz) quadrants
// with their stream offsets (HUGE_SKIP = 65536 words per line and per
// quadrant row), kx = 0 of the kz > N/2 half from the stream of the mirrored
// mode (0, -ky, -kz) with the conjugate phase, and the conjugate draw of
// (0, -ky, 0) for ky > N/2, kz = 0.  Writes the numerator
// e^{+-i 2 pi r2} (1 + 7.5 coeff / k^2) r1 P(|k|) s of every mode (zero for the
// modes the reference sets to zero); OP_ICS divides by the kernel.
__global__ void k_ics_modes(double2 *modes, int N, uint32_t seed, int ksphere, float coeff, IcsSpline sp, int *err)
{
    const int64_t line = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (line >= (int64_t)N * N) return;
    const int ky = (int)(line % N), kz = (int)(line / N);
    const int h = N / 2, kmax = h - 1;
    const float kmax2 = (float)(kmax * kmax);
    const uint64_t H = 65536;
    const double two_pi = 2.0 * 3.14159265358979323846;
    const double four_pi2 = (4.0 * 3.14159265358979323846) * 3.14159265358979323846;
    double2 *row = modes + (int64_t)(h + 1) * line;
    const bool yhi = ky > h, zhi = kz > h;
    const int ay = yhi ? N - ky : ky, az = zhi ? N - kz : kz;
    const float sy = ics_sinc(ay, N), sz = ics_sinc(az, N);

    auto mode = [&](int kx, float k2, float r1, float r2, double sign, float s) {
        const double th = two_pi * (double)r2;
        const float f = 1.0f + 7.5f * coeff / k2;
        double re = cos(th), im = sign * sin(th);
        re *= (double)f; im *= (double)f;
        re *= (double)r1; im *= (double)r1;
        const double pk = ics_spline(sp, (double)sqrtf(k2), err);
        re *= pk; im *= pk;
        re *= (double)s; im *= (double)s;
        row[kx] = make_double2(re, im);
    };

    uint64_t off;
    if (!yhi && !zhi) off = (ky > 0 || kz > 0) ? ((uint64_t)kz * H + (uint64_t)ky) * H : 0;
    else if (yhi && !zhi) off = ((H + (uint64_t)kz) * H + (uint64_t)(N - ky)) * H;
    else if (!yhi) off = ((2 * H + (uint64_t)(N - kz)) * H + (uint64_t)ky) * H;
    else off = ((3 * H + (uint64_t)(N - kz)) * H + (uint64_t)(N - ky)) * H;
    SitmoStream rs(seed, off);
    for (int kx = zhi ? 1 : 0; kx <= h; kx++) {
        float k2 = (float)(kx * kx) + (float)(ay * ay) + (float)(az * az);
        const bool zero = (!yhi && !zhi && k2 == 0.0f) || kx >= kmax || ay >= kmax || az >= kmax ||
                          (k2 >= kmax2 && ksphere > 0);
        if (zero) {
            row[kx] = make_double2(0.0, 0.0);
            continue;
        }
        const float s = ics_sinc(kx, N) * sy * sz;
        k2 = (float)((double)k2 * four_pi2);
        float r1 = ics_radius(rs);
        float r2 = ics_uniform(rs);
        if (yhi && !zhi && kx == 0 && kz == 0) {
            // (0, -ky, 0): the conjugate of the first quadrant's line N - ky
            SitmoStream cs(seed, (uint64_t)(N - ky) * H);
            r1 = ics_radius(cs);
            r2 = -ics_uniform(cs);
        }
        mode(kx, k2, r1, r2, 1.0, s);
    }
    if (zhi) {
        // kx = 0: the first draws of the mirrored mode's line, conjugated
        const uint64_t off0 = !yhi ? (((ky == 0 ? 0 : H) + (uint64_t)(N - kz)) * H + (uint64_t)ky) * H
                                   : ((uint64_t)(N - kz) * H + (uint64_t)(N - ky)) * H;
        float k2 = (float)(ay * ay) + (float)(az * az);
        if (ay >= kmax || az >= kmax || (k2 >= kmax2 && ksphere > 0)) {
            row[0] = make_double2(0.0, 0.0);
        } else {
            const float s = sy * sz;
            k2 = (float)((double)k2 * four_pi2);
            SitmoStream ms(seed, off0);
            const float r1 = ics_radius(ms);
            const float r2 = ics_uniform(ms);
            mode(0, k2, r1, r2, -1.0, s);
        }
    }
}

// Particle i = j + n (xt + T (yt + T zt)) of the template tiled T times per
// axis (its ID, as initializeParticlePositions numbers them), at
// (tile + template position) / T, displaced by the gradient of the
// displacement potential chi at its cell (displace_pcls_ic_basic with
// coeff 1: CIC-weighted forward differences / dx), wrapped into the box.
template <class R>
__global__ void k_ics_template(PView<R> p, const R *__restrict__ chi, const float *__restrict__ tmpl, int64_t ntmpl,
                               int numtile, int N, int64_t np)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int64_t j = i % ntmpl, t = i / ntmpl;
    const int tile[3] = {(int)(t % numtile), (int)((t / numtile) % numtile), (int)(t / ((int64_t)numtile * numtile))};
    double x[3], d[3];
    int c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        x[k] = ((double)tile[k] + (double)tmpl[3 * j + k]) / (double)numtile;
        const double s = x[k] * N, f = floor(s);
        d[k] = s - f;
        c[k] = (((int)f % N) + N) % N;
    }
    auto F = [&](int dx, int dy, int dz) { return ics_phi(chi, N, c[0] + dx, c[1] + dy, c[2] + dz); };
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
    const double dx = 1.0 / N;
    int cc[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double y = x[k] + g[k] / dx;
        y -= floor(y);
        const double s = y * N, f = floor(s);
        double o = s - f;
        int ci = (int)f;
        if (ci >= N) { ci = N - 1; o = 1.0 - 1e-16; }
        if (ci < 0) { ci = 0; o = 0.0; }
        cc[k] = ci;
        p.off[k * p.cap + i] = o;
        p.q[k * p.cap + i] = (R)0;
    }
    p.cell[i] = (uint32_t)sidx(N, cc[0], cc[1], cc[2]);
    p.id[i] = i;
}

void launch_ics_modes(double2 *modes, int N, uint32_t seed, int ksphere, float coeff, const IcsSpline &sp, int *err,
                      cudaStream_t st)
{
    const int64_t lines = (int64_t)N * N;
    k_ics_modes<<<cdiv(lines, 128), 128, 0, st>>>(modes, N, seed, ksphere, coeff, sp, err);
}
template <class R>
void launch_ics_template(PView<R> p, const R *chi, const float *tmpl, int64_t ntmpl, int numtile, int N, int64_t np,
                         cudaStream_t st)
{
    if (np > 0) k_ics_template<R><<<cdiv(np, 256), 256, 0, st>>>(p, chi, tmpl, ntmpl, numtile, N, np);
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
    template void launch_ics_velocity<R>(const PView<R> &, const R *, int, double, cudaStream_t);          \
    template void launch_ics_template<R>(PView<R>, const R *, const float *, int64_t, int, int, int64_t, cudaStream_t);
GEV_ICS_INST(float)
GEV_ICS_INST(double)
#undef GEV_ICS_INST

// ---- host side of gev_ics_basic ----

// Natural cubic spline through (x_i, y_i) (the spline GSL's gsl_interp_cspline
// builds, zero second derivative at both ends): second-derivative halves c_i
// from the tridiagonal system
//   h_{i-1} c_{i-1} + 2 (h_{i-1} + h_i) c_i + h_i c_{i+1}
//       = 3 ((y_{i+1} - y_i) / h_i - (y_i - y_{i-1}) / h_{i-1})
// (Thomas algorithm), then b_i = (y_{i+1} - y_i) / h_i - h_i (c_{i+1} + 2 c_i) / 3
// and d_i = (c_{i+1} - c_i) / (3 h_i) for y(x) = y_i + t (b_i + t (c_i + t d_i)).
void ics_natural_spline(const std::vector<double> &x, const std::vector<double> &y, std::vector<double> &b,
                        std::vector<double> &c, std::vector<double> &d)
{
    const size_t n = x.size();
    b.assign(n, 0.0);
    c.assign(n, 0.0);
    d.assign(n, 0.0);
    if (n > 2) {
        std::vector<double> cp(n, 0.0), dp(n, 0.0);
        for (size_t i = 1; i + 1 < n; i++) {
            const double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
            const double r = 3.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
            const double m = 2.0 * (h0 + h1) - (i > 1 ? h0 * cp[i - 1] : 0.0);
            cp[i] = h1 / m;
            dp[i] = (r - (i > 1 ? h0 * dp[i - 1] : 0.0)) / m;
        }
        for (size_t i = n - 2; i >= 1; i--) {
            c[i] = dp[i] - (i + 2 < n ? cp[i] * c[i + 1] : 0.0);
            if (i == 1) break;
        }
    }
    for (size_t i = 0; i + 1 < n; i++) {
        const double h = x[i + 1] - x[i];
        b[i] = (y[i + 1] - y[i]) / h - h * (c[i + 1] + 2.0 * c[i]) / 3.0;
        d[i] = (c[i + 1] - c[i]) / (3.0 * h);
    }
}

// generateCICKernel (ic_basic.hpp:805-1118) on the host: the kernel relating
// the displacement potential to the CIC density of the displaced template --
// for every template particle and each of the eight octants it can be
// mirrored into, the CIC-weighted second differences along each axis --
// normalised by N^2 Np / N^3 (renorm); without a template, the standard
// lattice Laplacian kernel 6 N^2 at the origin and -N^2 at its six
// neighbours.  Returns the non-zero sites (linear index x + N (y + N z)) with
// their values, accumulated in the field precision R in the reference's
// order; the weights are FP32 as there.
template <class R>
void ics_cic_kernel(int N, int64_t numpcl, const float *pcl, int numtile, std::vector<std::pair<int64_t, R>> &sites)
{
    sites.clear();
    std::map<int64_t, size_t> where;
    const long L = N;
    auto site = [&](long xx, long yy, long zz) -> R & {
        const int64_t idx = (int64_t)xx + (int64_t)L * ((int64_t)yy + (int64_t)L * zz);
        auto it = where.find(idx);
        if (it == where.end()) {
            where[idx] = sites.size();
            sites.push_back({idx, (R)0});
            return sites.back().second;
        }
        return sites[it->second].second;
    };
    auto wrap = [&](long v) { return ((v % L) + L) % L; };
    R renorm = (R)(L * L);
    if (numpcl == 0 || !pcl) {
        site(0, 0, 0) = (R)6 * renorm;
        site(1, 0, 0) = -renorm;
        site(L - 1, 0, 0) = -renorm;
        site(0, 1, 0) = -renorm;
        site(0, 0, 1) = -renorm;
        site(0, L - 1, 0) = -renorm;
        site(0, 0, L - 1) = -renorm;
        return;
    }
    renorm /= (R)(numpcl * (long)numtile * (long)numtile * (long)numtile) / (R)(L * L * L);
    // octant o: which axes use the complement 1 - p (bit set), and the signs
    const int comp[8] = {0, 1, 3, 2, 4, 5, 7, 6};   // bit 0: x, bit 1: y, bit 2: z
    const float fL = (float)L, fT = (float)numtile;
    for (int64_t i = 0; i < numpcl; i++) {
        for (int oct = 0; oct < 8; oct++) {
            float w[3];
            int sgn[3];
            bool inside = true;
            for (int k = 0; k < 3; k++) {
                const bool cmp = (comp[oct] >> k) & 1;
                const float a = cmp ? fL * (1.f - pcl[3 * i + k]) / fT : fL * pcl[3 * i + k] / fT;
                if (a >= 1.f) inside = false;
                w[k] = 1.f - a;
                sgn[k] = cmp ? -1 : 1;
            }
            if (!inside) continue;
            const float wx = w[0], wy = w[1], wz = w[2];
            const long px = wrap(sgn[0]), mx = wrap(-sgn[0]), py = wrap(sgn[1]), my = wrap(-sgn[1]);
            const long pz = wrap(sgn[2]), mz = wrap(-sgn[2]);
            // 0-direction
            float ww = (float)((R)(wy * wz) * renorm);
            float q1 = (wx > 0.9f) ? 2.f : 1.f;
            site(0, 0, 0) += ww * wy * wz * q1;
            site(px, 0, 0) -= ww * wy * wz;
            if (wx > 0.9f) site(mx, 0, 0) -= ww * wy * wz;
            site(0, 0, pz) += ww * wy * (1.f - wz) * q1;
            site(px, 0, pz) -= ww * wy * (1.f - wz);
            if (wx > 0.9f) site(mx, 0, pz) -= ww * wy * (1.f - wz);
            site(0, py, 0) += ww * (1.f - wy) * wz * q1;
            site(px, py, 0) -= ww * (1.f - wy) * wz;
            if (wx > 0.9f) site(mx, py, 0) -= ww * (1.f - wy) * wz;
            site(0, py, pz) += ww * (1.f - wy) * (1.f - wz) * q1;
            site(px, py, pz) -= ww * (1.f - wy) * (1.f - wz);
            if (wx > 0.9f) site(mx, py, pz) -= ww * (1.f - wy) * (1.f - wz);
            // 1-direction
            ww = (float)((R)(wx * wz) * renorm);
            q1 = (wy > 0.9f) ? 2.f : 1.f;
            site(0, 0, 0) += ww * wx * wz * q1;
            site(px, 0, 0) += ww * (1.f - wx) * wz * q1;
            site(0, 0, pz) += ww * wx * (1.f - wz) * q1;
            site(px, 0, pz) += ww * (1.f - wx) * (1.f - wz) * q1;
            site(0, py, 0) -= ww * wx * wz;
            site(px, py, 0) -= ww * (1.f - wx) * wz;
            site(0, py, pz) -= ww * wx * (1.f - wz);
            site(px, py, pz) -= ww * (1.f - wx) * (1.f - wz);
            if (wy > 0.9f) {
                site(0, my, 0) -= ww * wx * wz;
                site(px, my, 0) -= ww * (1.f - wx) * wz;
                site(0, my, pz) -= ww * wx * (1.f - wz);
                site(px, my, pz) -= ww * (1.f - wx) * (1.f - wz);
            }
            // 2-direction
            ww = (float)((R)(wx * wy) * renorm);
            q1 = (wz > 0.9f) ? 2.f : 1.f;
            site(0, 0, 0) += ww * wx * wy * q1;
            site(px, 0, 0) += ww * (1.f - wx) * wy * q1;
            site(0, py, 0) += ww * wx * (1.f - wy) * q1;
            site(px, py, 0) += ww * (1.f - wx) * (1.f - wy) * q1;
            site(0, 0, pz) -= ww * wx * wy;
            site(px, 0, pz) -= ww * (1.f - wx) * wy;
            site(0, py, pz) -= ww * wx * (1.f - wy);
            site(px, py, pz) -= ww * (1.f - wx) * (1.f - wy);
            if (wz > 0.9f) {
                site(0, 0, mz) -= ww * wx * wy;
                site(px, 0, mz) -= ww * (1.f - wx) * wy;
                site(0, py, mz) -= ww * wx * (1.f - wy);
                site(px, py, mz) -= ww * (1.f - wx) * (1.f - wy);
            }
        }
    }
}
template void ics_cic_kernel<float>(int, int64_t, const float *, int, std::vector<std::pair<int64_t, float>> &);
template void ics_cic_kernel<double>(int, int64_t, const float *, int, std::vector<std::pair<int64_t, double>> &);

}  // namespace gev

// The reference IC generator's random stream, words [start, start + n) of the
// stream of `seed` (sitmo.cuh), computed on the host.
extern "C" int gev_sitmo_words(uint32_t seed, uint64_t start, int64_t n, uint32_t *out)
{
    if (n < 0 || (n > 0 && !out)) return GEV_ERR_ARG;
    gev::SitmoStream rs(seed, start);
    for (int64_t i = 0; i < n; i++) out[i] = rs.next();
    return GEV_OK;
}
