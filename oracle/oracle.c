/*
 * oracle.c -- FP64 CPU restatement of gevolution-2.0's per-step PM cycle.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each function names the reference
 * code it restates; the arithmetic follows those lines term by term so that the
 * CUDA kernels can be checked against it.  Citations are file:line inside the
 * gevolution-2.0 source tree.
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

#define IDX(N, x, y, z) ((int64_t)(x) + (int64_t)(N) * ((int64_t)(y) + (int64_t)(N) * (int64_t)(z)))

static inline int wrap(int i, int N) { i %= N; return i < 0 ? i + N : i; }

/* ------------------------------------------------------------------------- */
/* FFT: mixed-radix recursive Cooley-Tukey, exact double twiddles.            */
/* Stands in for cuFFT/FFTW behind LATfield2's PlanFFT (main.cu:742 etc.).    */
/* ------------------------------------------------------------------------- */

static int smallest_factor(int n)
{
    for (int p = 2; p * p <= n; p++)
        if (n % p == 0) return p;
    return n;
}

/* exp(sign 2 pi i j / n) for j < n, from the exact angle of each j */
static cplx *twiddles(int n, int sign)
{
    cplx *w = malloc(sizeof(cplx) * n);
    for (int j = 0; j < n; j++) {
        double ang = sign * 2.0 * M_PI * (double)j / n;
        w[j] = cos(ang) + I * sin(ang);
    }
    return w;
}

/* DFT of length n of in[0], in[is], ...; w holds the twiddles of a length
 * n0 = n * ws transform, so exp(sign 2 pi i j / n) = w[j * ws] */
static void dft_rec(int n, const cplx *in, long is, cplx *out, const cplx *w, long ws)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = smallest_factor(n);
    if (p == n) {                       /* prime length: direct sum */
        for (int k = 0; k < n; k++) {
            cplx s = 0;
            for (int j = 0; j < n; j++) s += in[j * is] * w[((long)j * k % n) * ws];
            out[k] = s;
        }
        return;
    }
    int m = n / p;
    for (int r = 0; r < p; r++) dft_rec(m, in + r * is, is * p, out + r * m, w, ws * p);
    cplx tmp[p];
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) tmp[r] = out[r * m + k] * w[(long)r * k * ws];
        for (int q = 0; q < p; q++) {
            cplx s = 0;
            for (int r = 0; r < p; r++) s += tmp[r] * w[(long)((r * q) % p) * m * ws];
            out[k + q * m] = s;
        }
    }
}

void orc_fft1d(int n, double *re_im, int sign)
{
    cplx *a = (cplx *)re_im;
    cplx *in = malloc(sizeof(cplx) * n);
    cplx *w = twiddles(n, sign);
    memcpy(in, a, sizeof(cplx) * n);
    dft_rec(n, in, 1, a, w, 1);
    free(in);
    free(w);
}

/* transform along y (axis 1) and z (axis 2) of a (N/2+1) x N x N complex block */
static void fft_yz(int N, cplx *c, int sign, int axis_first_z)
{
    const int P = N / 2 + 1;
    cplx *w = twiddles(N, sign);
    for (int pass = 0; pass < 2; pass++) {
        int along_z = axis_first_z ? (pass == 0) : (pass == 1);
#pragma omp parallel
        {
            cplx *col = malloc(sizeof(cplx) * N), *res = malloc(sizeof(cplx) * N);
#pragma omp for collapse(2) schedule(static)
            for (int o = 0; o < N; o++)
                for (int kx = 0; kx < P; kx++) {
                    for (int t = 0; t < N; t++) {
                        long idx = along_z ? kx + (long)P * (o + (long)N * t) : kx + (long)P * (t + (long)N * o);
                        col[t] = c[idx];
                    }
                    dft_rec(N, col, 1, res, w, 1);
                    for (int t = 0; t < N; t++) {
                        long idx = along_z ? kx + (long)P * (o + (long)N * t) : kx + (long)P * (t + (long)N * o);
                        c[idx] = res[t];
                    }
                }
            free(col); free(res);
        }
    }
    free(w);
}

void orc_r2c(int N, const double *in, double *out_)
{
    const int P = N / 2 + 1;
    cplx *out = (cplx *)out_;
    cplx *w = twiddles(N, -1);
#pragma omp parallel
    {
        cplx *row = malloc(sizeof(cplx) * N), *res = malloc(sizeof(cplx) * N);
#pragma omp for collapse(2) schedule(static)
        for (int z = 0; z < N; z++)
            for (int y = 0; y < N; y++) {
                for (int x = 0; x < N; x++) row[x] = in[IDX(N, x, y, z)];
                dft_rec(N, row, 1, res, w, 1);
                for (int kx = 0; kx < P; kx++) out[kx + (long)P * (y + (long)N * z)] = res[kx];
            }
        free(row); free(res);
    }
    free(w);
    fft_yz(N, out, -1, 0);
}

/* C2R: inverse along z and y, then along x with the Hermitian extension of each
 * row; the imaginary parts of the kx=0 and kx=N/2 entries do not contribute. */
void orc_c2r(int N, const double *in_, double *out)
{
    const int P = N / 2 + 1;
    cplx *c = malloc(sizeof(cplx) * (size_t)P * N * N);
    memcpy(c, in_, sizeof(cplx) * (size_t)P * N * N);
    fft_yz(N, c, +1, 1);
    cplx *w = twiddles(N, +1);
#pragma omp parallel
    {
        cplx *row = malloc(sizeof(cplx) * N), *res = malloc(sizeof(cplx) * N);
#pragma omp for collapse(2) schedule(static)
        for (int z = 0; z < N; z++)
            for (int y = 0; y < N; y++) {
                const cplx *r = c + (long)P * (y + (long)N * z);
                for (int k = 0; k < N; k++) row[k] = (k < P) ? r[k] : conj(r[N - k]);
                row[0] = creal(row[0]);
                if (N % 2 == 0) row[N / 2] = creal(row[N / 2]);
                dft_rec(N, row, 1, res, w, 1);
                for (int x = 0; x < N; x++) out[IDX(N, x, y, z)] = creal(res[x]);
            }
        free(row); free(res);
    }
    free(w);
    free(c);
}

/* ------------------------------------------------------------------------- */
/* particle helpers: LATfield2 assigns a particle to the site floor(pos/dx)   */
/* and passes ref_dist = pos/dx - site (gevolution.hpp:1339,1358).            */
/* ------------------------------------------------------------------------- */

static inline void locate(int N, const double *p, int *c, double *d)
{
    for (int i = 0; i < 3; i++) {
        double s = p[i] * N;
        double f = floor(s);
        d[i] = s - f;
        c[i] = wrap((int)f, N);
    }
}

/* field value at site c + (dx,dy,dz), periodic */
static inline double F(const double *f, int N, const int *c, int dx, int dy, int dz)
{
    return f[IDX(N, wrap(c[0] + dx, N), wrap(c[1] + dy, N), wrap(c[2] + dz, N))];
}

static inline double *Fp(double *f, int N, const int *c, int dx, int dy, int dz)
{
    return f + IDX(N, wrap(c[0] + dx, N), wrap(c[1] + dy, N), wrap(c[2] + dz, N));
}

/* corner k = 4*bx + 2*by + bz, CIC weight (gevolution.hpp:1764-1771) */
static inline double cicw(const double *d, int k)
{
    int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
    return (bx ? d[0] : 1.0 - d[0]) * (by ? d[1] : 1.0 - d[1]) * (bz ? d[2] : 1.0 - d[2]);
}

/* particle_T00_project: gevolution.hpp:1729-1854 (host branch 1781-1818) */
void orc_project_T00(int N, int64_t np, const double *pos, const double *q, double mass0,
                     const double *phi, double a, double coeff, double *T00)
{
    const double dx = 1.0 / N;
    for (int64_t p = 0; p < np; p++) {
        int c[3]; double d[3];
        locate(N, pos + 3 * p, c, d);
        double mass = mass0 * coeff / (dx * dx * dx);
        if (phi) {
            const double *v = q + 3 * p;
            double f2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            double e = sqrt(f2 + a * a);
            double f = 3.0 * e + f2 / e;
            f2 = (0.5 * f * f + f2 / (1.0 + f2 / a / a)) / e;
            mass /= a;
            for (int k = 0; k < 8; k++) {
                int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
                double ph = F(phi, N, c, bx, by, bz);
                *Fp(T00, N, c, bx, by, bz) += cicw(d, k) * (e + f * ph + f2 * ph * ph) * mass;
            }
        } else {
            for (int k = 0; k < 8; k++) {
                int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
                *Fp(T00, N, c, bx, by, bz) += cicw(d, k) * mass;
            }
        }
    }
}

/* plain mass CIC used for the validation spectrum (gevolution.hpp:1902-1905,
 * LATfield2 meshprojection): rho += m/dx^3 * w */
void orc_project_cic(int N, int64_t np, const double *pos, double mass, double *rho)
{
    orc_project_T00(N, np, pos, NULL, mass, NULL, 1.0, 1.0, rho);
}

/* particle_Tij_project: gevolution.hpp:2582-2965, non-CIC_PROJECT_TIJ branch
 * (diagonal 2705-2724, off-diagonal 2778-2812, targets 2957-2962) */
void orc_project_Tij(int N, int64_t np, const double *pos, const double *q, double mass0,
                     const double *phi, double a, double coeff, double *Tij)
{
    const double dx = 1.0 / N;
    const int64_t n3 = (int64_t)N * N * N;
    double mass = mass0 * coeff / (dx * dx * dx) / a;
    for (int64_t p = 0; p < np; p++) {
        int c[3]; double d[3];
        locate(N, pos + 3 * p, c, d);
        const double *v = q + 3 * p;
        double f = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double e = sqrt(f + a * a);
        if (phi) {
            f = 4.0 + a * a / (f + a * a);
            double pint = 0;
            for (int k = 0; k < 8; k++)
                pint += cicw(d, k) * F(phi, N, c, (k >> 2) & 1, (k >> 1) & 1, k & 1);
            f = 1.0 + f * pint;
        } else {
            f = 1.0;
        }
        static const int diag_comp[3] = {0, 3, 5};
        for (int i = 0; i < 3; i++) {
            double w = f * mass * v[i] * v[i] / e;
            double *T = Tij + diag_comp[i] * n3;
            for (int k = 0; k < 8; k++)
                *Fp(T, N, c, (k >> 2) & 1, (k >> 1) & 1, k & 1) += w * cicw(d, k);
        }
        double w;
        w = f * mass * v[0] * v[1] / e;           /* (0,1): x and x+e2 */
        *Fp(Tij + 1 * n3, N, c, 0, 0, 0) += w * (1.0 - d[2]);
        *Fp(Tij + 1 * n3, N, c, 0, 0, 1) += w * d[2];
        w = f * mass * v[0] * v[2] / e;           /* (0,2): x and x+e1 */
        *Fp(Tij + 2 * n3, N, c, 0, 0, 0) += w * (1.0 - d[1]);
        *Fp(Tij + 2 * n3, N, c, 0, 1, 0) += w * d[1];
        w = f * mass * v[1] * v[2] / e;           /* (1,2): x and x+e0 */
        *Fp(Tij + 4 * n3, N, c, 0, 0, 0) += w * (1.0 - d[0]);
        *Fp(Tij + 4 * n3, N, c, 1, 0, 0) += w * d[0];
    }
}

/* particle_T0i_project: gevolution.hpp:2031-2201 (host branch 2090-2105) */
void orc_project_T0i(int N, int64_t np, const double *pos, const double *q, double mass0,
                     const double *phi, double coeff, double *T0i)
{
    const double dx = 1.0 / N;
    const int64_t n3 = (int64_t)N * N * N;
    double mass = mass0 * coeff / (dx * dx * dx);
    for (int64_t p = 0; p < np; p++) {
        int c[3]; double d[3];
        locate(N, pos + 3 * p, c, d);
        const double *v = q + 3 * p;
        double ph[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (phi)
            for (int k = 0; k < 8; k++) ph[k] = F(phi, N, c, (k >> 2) & 1, (k >> 1) & 1, k & 1);
        double *B0 = T0i, *B1 = T0i + n3, *B2 = T0i + 2 * n3;
        *Fp(B0, N, c, 0, 0, 0) += (1 - d[1]) * (1 - d[2]) * (1 + ph[0] + ph[4]) * mass * v[0];
        *Fp(B1, N, c, 0, 0, 0) += (1 - d[0]) * (1 - d[2]) * (1 + ph[0] + ph[2]) * mass * v[1];
        *Fp(B2, N, c, 0, 0, 0) += (1 - d[0]) * (1 - d[1]) * (1 + ph[0] + ph[1]) * mass * v[2];
        *Fp(B1, N, c, 1, 0, 0) += d[0] * (1 - d[2]) * (1 + ph[4] + ph[6]) * mass * v[1];
        *Fp(B2, N, c, 1, 0, 0) += d[0] * (1 - d[1]) * (1 + ph[4] + ph[5]) * mass * v[2];
        *Fp(B0, N, c, 0, 1, 0) += d[1] * (1 - d[2]) * (1 + ph[2] + ph[6]) * mass * v[0];
        *Fp(B2, N, c, 0, 1, 0) += d[1] * (1 - d[0]) * (1 + ph[2] + ph[3]) * mass * v[2];
        *Fp(B0, N, c, 0, 0, 1) += d[2] * (1 - d[1]) * (1 + ph[1] + ph[5]) * mass * v[0];
        *Fp(B1, N, c, 0, 0, 1) += d[2] * (1 - d[0]) * (1 + ph[1] + ph[3]) * mass * v[1];
        *Fp(B0, N, c, 0, 1, 1) += d[1] * d[2] * (1 + ph[3] + ph[7]) * mass * v[0];
        *Fp(B1, N, c, 1, 0, 1) += d[0] * d[2] * (1 + ph[5] + ph[7]) * mass * v[1];
        *Fp(B2, N, c, 1, 1, 0) += d[0] * d[1] * (1 + ph[6] + ph[7]) * mass * v[2];
    }
}

/* ------------------------------------------------------------------------- */
/* prepareFTsource (PHINONLINEAR on: config/defaults.mk)                     */
/* ------------------------------------------------------------------------- */

/* prepareFTsource_T00: gevolution.hpp:160-171; returns the sum of source (:162, :215) */
double orc_prepare_T00(int N, const double *phi, const double *chi, const double *source,
                       double bgmodel, double coeff, double coeff2, double coeff3,
                       double *result)
{
    double sum = 0;
#pragma omp parallel for collapse(2) reduction(+ : sum) schedule(static)
    for (int z = 0; z < N; z++)
        for (int y = 0; y < N; y++)
            for (int x = 0; x < N; x++) {
                int c[3] = {x, y, z};
                int64_t i = IDX(N, x, y, z);
                double s = source[i];
                double ph = phi[i];
                sum += s;
                double r = coeff2 * (s - bgmodel);
                r *= 1.0 - 2.0 * ph * (1.0 - ph);
                double g;
                g = F(phi, N, c, -1, 0, 0) - F(phi, N, c, 1, 0, 0); r += 0.125 * g * g;
                g = F(phi, N, c, 0, -1, 0) - F(phi, N, c, 0, 1, 0); r += 0.125 * g * g;
                g = F(phi, N, c, 0, 0, -1) - F(phi, N, c, 0, 0, 1); r += 0.125 * g * g;
                r += (coeff3 * (1.0 - 3.0 * ph) - coeff) * ph - coeff3 * chi[i];
                result[i] = r;
            }
    return sum;
}

/* prepareFTsource_Tij: gevolution.hpp:64-107 (6 planes 00,01,02,11,12,22) */
void orc_prepare_Tij(int N, const double *phi, const double *Tij, double coeff, double *Sij)
{
    const int64_t n3 = (int64_t)N * N * N;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < N; z++)
        for (int y = 0; y < N; y++)
            for (int x = 0; x < N; x++) {
                int c[3] = {x, y, z};
                int64_t i = IDX(N, x, y, z);
                double p0 = phi[i];
                double pp[3] = {F(phi, N, c, 1, 0, 0), F(phi, N, c, 0, 1, 0), F(phi, N, c, 0, 0, 1)};
                double pm[3] = {F(phi, N, c, -1, 0, 0), F(phi, N, c, 0, -1, 0), F(phi, N, c, 0, 0, -1)};
                double p01 = F(phi, N, c, 1, 1, 0), p02 = F(phi, N, c, 1, 0, 1), p12 = F(phi, N, c, 0, 1, 1);
                double t[6];
                for (int k = 0; k < 6; k++) t[k] = Tij[k * n3 + i];
                Sij[0 * n3 + i] = 0.5 * (pp[0] - pm[0]) * (pp[0] - pm[0]) + coeff * t[0];
                Sij[3 * n3 + i] = 0.5 * (pp[1] - pm[1]) * (pp[1] - pm[1]) + coeff * t[3];
                Sij[5 * n3 + i] = 0.5 * (pp[2] - pm[2]) * (pp[2] - pm[2]) + coeff * t[5];
                Sij[1 * n3 + i] = pp[0] * pp[1] - p0 * p01 + 0.5 * (p0 * p0 - pp[0] * pp[0] - pp[1] * pp[1] + p01 * p01) + coeff * t[1];
                Sij[2 * n3 + i] = pp[0] * pp[2] - p0 * p02 + 0.5 * (p0 * p0 - pp[0] * pp[0] - pp[2] * pp[2] + p02 * p02) + coeff * t[2];
                Sij[4 * n3 + i] = pp[1] * pp[2] - p0 * p12 + 0.5 * (p0 * p0 - pp[1] * pp[1] - pp[2] * pp[2] + p12 * p12) + coeff * t[4];
            }
}

/* ------------------------------------------------------------------------- */
/* Fourier-space solvers.  gridk2[i] = (2N sin(pi i/N))^2 and                 */
/* kshift[i] = 2N sin(pi i/N) exp(-i pi i/N) as in gevolution.hpp:269-275.    */
/* ------------------------------------------------------------------------- */

typedef struct { double *k2; cplx *ks; } ktab;

static ktab make_ktab(int N)
{
    ktab t;
    t.k2 = malloc(sizeof(double) * N);
    t.ks = malloc(sizeof(cplx) * N);
    for (int i = 0; i < N; i++) {
        double g = 2.0 * (double)N * sin(M_PI * (double)i / (double)N);
        t.ks[i] = g * (cos(M_PI * (double)i / (double)N) - I * sin(M_PI * (double)i / (double)N));
        t.k2[i] = g * g;
    }
    return t;
}

static void free_ktab(ktab t) { free(t.k2); free(t.ks); }

#define KLOOP(N)                                                        \
    _Pragma("omp parallel for collapse(2) schedule(static)")            \
    for (int kz = 0; kz < (N); kz++)                                    \
        for (int ky = 0; ky < (N); ky++)                                \
            for (int kx = 0; kx <= (N) / 2; kx++)

#define KIDX(N, kx, ky, kz) ((int64_t)(kx) + (int64_t)((N) / 2 + 1) * ((int64_t)(ky) + (int64_t)(N) * (int64_t)(kz)))

/* solveModifiedPoissonFT: gevolution.hpp:806-852 */
void orc_solve_poisson(int N, const double *srcFT_, double *potFT_, double coeff, double modif)
{
    const cplx *src = (const cplx *)srcFT_;
    cplx *pot = (cplx *)potFT_;
    ktab t = make_ktab(N);
    coeff /= -((double)N * (double)N * (double)N);
    KLOOP(N)
    {
        int64_t i = KIDX(N, kx, ky, kz);
        double den = t.k2[kx] + t.k2[ky] + t.k2[kz] + modif;
        pot[i] = (den != 0.0) ? src[i] * coeff / den : 0.0;
    }
    if (modif == 0) pot[0] = 0;
    free_ktab(t);
}

/* projectFTscalar: gevolution.hpp:251-340 */
void orc_project_scalar(int N, const double *SijFT_, double *chiFT_, int add)
{
    const cplx *S = (const cplx *)SijFT_;
    cplx *chi = (cplx *)chiFT_;
    const int64_t m = (int64_t)(N / 2 + 1) * N * N;
    ktab t = make_ktab(N);
    KLOOP(N)
    {
        int64_t i = KIDX(N, kx, ky, kz);
        double g0 = t.k2[kx], g1 = t.k2[ky], g2 = t.k2[kz];
        cplx k0 = t.ks[kx], k1 = t.ks[ky], k2 = t.ks[kz];
        double ksum = g0 + g1 + g2;
        cplx v = 0;
        if (ksum > 0) {
            v = ((g1 + g2 - 2.0 * g0) * S[0 * m + i] + (g0 + g2 - 2.0 * g1) * S[3 * m + i] +
                 (g0 + g1 - 2.0 * g2) * S[5 * m + i] - 6.0 * k0 * k1 * S[1 * m + i] -
                 6.0 * k0 * k2 * S[2 * m + i] - 6.0 * k1 * k2 * S[4 * m + i]) /
                (2.0 * ksum * ksum * N);
        }
        chi[i] = add ? chi[i] + v : v;
    }
    chi[0] = 0;
    free_ktab(t);
}

/* projectFTvector: gevolution.hpp:449-515 */
void orc_project_vector(int N, const double *SiFT_, double *BiFT_, double coeff, double modif)
{
    const cplx *S = (const cplx *)SiFT_;
    cplx *B = (cplx *)BiFT_;
    const int64_t m = (int64_t)(N / 2 + 1) * N * N;
    ktab t = make_ktab(N);
    KLOOP(N)
    {
        int64_t i = KIDX(N, kx, ky, kz);
        double k2 = t.k2[kx] + t.k2[ky] + t.k2[kz];
        cplx ks[3] = {t.ks[kx], t.ks[ky], t.ks[kz]};
        cplx s[3] = {S[i], S[m + i], S[2 * m + i]};
        if (k2 > 0) {
            cplx tmp = (ks[0] * s[0] + ks[1] * s[1] + ks[2] * s[2]) / k2;
            for (int c = 0; c < 3; c++) B[c * m + i] = (s[c] - conj(ks[c]) * tmp) * 4.0 * coeff / (k2 + modif);
        } else {
            for (int c = 0; c < 3; c++) B[c * m + i] = 0;
        }
    }
    free_ktab(t);
}

/* evolveFTvector: gevolution.hpp:359-429 */
void orc_evolve_vector(int N, const double *SijFT_, double *BiFT_, double a2dtau)
{
    const cplx *S = (const cplx *)SijFT_;
    cplx *B = (cplx *)BiFT_;
    const int64_t m = (int64_t)(N / 2 + 1) * N * N;
    ktab t = make_ktab(N);
    KLOOP(N)
    {
        int64_t i = KIDX(N, kx, ky, kz);
        double g0 = t.k2[kx], g1 = t.k2[ky], g2 = t.k2[kz];
        cplx k0 = t.ks[kx], k1 = t.ks[ky], k2 = t.ks[kz];
        double k4 = g0 + g1 + g2;
        k4 *= k4;
        if (k4 > 0) {
            cplx fac = I * (-2.0 * a2dtau / k4);
            cplx S00 = S[i], S01 = S[m + i], S02 = S[2 * m + i], S11 = S[3 * m + i], S12 = S[4 * m + i], S22 = S[5 * m + i];
            B[i] += fac * (conj(k0) * ((g1 + g2) * S00 - g1 * S11 - g2 * S22 - 2.0 * k1 * k2 * S12) + (g1 + g2 - g0) * (k1 * S01 + k2 * S02));
            B[m + i] += fac * (conj(k1) * ((g0 + g2) * S11 - g0 * S00 - g2 * S22 - 2.0 * k0 * k2 * S02) + (g0 + g2 - g1) * (k0 * S01 + k2 * S12));
            B[2 * m + i] += fac * (conj(k2) * ((g0 + g1) * S22 - g0 * S00 - g1 * S11 - 2.0 * k0 * k1 * S01) + (g0 + g1 - g2) * (k0 * S02 + k1 * S12));
        } else {
            B[i] = B[m + i] = B[2 * m + i] = 0;
        }
    }
    free_ktab(t);
}

/* TT projection numerators shared by projectFTtensor (gevolution.hpp:744-769)
 * and evolveFTtensor (:590-615, :636-661); out[c] before the 1/k^6 (or 1/k^4) */
static void tt_numerators(const double *g, const cplx *ks, double k2, const cplx *S, cplx *out)
{
    cplx Sxx = S[0], Sxy = S[1], Sxz = S[2], Syy = S[3], Syz = S[4], Szz = S[5];
    out[0] = (g[0] - k2) * ((g[0] - k2) * Sxx + 2.0 * ks[0] * (ks[1] * Sxy + ks[2] * Sxz)) +
             ((g[0] + k2) * (g[1] + k2) - 2.0 * k2 * k2) * Syy + ((g[0] + k2) * (g[2] + k2) - 2.0 * k2 * k2) * Szz +
             2.0 * (g[0] + k2) * ks[1] * ks[2] * Syz;
    out[1] = 2.0 * (g[0] - k2) * (g[1] - k2) * Sxy + (g[2] + k2) * conj(ks[0]) * conj(ks[1]) * Szz +
             (g[0] - k2) * conj(ks[1]) * (conj(ks[0]) * Sxx + 2.0 * ks[2] * Sxz) +
             (g[1] - k2) * conj(ks[0]) * (conj(ks[1]) * Syy + 2.0 * ks[2] * Syz);
    out[2] = 2.0 * (g[0] - k2) * (g[2] - k2) * Sxz + (g[1] + k2) * conj(ks[0]) * conj(ks[2]) * Syy +
             (g[0] - k2) * conj(ks[2]) * (conj(ks[0]) * Sxx + 2.0 * ks[1] * Sxy) +
             (g[2] - k2) * conj(ks[0]) * (conj(ks[2]) * Szz + 2.0 * ks[1] * Syz);
    out[3] = (g[1] - k2) * ((g[1] - k2) * Syy + 2.0 * ks[1] * (ks[0] * Sxy + ks[2] * Syz)) +
             ((g[1] + k2) * (g[0] + k2) - 2.0 * k2 * k2) * Sxx + ((g[1] + k2) * (g[2] + k2) - 2.0 * k2 * k2) * Szz +
             2.0 * (g[1] + k2) * ks[0] * ks[2] * Sxz;
    out[4] = 2.0 * (g[1] - k2) * (g[2] - k2) * Syz + (g[0] + k2) * conj(ks[1]) * conj(ks[2]) * Sxx +
             (g[1] - k2) * conj(ks[2]) * (conj(ks[1]) * Syy + 2.0 * ks[0] * Sxy) +
             (g[2] - k2) * conj(ks[1]) * (conj(ks[2]) * Szz + 2.0 * ks[0] * Sxz);
    out[5] = (g[2] - k2) * ((g[2] - k2) * Szz + 2.0 * ks[2] * (ks[0] * Sxz + ks[1] * Syz)) +
             ((g[2] + k2) * (g[0] + k2) - 2.0 * k2 * k2) * Sxx + ((g[2] + k2) * (g[1] + k2) - 2.0 * k2 * k2) * Syy +
             2.0 * (g[2] + k2) * ks[0] * ks[1] * Sxy;
}

/* projectFTtensor: gevolution.hpp:693-787 */
void orc_project_tensor(int N, const double *SijFT_, double *hijFT_)
{
    const cplx *S = (const cplx *)SijFT_;
    cplx *h = (cplx *)hijFT_;
    const int64_t m = (int64_t)(N / 2 + 1) * N * N;
    ktab t = make_ktab(N);
    KLOOP(N)
    {
        int64_t i = KIDX(N, kx, ky, kz);
        double g[3] = {t.k2[kx], t.k2[ky], t.k2[kz]};
        cplx ks[3] = {t.ks[kx], t.ks[ky], t.ks[kz]};
        double k2 = g[0] + g[1] + g[2];
        cplx s[6], o[6];
        for (int c = 0; c < 6; c++) s[c] = S[c * m + i];
        if (k2 > 0) {
            double k6 = k2 * k2 * k2 * N;
            tt_numerators(g, ks, k2, s, o);
            for (int c = 0; c < 6; c++) h[c * m + i] = o[c] / k6;
        } else {
            for (int c = 0; c < 6; c++) h[c * m + i] = 0;
        }
    }
    free_ktab(t);
}

/* evolveFTtensor: gevolution.hpp:537-674 */
void orc_evolve_tensor(int N, double *SijFT_, double *hijFT_, double *hijprimeFT_,
                       double hubble, double dtau, double dtau_old)
{
    cplx *S = (cplx *)SijFT_, *h = (cplx *)hijFT_, *hp = (cplx *)hijprimeFT_;
    const int64_t m = (int64_t)(N / 2 + 1) * N * N;
    ktab t = make_ktab(N);
    double dm = 0.5 * (dtau_old + dtau);
    double opd = 1.0 + hubble * dm, omd = 1.0 - hubble * dm;
    KLOOP(N)
    {
        int64_t i = KIDX(N, kx, ky, kz);
        double g[3] = {t.k2[kx], t.k2[ky], t.k2[kz]};
        cplx ks[3] = {t.ks[kx], t.ks[ky], t.ks[kz]};
        double k2 = g[0] + g[1] + g[2];
        double k4 = k2 * k2 * N;
        cplx s[6], o[6];
        for (int c = 0; c < 6; c++) s[c] = S[c * m + i];
        if (k2 * dm * dm < 1.0) {
            for (int c = 0; c < 6; c++) h[c * m + i] += hp[c * m + i] * dtau_old;
            if (k2 > 0) {
                tt_numerators(g, ks, k2, s, o);
                for (int c = 0; c < 6; c++)
                    hp[c * m + i] = (omd * hp[c * m + i] + (o[c] / k4 - k2 * h[c * m + i]) * dm) / opd;
            } else {
                cplx tr = s[0] + s[3] + s[5];
                S[0 * m + i] -= tr / 3.0;
                S[3 * m + i] -= tr / 3.0;
                S[5 * m + i] -= tr / 3.0;
                for (int c = 0; c < 6; c++)
                    hp[c * m + i] = (omd * hp[c * m + i] + 2.0 * S[c * m + i] * dm / N) / opd;
            }
        } else {
            tt_numerators(g, ks, k2, s, o);
            for (int c = 0; c < 6; c++) {
                hp[c * m + i] = 0;
                h[c * m + i] = (o[c] * dtau_old / k4 + 2.0 * hubble * h[c * m + i]) / (k2 * dtau_old + 2.0 * hubble);
            }
        }
    }
    free_ktab(t);
}

/* ------------------------------------------------------------------------- */
/* geodesic kick and drift                                                    */
/* ------------------------------------------------------------------------- */

/* update_q with GRADIENT_ORDER == 2: gevolution.hpp:888-1011.  Returns what
 * perfParticles::updateVel reports to main.cu:1232: the square root of the
 * largest per-particle return value v^2/a^2 (:1003), i.e. max |q|/a (the
 * square root is inferred from ic_basic.hpp:2433, which divides the result by a
 * to obtain a velocity from a functor that returns q^2). */
double orc_update_q(int N, int64_t np, const double *pos, double *q, const double *phi,
                    const double *chi, const double *Bi, int nfield, double dtau,
                    double a, double bcoeff)
{
    const double dx = 1.0 / N;
    const int64_t n3 = (int64_t)N * N * N;
    double vmax = 0;
#pragma omp parallel for reduction(max : vmax) schedule(static)
    for (int64_t p = 0; p < np; p++) {
        int c[3]; double d[3];
        locate(N, pos + 3 * p, c, d);
        double *v = q + 3 * p;
        double gradphi[3] = {0, 0, 0}, pgradB[3] = {0, 0, 0};
        double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double e2 = v2 + a * a;
        double phiint = 0;
        for (int k = 0; k < 8; k++) phiint += cicw(d, k) * F(phi, N, c, (k >> 2) & 1, (k >> 1) & 1, k & 1);
        phiint /= e2;
        phiint = 4. * phiint * v2 + (1. + a * a * phiint) * (v2 + e2) / e2;
        for (int i = 0; i < 3; i++) {
            int ei[3] = {i == 0, i == 1, i == 2};
            double g = 0;
            for (int k = 0; k < 8; k++) {
                int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
                g += 0.5 * cicw(d, k) * (F(phi, N, c, bx + ei[0], by + ei[1], bz + ei[2]) -
                                         F(phi, N, c, bx - ei[0], by - ei[1], bz - ei[2]));
            }
            gradphi[i] = g * phiint;
        }
        if (nfield >= 2 && chi) {
            gradphi[0] -= (1 - d[1]) * (1 - d[2]) * (F(chi, N, c, 1, 0, 0) - F(chi, N, c, 0, 0, 0));
            gradphi[1] -= (1 - d[0]) * (1 - d[2]) * (F(chi, N, c, 0, 1, 0) - F(chi, N, c, 0, 0, 0));
            gradphi[2] -= (1 - d[0]) * (1 - d[1]) * (F(chi, N, c, 0, 0, 1) - F(chi, N, c, 0, 0, 0));
            gradphi[0] -= d[1] * (1 - d[2]) * (F(chi, N, c, 1, 1, 0) - F(chi, N, c, 0, 1, 0));
            gradphi[1] -= d[0] * (1 - d[2]) * (F(chi, N, c, 1, 1, 0) - F(chi, N, c, 1, 0, 0));
            gradphi[2] -= d[0] * (1 - d[1]) * (F(chi, N, c, 1, 0, 1) - F(chi, N, c, 1, 0, 0));
            gradphi[0] -= (1 - d[1]) * d[2] * (F(chi, N, c, 1, 0, 1) - F(chi, N, c, 0, 0, 1));
            gradphi[1] -= (1 - d[0]) * d[2] * (F(chi, N, c, 0, 1, 1) - F(chi, N, c, 0, 0, 1));
            gradphi[2] -= (1 - d[0]) * d[1] * (F(chi, N, c, 0, 1, 1) - F(chi, N, c, 0, 1, 0));
            gradphi[0] -= d[1] * d[2] * (F(chi, N, c, 1, 1, 1) - F(chi, N, c, 0, 1, 1));
            gradphi[1] -= d[0] * d[2] * (F(chi, N, c, 1, 1, 1) - F(chi, N, c, 1, 0, 1));
            gradphi[2] -= d[0] * d[1] * (F(chi, N, c, 1, 1, 1) - F(chi, N, c, 1, 1, 0));
        }
        e2 = sqrt(e2);
        if (nfield >= 3 && Bi) {
            const double *B0 = Bi, *B1 = Bi + n3, *B2 = Bi + 2 * n3;
            /* gevolution.hpp:970-989 */
            pgradB[0] = ((1 - d[2]) * (F(B1, N, c, 1, 0, 0) - F(B1, N, c, 0, 0, 0)) + d[2] * (F(B1, N, c, 1, 0, 1) - F(B1, N, c, 0, 0, 1))) * v[1];
            pgradB[0] += ((1 - d[1]) * (F(B2, N, c, 1, 0, 0) - F(B2, N, c, 0, 0, 0)) + d[1] * (F(B2, N, c, 1, 1, 0) - F(B2, N, c, 0, 1, 0))) * v[2];
            pgradB[0] += (1 - d[1]) * (1 - d[2]) * ((d[0] - 1) * F(B0, N, c, -1, 0, 0) + (1 - 2 * d[0]) * F(B0, N, c, 0, 0, 0) + d[0] * F(B0, N, c, 1, 0, 0)) * v[0];
            pgradB[0] += d[1] * (1 - d[2]) * ((d[0] - 1) * F(B0, N, c, -1, 1, 0) + (1 - 2 * d[0]) * F(B0, N, c, 0, 1, 0) + d[0] * F(B0, N, c, 1, 1, 0)) * v[0];
            pgradB[0] += (1 - d[1]) * d[2] * ((d[0] - 1) * F(B0, N, c, -1, 0, 1) + (1 - 2 * d[0]) * F(B0, N, c, 0, 0, 1) + d[0] * F(B0, N, c, 1, 0, 1)) * v[0];
            pgradB[0] += d[1] * d[2] * ((d[0] - 1) * F(B0, N, c, -1, 1, 1) + (1 - 2 * d[0]) * F(B0, N, c, 0, 1, 1) + d[0] * F(B0, N, c, 1, 1, 1)) * v[0];

            pgradB[1] = ((1 - d[0]) * (F(B2, N, c, 0, 1, 0) - F(B2, N, c, 0, 0, 0)) + d[0] * (F(B2, N, c, 1, 1, 0) - F(B2, N, c, 1, 0, 0))) * v[2];
            pgradB[1] += ((1 - d[2]) * (F(B0, N, c, 0, 1, 0) - F(B0, N, c, 0, 0, 0)) + d[2] * (F(B0, N, c, 0, 1, 1) - F(B0, N, c, 0, 0, 1))) * v[0];
            pgradB[1] += (1 - d[0]) * (1 - d[2]) * ((d[1] - 1) * F(B1, N, c, 0, -1, 0) + (1 - 2 * d[1]) * F(B1, N, c, 0, 0, 0) + d[1] * F(B1, N, c, 0, 1, 0)) * v[1];
            pgradB[1] += d[0] * (1 - d[2]) * ((d[1] - 1) * F(B1, N, c, 1, -1, 0) + (1 - 2 * d[1]) * F(B1, N, c, 1, 0, 0) + d[1] * F(B1, N, c, 1, 1, 0)) * v[1];
            pgradB[1] += (1 - d[0]) * d[2] * ((d[1] - 1) * F(B1, N, c, 0, -1, 1) + (1 - 2 * d[1]) * F(B1, N, c, 0, 0, 1) + d[1] * F(B1, N, c, 0, 1, 1)) * v[1];
            pgradB[1] += d[0] * d[2] * ((d[1] - 1) * F(B1, N, c, 1, -1, 1) + (1 - 2 * d[1]) * F(B1, N, c, 1, 0, 1) + d[1] * F(B1, N, c, 1, 1, 1)) * v[1];

            pgradB[2] = ((1 - d[1]) * (F(B0, N, c, 0, 0, 1) - F(B0, N, c, 0, 0, 0)) + d[1] * (F(B0, N, c, 0, 1, 1) - F(B0, N, c, 0, 1, 0))) * v[0];
            pgradB[2] += ((1 - d[0]) * (F(B1, N, c, 0, 0, 1) - F(B1, N, c, 0, 0, 0)) + d[0] * (F(B1, N, c, 1, 0, 1) - F(B1, N, c, 1, 0, 0))) * v[1];
            pgradB[2] += (1 - d[0]) * (1 - d[1]) * ((d[2] - 1) * F(B2, N, c, 0, 0, -1) + (1 - 2 * d[2]) * F(B2, N, c, 0, 0, 0) + d[2] * F(B2, N, c, 0, 0, 1)) * v[2];
            pgradB[2] += d[0] * (1 - d[1]) * ((d[2] - 1) * F(B2, N, c, 1, 0, -1) + (1 - 2 * d[2]) * F(B2, N, c, 1, 0, 0) + d[2] * F(B2, N, c, 1, 0, 1)) * v[2];
            pgradB[2] += (1 - d[0]) * d[1] * ((d[2] - 1) * F(B2, N, c, 0, 1, -1) + (1 - 2 * d[2]) * F(B2, N, c, 0, 1, 0) + d[2] * F(B2, N, c, 0, 1, 1)) * v[2];
            pgradB[2] += d[0] * d[1] * ((d[2] - 1) * F(B2, N, c, 1, 1, -1) + (1 - 2 * d[2]) * F(B2, N, c, 1, 1, 0) + d[2] * F(B2, N, c, 1, 1, 1)) * v[2];

            for (int i = 0; i < 3; i++) gradphi[i] += pgradB[i] / bcoeff / e2;
        }
        v2 = 0;
        for (int i = 0; i < 3; i++) {
            v[i] -= dtau * e2 * gradphi[i] / dx;
            v2 += v[i] * v[i];
        }
        double r = v2 / a / a;
        if (r > vmax) vmax = r;
    }
    return sqrt(vmax);
}

/* update_q_Newton: gevolution.hpp:1051-1118 (GRADIENT_ORDER 2, nfield 1):
 * q -= dtau * a * grad psi / dx; returns max q^2 / a^2 over the particles */
double orc_update_q_newton(int N, int64_t np, const double *pos, double *q, const double *psi, double dtau,
                           double a)
{
    const double dx = 1.0 / N;
    double vmax = 0;
#pragma omp parallel for reduction(max : vmax) schedule(static)
    for (int64_t p = 0; p < np; p++) {
        int c[3]; double d[3];
        locate(N, pos + 3 * p, c, d);
        double *v = q + 3 * p;
        double v2 = 0;
        for (int i = 0; i < 3; i++) {
            int ei[3] = {i == 0, i == 1, i == 2};
            double g = 0;
            for (int k = 0; k < 8; k++) {
                int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
                g += 0.5 * cicw(d, k) * (F(psi, N, c, bx + ei[0], by + ei[1], bz + ei[2]) -
                                         F(psi, N, c, bx - ei[0], by - ei[1], bz - ei[2]));
            }
            v[i] -= dtau * a * g / dx;
            v2 += v[i] * v[i];
        }
        if (v2 / a / a > vmax) vmax = v2 / a / a;
    }
    return vmax;
}

/* initialize_q_ic_basic: ic_basic.hpp:133-166 with one field (nfield = 1):
 * q = -coeff grad phi / dx, the gradient from the cell's edge differences with
 * bilinear weights.  Restated from the source; not pinned to a build of the
 * reference (ic_basic.hpp needs more of LATfield2 than the CPU stand-in has). */
void orc_initialize_q(int N, int64_t np, const double *pos, double *q, const double *phi, double coeff)
{
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < np; p++) {
        int c[3]; double d[3];
        locate(N, pos + 3 * p, c, d);
        double g[3];
        g[0] = (1. - d[1]) * (1. - d[2]) * (F(phi, N, c, 1, 0, 0) - F(phi, N, c, 0, 0, 0));
        g[1] = (1. - d[0]) * (1. - d[2]) * (F(phi, N, c, 0, 1, 0) - F(phi, N, c, 0, 0, 0));
        g[2] = (1. - d[0]) * (1. - d[1]) * (F(phi, N, c, 0, 0, 1) - F(phi, N, c, 0, 0, 0));
        g[0] += d[1] * (1. - d[2]) * (F(phi, N, c, 1, 1, 0) - F(phi, N, c, 0, 1, 0));
        g[1] += d[0] * (1. - d[2]) * (F(phi, N, c, 1, 1, 0) - F(phi, N, c, 1, 0, 0));
        g[2] += d[0] * (1. - d[1]) * (F(phi, N, c, 1, 0, 1) - F(phi, N, c, 1, 0, 0));
        g[0] += (1. - d[1]) * d[2] * (F(phi, N, c, 1, 0, 1) - F(phi, N, c, 0, 0, 1));
        g[1] += (1. - d[0]) * d[2] * (F(phi, N, c, 0, 1, 1) - F(phi, N, c, 0, 0, 1));
        g[2] += (1. - d[0]) * d[1] * (F(phi, N, c, 0, 1, 1) - F(phi, N, c, 0, 1, 0));
        g[0] += d[1] * d[2] * (F(phi, N, c, 1, 1, 1) - F(phi, N, c, 0, 1, 1));
        g[1] += d[0] * d[2] * (F(phi, N, c, 1, 1, 1) - F(phi, N, c, 1, 0, 1));
        g[2] += d[0] * d[1] * (F(phi, N, c, 1, 1, 1) - F(phi, N, c, 1, 1, 0));
        for (int k = 0; k < 3; k++) q[3 * p + k] = -g[k] * N * coeff;
    }
}

/* update_pos_Newton: gevolution.hpp:1270-1273, pos += dtau q / a (positions
 * left unwrapped: the differentiable run keeps continuous coordinates) */
void orc_update_pos_newton(int64_t np, double *pos, const double *q, double dtau, double a)
{
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < 3 * np; p++) pos[p] += dtau * q[p] / a;
}

/* update_pos: gevolution.hpp:1162-1232; positions wrapped into [0,1) as
 * LATfield2's moveParticles re-bins them on the periodic lattice. */
void orc_update_pos(int N, int64_t np, double *pos, const double *q, const double *phi,
                    const double *chi, const double *Bi, int nfield, double dtau,
                    double a, double bcoeff)
{
    const int64_t n3 = (int64_t)N * N * N;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < np; p++) {
        int c[3]; double d[3];
        double *x = pos + 3 * p;
        locate(N, x, c, d);
        const double *v = q + 3 * p;
        double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double e2 = v2 + a * a;
        double ph = 0, ch = 0;
        if (nfield >= 1)
            for (int k = 0; k < 8; k++) ph += cicw(d, k) * F(phi, N, c, (k >> 2) & 1, (k >> 1) & 1, k & 1);
        if (nfield >= 2)
            for (int k = 0; k < 8; k++) ch += cicw(d, k) * F(chi, N, c, (k >> 2) & 1, (k >> 1) & 1, k & 1);
        v2 = (1. + (3. - v2 / e2) * ph - ch) / sqrt(e2);
        double vel[3] = {v[0] * v2, v[1] * v2, v[2] * v2};
        if (nfield >= 3) {
            const double *B0 = Bi, *B1 = Bi + n3, *B2 = Bi + 2 * n3;
            double b[3];
            b[0] = F(B0, N, c, 0, 0, 0) * (1 - d[1]) * (1 - d[2]) + F(B0, N, c, 0, 1, 0) * d[1] * (1 - d[2]) +
                   F(B0, N, c, 0, 0, 1) * (1 - d[1]) * d[2] + F(B0, N, c, 0, 1, 1) * d[1] * d[2];
            b[1] = F(B1, N, c, 0, 0, 0) * (1 - d[0]) * (1 - d[2]) + F(B1, N, c, 1, 0, 0) * d[0] * (1 - d[2]) +
                   F(B1, N, c, 0, 0, 1) * (1 - d[0]) * d[2] + F(B1, N, c, 1, 0, 1) * d[0] * d[2];
            b[2] = F(B2, N, c, 0, 0, 0) * (1 - d[0]) * (1 - d[1]) + F(B2, N, c, 1, 0, 0) * d[0] * (1 - d[1]) +
                   F(B2, N, c, 0, 1, 0) * (1 - d[0]) * d[1] + F(B2, N, c, 1, 1, 0) * d[0] * d[1];
            for (int l = 0; l < 3; l++) x[l] += dtau * (vel[l] + b[l] / bcoeff);
        } else {
            for (int l = 0; l < 3; l++) x[l] += dtau * vel[l];
        }
        for (int l = 0; l < 3; l++) x[l] -= floor(x[l]);
    }
}

/* ------------------------------------------------------------------------- */
/* background: background.hpp:200-244, :268-291                               */
/* ------------------------------------------------------------------------- */

double orc_hconf(double a, double fourpiG, const orc_cosmo *c)
{
    return sqrt((2. * fourpiG / 3.) * ((c->Omega_m / a) + (c->Omega_Lambda * a * a) + (c->Omega_rad / a / a)));
}

void orc_rk4bg(double *a_, double fourpiG, const orc_cosmo *c, double dtau)
{
    double a = *a_;
    double k1a = a * orc_hconf(a, fourpiG, c);
    double k2a = (a + k1a * dtau / 2.) * orc_hconf(a + k1a * dtau / 2., fourpiG, c);
    double k3a = (a + k2a * dtau / 2.) * orc_hconf(a + k2a * dtau / 2., fourpiG, c);
    double k4a = (a + k3a * dtau) * orc_hconf(a + k3a * dtau, fourpiG, c);
    *a_ = a + dtau * (k1a + 2. * k2a + 2. * k3a + k4a) / 6.;
}

static double ph_integrand(double s, const orc_cosmo *c) { return 2. / (s * orc_hconf(s * s, 1., c)); }

static double simpson_adapt(double lo, double hi, double flo, double fmid, double fhi, double whole,
                            double tol, int depth, const orc_cosmo *c)
{
    double mid = 0.5 * (lo + hi);
    double lm = 0.5 * (lo + mid), rm = 0.5 * (mid + hi);
    double flm = ph_integrand(lm, c), frm = ph_integrand(rm, c);
    double left = (mid - lo) / 6. * (flo + 4 * flm + fmid), right = (hi - mid) / 6. * (fmid + 4 * frm + fhi);
    if (depth <= 0 || fabs(left + right - whole) <= 15 * tol) return left + right + (left + right - whole) / 15.;
    return simpson_adapt(lo, mid, flo, flm, fmid, left, tol / 2, depth - 1, c) +
           simpson_adapt(mid, hi, fmid, frm, fhi, right, tol / 2, depth - 1, c);
}

/* particleHorizon: integral of 2/(sqrt(a) Hconf(a,1)) d sqrt(a) from sqrt(a)*1e-7
 * (the reference uses GSL QNG with rel. tolerance 1e-7; this is adaptive Simpson). */
double orc_particle_horizon(double a, double fourpiG, const orc_cosmo *c)
{
    double lo = sqrt(a) * 1.0e-7, hi = sqrt(a);
    double flo = ph_integrand(lo, c), fhi = ph_integrand(hi, c), fmid = ph_integrand(0.5 * (lo + hi), c);
    double whole = (hi - lo) / 6. * (flo + 4 * fmid + fhi);
    double r = simpson_adapt(lo, hi, flo, fmid, fhi, whole, 1e-13, 60, c);
    return r / sqrt(fourpiG);
}

/* ------------------------------------------------------------------------- */
/* power spectrum: extractCrossSpectrum, KTYPE_LINEAR, deconvolve (tools.hpp:65-314)
 * kmax <= 0 selects the reference's kmax = sqrt(3) * pi * N.                 */
/* ------------------------------------------------------------------------- */

void orc_power_spectrum(int N, const double *fieldFT_, int numbins, double *kbin,
                        double *power, double *kscatter, double *pscatter,
                        int *occupation, double kmax)
{
    const cplx *f = (const cplx *)fieldFT_;
    double *typek2 = malloc(sizeof(double) * N), *sinc = malloc(sizeof(double) * N);
    for (int i = 0; i <= N / 2; i++) { typek2[i] = 2. * M_PI * i; typek2[i] *= typek2[i]; }
    for (int i = N / 2 + 1; i < N; i++) { typek2[i] = 2. * M_PI * (N - i); typek2[i] *= typek2[i]; }
    sinc[0] = 1.;
    for (int i = 1; i <= N / 2; i++) sinc[i] = sin(M_PI * (float)i / (float)N) * (float)N / (M_PI * (float)i);
    for (int i = N / 2 + 1; i < N; i++) sinc[i] = sinc[N - i];
    if (kmax <= 0) kmax = sqrt(3. * typek2[N / 2]);
    double *acc = calloc(4 * (size_t)numbins, sizeof(double));
    long *occ = calloc(numbins, sizeof(long));
    for (int kz = 0; kz < N; kz++)
        for (int ky = 0; ky < N; ky++)
            for (int kx = 0; kx <= N / 2; kx++) {
                if (kx == 0 && ky == 0 && kz == 0) continue;
                int weight = (kx == 0 || (kx == N / 2 && N % 2 == 0)) ? 1 : 2;
                double k2 = typek2[kx] + typek2[ky] + typek2[kz];
                double s = sinc[kx] * sinc[ky] * sinc[kz];
                s *= s;
                cplx v = f[KIDX(N, kx, ky, kz)];
                double p = creal(v) * creal(v) + cimag(v) * cimag(v);
                double sk = sqrt(k2);
                int bin = (int)floor((double)numbins * sk / kmax);
                if (bin < numbins) {
                    acc[bin] += weight * sk;
                    acc[numbins + bin] += weight * k2;
                    acc[2 * numbins + bin] += weight * p * k2 * sk / s;
                    acc[3 * numbins + bin] += weight * p * p * k2 * k2 * k2 / s / s;
                    occ[bin] += weight;
                }
            }
    for (int i = 0; i < numbins; i++) {
        occupation[i] = (int)occ[i];
        if (occ[i] > 0) {
            kbin[i] = acc[i];
            kscatter[i] = sqrt(acc[numbins + i] * occ[i] - kbin[i] * kbin[i]) / occ[i];
            if (!isfinite(kscatter[i])) kscatter[i] = 0;
            kbin[i] /= occ[i];
            power[i] = acc[2 * numbins + i] / occ[i];
            pscatter[i] = sqrt(acc[3 * numbins + i] / occ[i] - power[i] * power[i]);
            if (!isfinite(pscatter[i])) pscatter[i] = 0;
        } else {
            kbin[i] = power[i] = kscatter[i] = pscatter[i] = 0;
        }
    }
    free(acc); free(occ); free(typek2); free(sinc);
}

/* ------------------------------------------------------------------------- */
/* lightcone crossing                                                         */
/* ------------------------------------------------------------------------- */

/* The reference keeps at most MAX_INTERSECTS = 12 periodic images
 * (metadata.hpp:35-37) and warns that data is lost beyond that (tools.hpp:877-882);
 * one domain covering the whole box needs more for shells near a box length,
 * so up to 64 are kept here (and in the CUDA library). */
#define ORC_MAX_INTERSECTS 64
#define ORC_IDCHECK_ZONE 0.05      /* metadata.hpp:38-40 */
#define ORC_GADGET_VEL 3.335640952e-6  /* GADGET_VELOCITY_CONVERSION, metadata.hpp */

/* findIntersectingLightcones: tools.hpp:637-886.  domain = {x0,y0,z0,x1,y1,z1}. */
int orc_find_intersecting(const double *lcv, const double *dir, double opening, double outer, double inner,
                          const double *domain, double *vertex_out)
{
    int range = (int)ceil(outer) + 1, n = 0;
    double cen[3], rdom = 0;
    for (int i = 0; i < 3; i++) {
        cen[i] = 0.5 * domain[i] + 0.5 * domain[i + 3];
        rdom += (domain[i + 3] - domain[i]) * (domain[i + 3] - domain[i]);
    }
    rdom = 0.5 * sqrt(rdom);
    for (int u = -range; u <= range; u++)
        for (int v = -range; v <= range; v++)
            for (int w = -range; w <= range; w++) {
                double vx[3] = {lcv[0] + u, lcv[1] + v, lcv[2] + w};
                /* distance from the vertex to the domain box */
                double dd = 0;
                for (int i = 0; i < 3; i++) {
                    double e = 0;
                    if (vx[i] < domain[i]) e = domain[i] - vx[i];
                    else if (vx[i] > domain[i + 3]) e = vx[i] - domain[i + 3];
                    dd += e * e;
                }
                if (sqrt(dd) > outer) continue;
                /* domain entirely inside the inner sphere */
                int inside = 1;
                for (int c = 0; c < 8 && inside; c++) {
                    double cc[3] = {domain[(c & 1) ? 3 : 0], domain[(c & 2) ? 4 : 1], domain[(c & 4) ? 5 : 2]};
                    double r = sqrt((cc[0] - vx[0]) * (cc[0] - vx[0]) + (cc[1] - vx[1]) * (cc[1] - vx[1]) + (cc[2] - vx[2]) * (cc[2] - vx[2]));
                    if (!(r < inner)) inside = 0;
                }
                if (inside) continue;
                double dist = sqrt((cen[0] - vx[0]) * (cen[0] - vx[0]) + (cen[1] - vx[1]) * (cen[1] - vx[1]) + (cen[2] - vx[2]) * (cen[2] - vx[2]));
                int take = 0;
                if (dist <= rdom) take = 1;
                else {
                    double cosang = ((cen[0] - vx[0]) * dir[0] + (cen[1] - vx[1]) * dir[1] + (cen[2] - vx[2]) * dir[2]) / dist;
                    if (cosang >= opening) take = 1;
                    else if (dist > outer && acos(cosang) - acos(opening) <= acos((outer * outer + dist * dist - rdom * rdom) / (2. * outer * dist))) take = 1;
                    else if (dist <= outer && acos(cosang) - acos(opening) <= asin(rdom / dist)) take = 1;
                }
                if (take) {
                    if (n < ORC_MAX_INTERSECTS)
                        for (int i = 0; i < 3; i++) vertex_out[3 * n + i] = vx[i];
                    n++;
                }
            }
    return n < ORC_MAX_INTERSECTS ? n : ORC_MAX_INTERSECTS;
}

/* Selection and interpolation of lightcone particles for one shell and one
 * cycle: buffer_tracer_particles (Particles_gevolution.hpp:1381-1466) with
 * bufferTracerParticle under EXACT_OUTPUT_REDSHIFTS (:500-560), for the whole
 * box as one domain (output.hpp:1174-1186).  Returns the number written; the ID
 * backlog de-duplication is the caller's (it needs the previous cycle). */
int64_t orc_lightcone_select(int N, int64_t np, const double *pos, const double *q, const int64_t *id,
                             const double *phi, const orc_lightcone *lc, double tau, double dtau,
                             double dtau_old, double a, double dadtau, int64_t max_out, float *out_pos,
                             float *out_vel, int64_t *out_id, double boxsize)
{
    (void)id;
    double dist = lc->dist_hi;                 /* caller passes d - tau in dist_hi */
    double inner = dist - 0.5 * dtau;
    double outer = dist + (0.5 + ORC_IDCHECK_ZONE) * dtau_old;
    double domain[6] = {-0.5 / N, -0.5 / N, -0.5 / N, (N + 0.5) / N, (N + 0.5) / N, (N + 0.5) / N};
    double vtx[ORC_MAX_INTERSECTS * 3];
    int nv = orc_find_intersecting(lc->vertex, lc->direction, lc->opening, outer, inner, domain, vtx);
    const double dx = 1.0 / N;
    int64_t n = 0;
    (void)tau;
    for (int64_t p = 0; p < np; p++) {
        const double *x = pos + 3 * p, *v = q + 3 * p;
        for (int k = 0; k < nv; k++) {
            const double *V = vtx + 3 * k;
            double d = sqrt((x[0] - V[0]) * (x[0] - V[0]) + (x[1] - V[1]) * (x[1] - V[1]) + (x[2] - V[2]) * (x[2] - V[2]));
            if (!(d >= inner && d < outer)) continue;
            if (!(lc->opening == -1. || ((x[0] - V[0]) * lc->direction[0] + (x[1] - V[1]) * lc->direction[1] + (x[2] - V[2]) * lc->direction[2]) / d > lc->opening)) continue;
            double vlos = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + a * (a + dtau_old * dadtau));
            vlos = (v[0] * (x[0] - V[0]) + v[1] * (x[1] - V[1]) + v[2] * (x[2] - V[2])) / d / vlos;
            double dtau_pos = (dist - d) / (1. + vlos);
            double dtau_vel = dtau_pos + 0.5 * dtau_old;
            double at = a + dtau_pos * dadtau;
            /* bufferTracerParticle, EXACT_OUTPUT_REDSHIFTS branch */
            int c[3]; double fr[3];
            locate(N, x, c, fr);
            double phip = 0, g[3] = {0, 0, 0};
            if (phi) {
                for (int kk = 0; kk < 8; kk++) phip += cicw(fr, kk) * F(phi, N, c, (kk >> 2) & 1, (kk >> 1) & 1, kk & 1);
                g[0] = (1 - fr[1]) * (1 - fr[2]) * (F(phi, N, c, 1, 0, 0) - F(phi, N, c, 0, 0, 0)) + fr[1] * (1 - fr[2]) * (F(phi, N, c, 1, 1, 0) - F(phi, N, c, 0, 1, 0)) +
                       (1 - fr[1]) * fr[2] * (F(phi, N, c, 1, 0, 1) - F(phi, N, c, 0, 0, 1)) + fr[1] * fr[2] * (F(phi, N, c, 1, 1, 1) - F(phi, N, c, 0, 1, 1));
                g[1] = (1 - fr[0]) * (1 - fr[2]) * (F(phi, N, c, 0, 1, 0) - F(phi, N, c, 0, 0, 0)) + fr[0] * (1 - fr[2]) * (F(phi, N, c, 1, 1, 0) - F(phi, N, c, 1, 0, 0)) +
                       (1 - fr[0]) * fr[2] * (F(phi, N, c, 0, 1, 1) - F(phi, N, c, 0, 0, 1)) + fr[0] * fr[2] * (F(phi, N, c, 1, 1, 1) - F(phi, N, c, 1, 0, 1));
                g[2] = (1 - fr[0]) * (1 - fr[1]) * (F(phi, N, c, 0, 0, 1) - F(phi, N, c, 0, 0, 0)) + fr[0] * (1 - fr[1]) * (F(phi, N, c, 1, 0, 1) - F(phi, N, c, 1, 0, 0)) +
                       (1 - fr[0]) * fr[1] * (F(phi, N, c, 0, 1, 1) - F(phi, N, c, 0, 1, 0)) + fr[0] * fr[1] * (F(phi, N, c, 1, 1, 1) - F(phi, N, c, 1, 1, 0));
            }
            double q2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            double f1 = q2 + at * at, f2 = sqrt(f1), f0 = q2 + f1;
            f1 = 1. + (4. - f0 / f1) * phip;
            double rescale_vel = 1. / sqrt(at) / ORC_GADGET_VEL;
            if (n < max_out) {
                for (int i = 0; i < 3; i++) {
                    float off = (float)(lc->vertex[i] - V[i]);
                    out_pos[3 * n + i] = ((float)(x[i] + dtau_pos * v[i] * f1 / f2) + off) * (float)boxsize;
                    out_vel[3 * n + i] = (float)((v[i] - dtau_vel * f0 * g[i] / dx / f2) * rescale_vel) / (float)at;
                }
                out_id[n] = id ? id[p] : p;
            }
            n++;
            break;
        }
    }
    return n;
}

/* ------------------------------------------------------------------------- */
/* one PM cycle, GR weak-field gauge, CDM only, elliptic B (main.cu:608-1317) */
/* ------------------------------------------------------------------------- */

void orc_step(const orc_sim *sim, orc_state *st, int64_t np, double *pos, double *q,
              double *phi, double *chi, double *Bi)
{
    const int N = sim->N;
    const int64_t n3 = (int64_t)N * N * N, nk = (int64_t)(N / 2 + 1) * N * N;
    const double dx = 1.0 / N;
    double a = st->a;
    double *source = calloc(n3, sizeof(double));
    double *Sij = calloc(6 * n3, sizeof(double));
    double *FT = malloc(sizeof(double) * 2 * 6 * nk);

    /* T00 and Tij with the previous phi (main.cu:623, :756) */
    orc_project_T00(N, np, pos, q, sim->mass, phi, a, 1.0, source);
    orc_project_Tij(N, np, pos, q, sim->mass, phi, a, 1.0, Sij);

    /* phi (main.cu:719-809) */
    if (st->dtau_old > 0.) {
        double H = orc_hconf(a, sim->fourpiG, &sim->cosmo);
        double sum = orc_prepare_T00(N, phi, chi, source, sim->cosmo.Omega_m, 3. * H * dx * dx / st->dtau_old,
                                     sim->fourpiG * dx * dx / a, 3. * H * H * dx * dx, source);
        st->T00hom = sum / (double)n3;
        orc_r2c(N, source, FT);
        orc_solve_poisson(N, FT, FT, 1. / (dx * dx), 3. * H / st->dtau_old);
        st->phi_hom = FT[0];
        orc_c2r(N, FT, phi);
    }

    /* chi (main.cu:820-903) */
    orc_prepare_Tij(N, phi, Sij, 2. * sim->fourpiG * dx * dx / a, Sij);
    for (int c = 0; c < 6; c++) orc_r2c(N, Sij + c * n3, FT + 2 * c * nk);
    double *chiFT = malloc(sizeof(double) * 2 * nk);
    orc_project_scalar(N, FT, chiFT, 0);
    orc_c2r(N, chiFT, chi);
    free(chiFT);

    /* B, elliptic (main.cu:836-955) with the new phi */
    if (sim->with_B) {
        memset(Bi, 0, sizeof(double) * 3 * n3);
        orc_project_T0i(N, np, pos, q, sim->mass, phi, 1.0, Bi);
        for (int c = 0; c < 3; c++) orc_r2c(N, Bi + c * n3, FT + 2 * c * nk);
        orc_project_vector(N, FT, FT, sim->fourpiG * dx * dx, 0.);
        for (int c = 0; c < 3; c++) orc_c2r(N, FT + 2 * c * nk, Bi + c * n3);
    }

    /* kick, half background step, drift, half background step (main.cu:1225-1283) */
    int nk_field = (1. / a < sim->z_relax + 1.) ? 3 : 2;
    double mv = orc_update_q(N, np, pos, q, phi, chi, Bi, nk_field, 0.5 * (st->dtau + st->dtau_old), a, a * a * N);
    orc_rk4bg(&a, sim->fourpiG, &sim->cosmo, 0.5 * st->dtau);
    int nd_field = (1. / a < sim->z_relax + 1.) ? 3 : 0;
    orc_update_pos(N, np, pos, q, phi, chi, Bi, nd_field, st->dtau, a, a * a * N);
    orc_rk4bg(&a, sim->fourpiG, &sim->cosmo, 0.5 * st->dtau);
    st->maxvel = mv / sqrt(mv * mv + 1.0);

    /* step control (main.cu:1286-1310) */
    st->tau += st->dtau;
    st->dtau_old = st->dtau;
    double H = orc_hconf(a, sim->fourpiG, &sim->cosmo);
    st->dtau = (sim->Cf * dx < sim->steplimit / H) ? sim->Cf * dx : sim->steplimit / H;
    st->a = a;
    st->cycle++;
    free(source); free(Sij); free(FT);
}
