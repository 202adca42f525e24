/*
 * oracle.h -- FP64 CPU restatement of gevolution-2.0's per-step particle-mesh cycle.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path may link or call this
 * library; it is the checker that the CUDA implementation is compared against
 * (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg only).
 *
 * Every function cites the reference function it restates (file:line inside the
 * gevolution-2.0 tree).  The restatement itself is pinned against the
 * reference's own code compiled on the CPU (oracle/_ref, built by
 * oracle/refshim/Makefile from the reference sources where they lie).
 *
 * Conventions shared with the CUDA library (include/gev.h):
 *   - real fields: N^3 doubles, index x + N*(y + N*z), periodic, no halo;
 *   - symmetric tensors: 6 planes (00,01,02,11,12,22); vectors: 3 planes;
 *   - Fourier fields: (N/2+1)*N*N complex, index kx + (N/2+1)*(ky + N*kz),
 *     forward transform exp(-2 pi i k.x/N), both directions unnormalised
 *     (the solvers carry the 1/N^3 and 1/N factors like the reference);
 *   - particles: pos[3*np] in box units [0,1), q[3*np] (momentum per unit mass),
 *     one "part_simple" per particle as in LATfield2's perfParticles.
 */
#ifndef GEV_ORACLE_H
#define GEV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FFT (the reference uses cuFFT/FFTW through LATfield2's PlanFFT) ---- */
void orc_fft1d(int n, double *re_im, int sign);            /* in place, interleaved */
void orc_r2c(int N, const double *in, double *out);         /* out: (N/2+1)N^2 complex */
void orc_c2r(int N, const double *in, double *out);         /* in is not modified */

/* ---- particle-mesh projections (accumulate into the target, like the reference) ---- */
void orc_project_T00(int N, int64_t np, const double *pos, const double *q, double mass,
                     const double *phi, double a, double coeff, double *T00);
void orc_project_Tij(int N, int64_t np, const double *pos, const double *q, double mass,
                     const double *phi, double a, double coeff, double *Tij);
void orc_project_T0i(int N, int64_t np, const double *pos, const double *q, double mass,
                     const double *phi, double coeff, double *T0i);
void orc_project_cic(int N, int64_t np, const double *pos, double mass, double *rho);

/* ---- source preparation ---- */
double orc_prepare_T00(int N, const double *phi, const double *chi, const double *source,
                       double bgmodel, double coeff, double coeff2, double coeff3,
                       double *result);
void orc_prepare_Tij(int N, const double *phi, const double *Tij, double coeff, double *Sij);

/* ---- Fourier-space solvers (complex arrays are interleaved re/im doubles) ---- */
void orc_solve_poisson(int N, const double *srcFT, double *potFT, double coeff, double modif);
void orc_project_scalar(int N, const double *SijFT, double *chiFT, int add);
void orc_project_vector(int N, const double *SiFT, double *BiFT, double coeff, double modif);
void orc_evolve_vector(int N, const double *SijFT, double *BiFT, double a2dtau);
void orc_project_tensor(int N, const double *SijFT, double *hijFT);
void orc_evolve_tensor(int N, double *SijFT, double *hijFT, double *hijprimeFT,
                       double hubble, double dtau, double dtau_old);

/* ---- geodesic kick and drift ---- */
double orc_update_q(int N, int64_t np, const double *pos, double *q, const double *phi,
                    const double *chi, const double *Bi, int nfield, double dtau,
                    double a, double bcoeff);
void orc_update_pos(int N, int64_t np, double *pos, const double *q, const double *phi,
                    const double *chi, const double *Bi, int nfield, double dtau,
                    double a, double bcoeff);

/* ---- Newtonian kick and drift (main.cu's gr_flag == 0 branch) ---- */
double orc_update_q_newton(int N, int64_t np, const double *pos, double *q, const double *psi, double dtau,
                           double a);
void orc_update_pos_newton(int64_t np, double *pos, const double *q, double dtau, double a);

/* ---- initial-condition momenta (ic_basic.hpp:133-166) ---- */
void orc_initialize_q(int N, int64_t np, const double *pos, double *q, const double *phi, double coeff);

/* ---- background (CDM + Lambda + radiation, no ncdm / fluid) ---- */
typedef struct {
    double Omega_m, Omega_Lambda, Omega_rad;
} orc_cosmo;
double orc_hconf(double a, double fourpiG, const orc_cosmo *c);
void orc_rk4bg(double *a, double fourpiG, const orc_cosmo *c, double dtau);
double orc_particle_horizon(double a, double fourpiG, const orc_cosmo *c);

/* ---- validation metric: binned power spectrum ---- */
void orc_power_spectrum(int N, const double *fieldFT, int numbins, double *kbin,
                        double *power, double *kscatter, double *pscatter,
                        int *occupation, double kmax);

/* ---- lightcone crossing (particle selection and interpolation) ---- */
typedef struct {
    double vertex[3];      /* observer position, box units */
    double direction[3];   /* cone axis (unit vector) */
    double opening;        /* cos(half opening angle); -1 for full sky */
    double dist_lo;        /* unused */
    double dist_hi;        /* d - tau: comoving distance of the crossing surface */
} orc_lightcone;
int orc_find_intersecting(const double *lcv, const double *dir, double opening, double outer,
                          double inner, const double *domain, double *vertex_out);
int64_t orc_lightcone_select(int N, int64_t np, const double *pos, const double *q,
                             const int64_t *id, const double *phi, const orc_lightcone *lc,
                             double tau, double dtau, double dtau_old, double a,
                             double dadtau, int64_t max_out, float *out_pos,
                             float *out_vel, int64_t *out_id, double boxsize);

/* ---- one full PM cycle in the reference's order (main.cu:608-1317) ---- */
typedef struct {
    int N;
    double boxsize;        /* Mpc/h */
    double fourpiG;
    double mass;           /* per-particle mass (Omega_m / Np) */
    orc_cosmo cosmo;
    double z_relax;        /* B enters the geodesic below this redshift */
    double Cf, steplimit;
    int with_B;            /* elliptic vector method */
} orc_sim;

typedef struct {
    double a, tau, dtau, dtau_old;
    int cycle;
    double T00hom, phi_hom, maxvel;
} orc_state;

/* fields: phi, chi (N^3), Bi (3 N^3); scratch allocated internally. */
void orc_step(const orc_sim *sim, orc_state *st, int64_t np, double *pos, double *q,
              double *phi, double *chi, double *Bi);

#ifdef __cplusplus
}
#endif
#endif
