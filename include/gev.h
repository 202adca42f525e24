/*
 * gev.h -- C ABI of the B200 (sm_100a) implementation of gevolution-2.0's
 * per-step particle-mesh cycle on one GPU.
 *
 * Plain C types only.  Every function returns a status (GEV_OK = 0); on failure
 * gev_last_error() returns a message.  Host pointers are borrowed for the
 * duration of the call.  A context owns all device memory, is used from one host
 * thread at a time, and orders its work on its own CUDA stream; calls that
 * return scalars synchronise that stream.
 *
 * Layout conventions (the reference's LATfield2 conventions on one rank):
 *   real fields      N^3 values, index x + N*(y + N*z), periodic;
 *   symmetric tensor 6 planes in the order 00,01,02,11,12,22;
 *   vector           3 planes;
 *   Fourier fields   (N/2+1)*N*N complex values, index kx + (N/2+1)*(ky + N*kz),
 *                    forward transform exp(-2 pi i k.x/N), unnormalised;
 *   particles        pos[3n] in box units [0,1), q[3n] momentum per unit mass
 *                    (LATfield2 part_simple pos/vel), id[n].
 *
 * Each entry point names the reference interface it replaces (file:line inside
 * the gevolution-2.0 tree).
 */
#ifndef GEV_B200_H
#define GEV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gev_ctx gev_ctx;

/* status codes */
#define GEV_OK          0
#define GEV_ERR_ARG     1   /* invalid argument (size, pointer, mode) */
#define GEV_ERR_CUDA    2   /* CUDA runtime error */
#define GEV_ERR_STATE   3   /* call out of order (e.g. no particles loaded) */
#define GEV_ERR_DEVICE  4   /* a kernel raised its device error word */
#define GEV_ERR_NOMEM   5   /* device allocation failed */
#define GEV_ERR_CAPACITY 6  /* output buffer too small */
#define GEV_ERR_SIZE    7   /* grid larger than a fixed-size scratch allows */

/* precision modes: FP64 everywhere, or FP32 fields/FFTs with particle
 * positions kept as cell index + FP64 offset and FP64 reductions */
#define GEV_FP64   0
#define GEV_MIXED  1

/* vector methods (metadata.hpp:84-85) */
#define GEV_VECTOR_PARABOLIC 0
#define GEV_VECTOR_ELLIPTIC  1

/* field identifiers for gev_field_get / gev_field_set */
#define GEV_FIELD_PHI     0   /* 1 plane  */
#define GEV_FIELD_CHI     1   /* 1 plane  */
#define GEV_FIELD_SOURCE  2   /* 1 plane: T00 (main.cu "source") */
#define GEV_FIELD_SIJ     3   /* 6 planes: Tij, then Sij */
#define GEV_FIELD_BI      4   /* 3 planes: T0i, then B_i */
#define GEV_FIELD_HIJ_FT  5   /* 6 complex planes: h_ij in Fourier space */
#define GEV_FIELD_HIJP_FT 6   /* 6 complex planes: h_ij' in Fourier space */
#define GEV_FIELD_BI_FT   7   /* 3 complex planes: B_i in Fourier space (parabolic state) */

/* projection selectors for gev_project */
#define GEV_PROJ_T00 1u
#define GEV_PROJ_TIJ 2u
#define GEV_PROJ_T0I 4u
#define GEV_PROJ_CIC 8u
#define GEV_PROJ_T0I_SUMS 16u

typedef struct {
    int32_t N;              /* grid points per side: multiple of 8, N/8 a power of two or 3x one, 16..1024 */
    int32_t precision;      /* GEV_FP64 or GEV_MIXED */
    int64_t capacity;       /* maximum number of particles */
    double boxsize;         /* Mpc/h; used for lightcone output units */
    int32_t vector_method;  /* GEV_VECTOR_ELLIPTIC or GEV_VECTOR_PARABOLIC */
    int32_t tensor;         /* nonzero: keep h_ij / h_ij' state (projectFTtensor / evolveFTtensor) */
    int32_t device;         /* CUDA device ordinal */
    int32_t reserved;
} gev_config;

/* Context life cycle.  Replaces LATfield2's Lattice/Field/PlanFFT set-up in
 * main.cu:298-385 (fields, Fourier fields and FFT plans) and the particle
 * container initialisation of ic_basic.hpp:2206. */
int gev_ctx_create(const gev_config *cfg, gev_ctx **out);
int gev_ctx_destroy(gev_ctx *ctx);
const char *gev_last_error(const gev_ctx *ctx);
const char *gev_version(void);

/* Particles.  set: perfParticles::initialize + addParticle_global +
 * updateRowBuffers (ic_basic.hpp:2206-2211); mass is part_simple_info.mass
 * (ic_basic.hpp:2198-2201).  get: perfParticles::sampleParticles
 * (unit_tests.cu:537).  Positions are wrapped into [0,1). */
int gev_particles_set(gev_ctx *ctx, const double *pos, const double *q, const int64_t *id,
                      int64_t n, double mass);
int gev_particles_get(gev_ctx *ctx, double *pos, double *q, int64_t *id, int64_t capacity,
                      int64_t *n_out);
int gev_particles_count(const gev_ctx *ctx, int64_t *n_out);
/* get followed by set in one call, with both directions of the host link in
 * use at once: copies the current particles to (pos_out, q_out, id_out) as
 * gev_particles_get does, and replaces them by the n_in particles of
 * (pos_in, q_in, id_in) as gev_particles_set does (every array required),
 * chunk by chunk, downloads and uploads on two copy streams.  The input
 * arrays may be the output arrays themselves (each chunk is uploaded after it
 * was downloaded: the state goes out and comes back in); other overlaps of an
 * input with an output array are taken one direction after the other.
 * Returns when both directions are complete.  No reference counterpart: it
 * serves callers that keep the particle state on the host between cycles. */
int gev_particles_exchange(gev_ctx *ctx, double *pos_out, double *q_out, int64_t *id_out, int64_t capacity,
                           int64_t *n_out, const double *pos_in, const double *q_in, const int64_t *id_in,
                           int64_t n_in, double mass);

/* Field transfer in double precision (converted to/from the context precision). */
int gev_field_get(gev_ctx *ctx, int32_t field, double *host);
int gev_field_set(gev_ctx *ctx, int32_t field, const double *host);
int gev_field_components(int32_t field);

/* Particle-mesh projections.  which is a mask of GEV_PROJ_*:
 *   T00: projection_T00_project (gevolution.hpp:1887) + projection_T00_comm
 *        (:1726) into GEV_FIELD_SOURCE, params {a, coeff};
 *   TIJ: projection_Tij_project / _Async (:2999, :3030) + projection_Tij_comm
 *        (:2573-2578) into GEV_FIELD_SIJ, params {a, coeff};
 *   T0I: projection_T0i_project / _Async (:2232, :2242) + projection_T0i_comm
 *        (:2028) into GEV_FIELD_BI, params {coeff};
 *   CIC: scalarProjectionCIC_project (:1902) + comm into GEV_FIELD_SOURCE.
 * use_phi != 0 applies the Bardeen-potential corrections with GEV_FIELD_PHI
 * (the reference's phi != nullptr).  accumulate == 0 overwrites the targets
 * (the reference zeroes them first, main.cu:616, :681, :840); accumulate != 0
 * adds to them.
 *   T0I_SUMS (only as T00 | TIJ | T0I_SUMS, use_phi != 0, accumulate == 0):
 *        the same deposit also leaves in GEV_FIELD_BI the T0i sums without
 *        their potential factor; the next gev_solve_B multiplies them by
 *        1 + phi(x) + phi(x + e_i) with the phi of that call, which gives
 *        projection_T0i_project with that phi (the potential enters T0i only
 *        through that per-vertex factor, and main.cu projects T0i after the
 *        phi update with the particles unmoved).  params {a, coeff}; one
 *        deposit instead of two per cycle (gev_step uses it with elliptic B). */
int gev_project(gev_ctx *ctx, uint32_t which, double a, double coeff, int32_t use_phi,
                int32_t accumulate);

/* Phi update: prepareFTsource (gevolution.hpp:183) fused into the forward FFT
 * (main.cu:725, :742), solveModifiedPoissonFT (:806; main.cu:769) in Fourier
 * space, backward FFT into GEV_FIELD_PHI (main.cu:794).  Reads SOURCE, PHI, CHI.
 * T00sum receives the sum of the source field (the return value of
 * prepareFTsource), phi_hom the k=0 mode after the solve (main.cu:808-809).
 * prepare == 0 skips prepareFTsource (Newtonian / first cycle). */
int gev_solve_phi(gev_ctx *ctx, int32_t prepare, double bgmodel, double coeff, double coeff2,
                  double coeff3, double poisson_coeff, double modif, double *T00sum,
                  double *phi_hom);

/* prepareFTsource as separate, in-place passes, for callers that keep the
 * reference's unfused call sequence (main.cu:725 then :742, :822 then :829):
 *   gev_prepare_T00: prepareFTsource(phi, chi, source, bgmodel, source, coeff,
 *     coeff2, coeff3) (gevolution.hpp:183, :160-171) -- GEV_FIELD_SOURCE becomes
 *     the nonlinear phi source; T00sum receives the sum of the source field
 *     before the preparation (the reference's return value).  Follow it with
 *     gev_solve_phi(prepare = 0, ...).
 *   gev_prepare_Tij: prepareFTsource(phi, Sij, Sij, coeff) (gevolution.hpp:119,
 *     :64-107) on GEV_FIELD_SIJ.  gev_solve_chi prepares Sij itself, so this
 *     pass is for callers that transform Sij by other means. */
int gev_prepare_T00(gev_ctx *ctx, double bgmodel, double coeff, double coeff2, double coeff3, double *T00sum);
int gev_prepare_Tij(gev_ctx *ctx, double coeff);

/* Chi update: prepareFTsource(phi, Sij, Sij, coeff) (gevolution.hpp:119;
 * main.cu:822) fused into the 6 forward FFTs (main.cu:829), projectFTscalar
 * (:251; main.cu:873) and the backward FFT into GEV_FIELD_CHI (main.cu:895).
 * With the tensor state enabled, projectFTtensor (:693) (first cycle, cycle0 != 0)
 * or evolveFTtensor (:537) (main.cu:961-965) runs on the same Fourier pencils.
 * With the parabolic vector method, evolveFTvector (:359; main.cu:933) updates
 * the B_i Fourier state with a2dtau and GEV_FIELD_BI receives B_i. */
int gev_solve_chi(gev_ctx *ctx, double coeff, int32_t cycle0, double hubble, double dtau,
                  double dtau_old, double a2dtau);

/* Elliptic B_i: forward FFT of T0i (main.cu:918), projectFTvector (:449;
 * main.cu:925), backward FFT into GEV_FIELD_BI (main.cu:948). */
int gev_solve_B(gev_ctx *ctx, double coeff, double modif);

/* Geodesic kick and drift.  kick: perfParticles::updateVel(update_q_functor,
 * dtau, {phi,chi,Bi}, nfield, {a, a^2 N}) (main.cu:1230-1235, gevolution.hpp:888);
 * maxvel receives sqrt(max q^2/a^2), the value updateVel returns.  drift:
 * perfParticles::moveParticles(update_pos_functor, dtau, fields, nfield,
 * {a, a^2 N}) (main.cu:1252-1268, gevolution.hpp:1162), including the re-binning
 * of particles into cells.  gev_kick_drift runs both in one pass (the kick's
 * fields are the drift's fields, as in the reference's sequence). */
int gev_kick(gev_ctx *ctx, double dtau, double a, double bcoeff, int32_t nfield, double *maxvel);
int gev_drift(gev_ctx *ctx, double dtau, double a, double bcoeff, int32_t nfield);
int gev_kick_drift(gev_ctx *ctx, double dtau_kick, double a_kick, double bcoeff_kick,
                   int32_t nfield_kick, double dtau_drift, double a_drift, double bcoeff_drift,
                   int32_t nfield_drift, double *maxvel);

/* Validation spectrum: scalarProjectionCIC_project (gevolution.hpp:1902),
 * forward FFT, extractPowerSpectrum (tools.hpp:339 -> :65-314) with CIC
 * deconvolution and linear k bins up to sqrt(3) pi N (or kmax if > 0).
 * The CIC density is left in GEV_FIELD_SOURCE. */
int gev_power_spectrum(gev_ctx *ctx, int32_t numbins, double kmax, double *kbin, double *power,
                       double *kscatter, double *pscatter, int32_t *occupation);

/* Lightcone crossing: the particle branch of writeLightcones
 * (output.hpp:2093-2160): findIntersectingLightcones (tools.hpp:637) and the
 * selection, ID-backlog de-duplication and interpolation of
 * perfParticles_gevolution::saveGadget2 (Particles_gevolution.hpp:1567,
 * :1271-1466, :500-593).  Outputs Gadget-2 lightcone blocks in float:
 * pos (Mpc/h), vel (Gadget units), ids.  Each shell keeps its own ID backlog
 * (lightcone_id_backlog.hpp) inside the context, as a device hash set; particle
 * ID -1 is reserved.  The selected particles stay in a device buffer of
 * `capacity` slots; pos/vel/ids may be NULL to leave them there (copy them
 * later with gev_lightcone_fetch).  n_out receives the number selected; more
 * than `capacity` fails with GEV_ERR_CAPACITY and n_out the size needed. */
typedef struct {
    double vertex[3];     /* box units */
    double direction[3];
    double opening;       /* cos of the half opening angle; -1 for the full sky */
    double distance[2];   /* [outer, inner] limits in box units (metadata.hpp lightcone_geometry) */
    double d;             /* particleHorizon at the lightcone redshift (output.hpp:1213) */
    int32_t tracer_factor;
    int32_t shell;        /* backlog slot, 0..7 */
} gev_lightcone_args;

int gev_lightcone(gev_ctx *ctx, const gev_lightcone_args *lc, double tau, double dtau,
                  double dtau_old, double a, double dadtau, int64_t capacity, float *pos,
                  float *vel, int64_t *ids, int64_t *n_out);
/* Copy the last gev_lightcone result to host arrays of `capacity` particles
 * (the host side of saveGadget2's write, Particles_gevolution.hpp:1567). */
int gev_lightcone_fetch(gev_ctx *ctx, int64_t capacity, float *pos, float *vel, int64_t *ids,
                        int64_t *n_out);

/* One full cycle of main.cu:608-1317 for CDM in the weak-field GR gauge:
 * T00 and Tij projections, Phi, chi (and h_ij), T0i projection and B_i, kick,
 * background half steps, drift, step control (gev_step_lightcone adds the
 * lightcone shell between the solves and the kick).  The caller's state
 * struct is advanced in place. */
typedef struct {
    double Omega_m, Omega_Lambda, Omega_rad;
    double fourpiG;        /* 1.5 L^2 / c^2 (main.cu:418) */
    double Cf, steplimit;  /* step control (main.cu:1307-1310) */
    double z_relax;        /* B enters the geodesic for z < z_relax (main.cu:1232) */
    double boxsize;
} gev_cosmo;

typedef struct {
    double a, tau, dtau, dtau_old;
    int64_t cycle;
    double T00hom, phi_hom, maxvel;
} gev_state;

int gev_step(gev_ctx *ctx, const gev_cosmo *cosmo, gev_state *st);
/* gev_step with one lightcone shell written where main.cu writes it: after
 * the field solves and before the kick (writeLightcones, main.cu:1040-1100),
 * with this cycle's phi, a, tau, dtau, dtau_old and dadtau = a Hconf(a).  The
 * selected particles stay in the context's device buffer of `capacity` slots
 * (gev_lightcone_fetch); n_out receives their number.  If they do not fit, the
 * cycle still completes and the call returns GEV_ERR_CAPACITY with n_out the
 * size needed. */
int gev_step_lightcone(gev_ctx *ctx, const gev_cosmo *cosmo, gev_state *st, const gev_lightcone_args *lc,
                       int64_t capacity, int64_t *n_out);

/* Background (background.hpp:200-207, :235-244, :268-291). */
double gev_hconf(double a, double fourpiG, const gev_cosmo *cosmo);
void gev_rungekutta4bg(double *a, double fourpiG, const gev_cosmo *cosmo, double dtau);
double gev_particle_horizon(double a, double fourpiG, const gev_cosmo *cosmo);

/* Poisson solve on caller-owned device arrays, allocating no device memory.
 * No counterpart in the reference: it serves host codes that cannot allocate
 * at the point of the solve (their own memory pool owns every device buffer,
 * or they are recording work into a stream).  source and phi are device
 * arrays of N^3 values, double for GEV_FP64 and float for GEV_MIXED, layout
 * x + N*(y + N*z); phi receives the inverse transform of
 * coeff * FT(source) / (-N^3 (k^2 + modif)) -- the pass sequence of
 * gev_solve_phi with prepare == 0 (solveModifiedPoissonFT, gevolution.hpp:806).
 * Work is queued on `stream` (a cudaStream_t; NULL = the legacy default
 * stream) and the call does not synchronise.
 *   - N must be 16, 32, 64 or 128: the spectrum scratch is a static device
 *     array sized for N = 128 in FP64 (about 17.3 MB); N = 256..768 returns
 *     GEV_ERR_SIZE, other N and null pointers GEV_ERR_ARG.
 *   - No part of the scratch has to start at zero.
 *   - All callers on one device share that scratch: calls whose work overlaps
 *     in time (unordered streams) race.  Order them on one stream.
 *   - The host needs the scratch's device address: the first call on each
 *     device, and the first call after that device's context was destroyed
 *     and re-created (cudaDeviceReset), looks it up (cudaGetSymbolAddress,
 *     which may also load the library's device code); make that call before
 *     any stream capture begins.
 *   - A Fourier pass whose bulk tensor copy does not complete within its wait
 *     limit leaves phi filled with NaN: the failure shows in the output, not
 *     in the return code, which reports argument and launch errors only. */
int gev_poisson_noalloc(int32_t N, int32_t precision, const void *source, void *phi,
                        double poisson_coeff, double modif, void *stream);

/* ---- Zel'dovich initial conditions ----
 * The path of the reference's IC generator with a tabulated power spectrum
 * (ic_basic.hpp:1896-1922, 2404-2437, "mPk" branch): a Gaussian white-noise
 * field (counter-based Philox4x32-10 stream of `seed`, or the caller's
 * `noise`), shaped into the Zel'dovich displacement psi = grad del^-2 delta
 * with delta_k = sqrt(P(k) N^3 / L^3) w_k (P interpolated linearly in
 * ln k / ln P; modes with |n| > N/2 dropped when ksphere != 0), one particle
 * per cell at the cell centre displaced by psi at its vertex (ID = cell
 * index, mass = Omega_m / N^3), phi from the CIC density of those particles
 * by solveModifiedPoissonFT(fourpiG/a, 3 gr (H^2 + fourpiG Omega_m / a)) with
 * the k = 0 mode removed, and momenta q = -rescale grad phi
 * (initialize_q_ic_basic, ic_basic.hpp:133-166) with
 * rescale = a / H_conf / (1.5 Omega_m(a) + 2 Omega_rad(a)).  Replaces the
 * context's particles and phi. */
typedef struct {
    double boxsize;       /* L, Mpc/h */
    double a;             /* scale factor of the initial conditions */
    double fourpiG;       /* 4 pi G in the code's units */
    double Omega_m, Omega_Lambda, Omega_rad;
    uint64_t seed;
    const double *pk_k;   /* host: k [h/Mpc], strictly increasing, n_pk values */
    const double *pk_p;   /* host: P(k) [(Mpc/h)^3] > 0 at a */
    int32_t n_pk;
    int32_t ksphere;      /* nonzero: drop modes with |n| > N/2 */
    int32_t gr;           /* nonzero: GR modification of the Poisson equation */
    int32_t reserved;
    const double *noise;  /* optional host N^3 unit white noise used instead of the stream */
    double *noise_out;    /* optional host N^3: receives the white noise used */
} gev_ics_params;

int gev_ics_zeldovich(gev_ctx *ctx, const gev_ics_params *p);

/* The reference's own initial conditions: generateIC_basic with a tabulated
 * power spectrum (ic_basic.hpp:1834-2509, the "mPk" branch; CDM only, baryon
 * treatment "ignore", no ncdm), reproduced realisation for realisation:
 *   1. the convolution kernel of generateCICKernel (:805-1118) -- built from
 *      the particle template when correct_displacement != 0, the standard
 *      lattice Laplacian kernel otherwise -- Fourier transformed;
 *   2. generateDisplacementField (:1165-1610) with the reference's random
 *      stream (sitmo::prng_engine of `seed`, Threefry-4x64-20, the same word
 *      for every mode: gev_sitmo_words gives the stream), the spectrum as
 *      loadPowerSpectrum (:370-516) and :1903-1913 turn it into a natural
 *      cubic spline of sqrt(P L / 2) / L^2 over k L, the sinc deconvolution,
 *      the gauge factor 1 + 7.5 gr H_conf^2 / k^2 and the k-sphere cut;
 *      inverse transform into the displacement potential;
 *   3. the template tiled numtile times per axis (initializeParticlePositions,
 *      :1613-1668: particle j of tile (x, y, z) gets ID
 *      j + n (x + T (y + T z))), displaced by the potential's gradient
 *      (displace_pcls_ic_basic, :65-96), mass Omega_m / (n T^3);
 *   4. phi from the particles' CIC density (:2404-2427), momenta from phi
 *      (initialize_q_ic_basic, :2431-2437), B_i (:2468-2477: T0i projection,
 *      projectFTvector with fourpiG / N^2) and chi (:2479-2489: Tij
 *      projection, prepareFTsource with 2 fourpiG / (a N^2), projectFTscalar).
 * Replaces the context's particles, phi, chi and B_i.  The particle count
 * n T^3 must fit the context's capacity.  The parabolic vector method's
 * Fourier state and the tensor state are left as they are (zero after
 * gev_ctx_create). */
typedef struct {
    double boxsize;                 /* L, Mpc/h */
    double a;                       /* 1 / (1 + z_in) */
    double fourpiG;                 /* 4 pi G in the code's units */
    double Omega_m, Omega_Lambda, Omega_rad;
    const double *pk_k;             /* host: the mPk file's k [h/Mpc], strictly increasing */
    const double *pk_p;             /* host: its P(k) [(Mpc/h)^3] >= 0 */
    int32_t n_pk;                   /* >= 3 (a cubic spline) */
    uint32_t seed;                  /* ic.seed */
    int32_t ksphere;                /* k-domain = sphere */
    int32_t correct_displacement;   /* correct displacement = yes */
    int32_t gr;                     /* gravity theory = GR (sim.gr_flag) */
    int32_t numtile;                /* tiling factor T (ic.numtile) */
    const float *template_pos;      /* host: the template's n positions in [0, 1], xyz (loadHomogeneousTemplate) */
    int64_t template_n;
} gev_ics_basic_params;

int gev_ics_basic(gev_ctx *ctx, const gev_ics_basic_params *p);

/* Words [start, start + n) of the reference IC generator's random stream for
 * `seed` (sitmo::prng_engine after seed(seed) and discard(start)), on the
 * host. */
int gev_sitmo_words(uint32_t seed, uint64_t start, int64_t n, uint32_t *out);

/* ---- Gadget-2 files (the lightcone output and snapshots) ----
 * The header mirrors gadget2_header (metadata.hpp:159-178), 256 bytes.  Files
 * hold four blocks with uint32 record lengths before and after each: header,
 * POS (3n float), VEL (3n float), ID (n int64), as the reference's
 * saveGadget2 writes them (Particles_gevolution.hpp:300-323, :826-840).
 * npart[1], npartTotal[1] and npartTotalHW[1] are set from n; the other
 * fields are the caller's (the reference fills them at output.hpp:2097-2123). */
typedef struct {
    uint32_t npart[6];
    double mass[6];
    double time;
    double redshift;
    int32_t flag_sfr;
    int32_t flag_feedback;
    uint32_t npartTotal[6];
    int32_t flag_cooling;
    int32_t num_files;
    double BoxSize;
    double Omega0;
    double OmegaLambda;
    double HubbleParam;
    int32_t flag_age;
    int32_t flag_metals;
    uint32_t npartTotalHW[6];
    char fill[64];
} gev_gadget2_header;

/* Write host arrays (e.g. gev_lightcone_fetch output, positions already in the
 * header's length unit) as one Gadget-2 file. */
int gev_gadget2_write(const char *path, const gev_gadget2_header *hdr, const float *pos, const float *vel,
                      const int64_t *ids, int64_t n);
/* Read one Gadget-2 file of this layout (one particle species, 8-byte IDs):
 * the header, then -- when pos, vel and ids are given -- the POS, VEL and ID
 * blocks into host arrays of `capacity` particles (GEV_ERR_CAPACITY if the
 * file holds more; n_out receives the count either way).  With pos, vel and
 * ids all NULL only the header and the count are read. */
int gev_gadget2_read(const char *path, gev_gadget2_header *hdr, float *pos, float *vel, int64_t *ids, int64_t capacity,
                     int64_t *n_out);
/* The particles of a Gadget-2 file into the context, converted as
 * perfParticles_gevolution::loadGadget2 does (Particles_gevolution.hpp:183,
 * :2565-2568; the reference's particle-file ICs, ic_read.hpp): positions /
 * BoxSize, momenta = vel a^1.5 GADGET_VELOCITY_CONVERSION with a = hdr.time.
 * hdr_out (may be NULL) receives the header. */
int gev_particles_load_gadget2(gev_ctx *ctx, const char *path, double mass, gev_gadget2_header *hdr_out);
/* Snapshot of the context's particles (saveGadget2, Particles_gevolution.hpp:
 * 218-420 without the redshift interpolation): particles whose ID is a
 * multiple of tracer_factor, pos * hdr->BoxSize, vel = q / a^1.5 in Gadget
 * velocity units with a = hdr->time. */
int gev_snapshot_gadget2(gev_ctx *ctx, const char *path, const gev_gadget2_header *hdr, int32_t tracer_factor);

/* ---- Checkpoint and restart ----
 * Everything a context needs to continue a run: particles (positions,
 * momenta, IDs, mass), the metric fields phi, chi, B_i, the h_ij / h_ij'
 * Fourier state (tensor contexts) and the parabolic B_i state, in FP64, plus
 * the caller's gev_state.  Reading requires a context of the same N, vector
 * method and tensor flag with enough capacity; the precision may differ.  The
 * reference's GPU build stops at its hibernation points instead of writing a
 * checkpoint (main.cu:1288-1303; the CPU build's writer is hibernation.hpp),
 * so this is the restart path of this library. */
/* Express particle files: saveExpress / loadExpress
 * (Particles_gevolution.hpp:98-143, :2641-2902), the reference's fast
 * particle dump and restart input (ic.flags ICFLAG_EXPRESSREADER).  One file
 * per rank named "<filename without a numeric suffix>.<rank>"; this library is
 * one rank, so it writes and reads "<base>.0": the express header, positions
 * (box units) and momenta in Real (real_bytes 4 or 8: the writing build's
 * sizeof(Real)), IDs, and the Gadget-2 header (hdr with npart / npartTotal /
 * num_files set to this file, as saveExpress sets them).  The reader accepts
 * either Real size, checks the layout as loadExpress does (one rank, 1 x 1
 * grid, this context's N) and replaces the context's particles. */
int gev_express_write(gev_ctx *ctx, const char *filename, const gev_gadget2_header *hdr, int32_t real_bytes);
int gev_express_read(gev_ctx *ctx, const char *filename, double mass, gev_gadget2_header *hdr_out);

int gev_checkpoint_write(gev_ctx *ctx, const char *path, const gev_state *st);
int gev_checkpoint_read(gev_ctx *ctx, const char *path, gev_state *st);

/* ---- Differentiable Newtonian PM run and its adjoint ----
 * A run of nsteps Newtonian particle-mesh steps, main.cu's gr_flag == 0 branch
 * for CDM: scalarProjectionCIC_project (gevolution.hpp:1902), FFT,
 * solveModifiedPoissonFT(src, pot, pc_n) (:806; main.cu:765), FFT^-1,
 * update_q_Newton (:1051, GRADIENT_ORDER 2; main.cu:1238) and update_pos_Newton
 * (:1270; main.cu:1264), followed by the CIC density contrast of the final
 * positions.  gev_pm_adjoint is the hand-written reverse of that run: it
 * returns d(loss)/d(x0), d(loss)/d(q0) for a given d(loss)/d(delta), recomputing
 * the states from checkpoints (x, q) kept every checkpoint_every steps.  No
 * counterpart in the reference (gevolution has no adjoint).
 * Particles are in ID order: x0, q0 are device arrays of np*3 doubles (box units,
 * unwrapped; momentum per unit mass), delta N^3 doubles.  coef holds 3 host
 * doubles per step: kq_n = dtau_kick * a * N (update_q_Newton's dtau * a / dx),
 * kx_n = dtau / a_half (update_pos_Newton's dtau / a), pc_n = fourpiG / a (the
 * Poisson coefficient).  Both calls synchronise. */
typedef struct gev_pm gev_pm;
typedef struct {
    int32_t N;                 /* grid points per side (as gev_config) */
    int32_t precision;         /* GEV_FP64 or GEV_MIXED (FP32 fields and FFTs) */
    int64_t np;                /* number of particles */
    double mass;               /* per-particle mass of the Poisson source (part_simple_info.mass) */
    int32_t checkpoint_every;  /* steps between stored (x, q) checkpoints */
    int32_t device;
} gev_pm_config;

int gev_pm_create(const gev_pm_config *cfg, gev_pm **out);
int gev_pm_destroy(gev_pm *pm);
const char *gev_pm_last_error(const gev_pm *pm);
int gev_pm_forward(gev_pm *pm, int32_t nsteps, const double *coef, const double *x0, const double *q0,
                   double *delta, double *x_out, double *q_out);
int gev_pm_adjoint(gev_pm *pm, const double *ddelta, double *gx0, double *gq0);
void *gev_pm_stream(gev_pm *pm);

/* Stream and synchronisation helpers for callers that time or overlap work.
 * gev_kernel_launches counts the kernels this context has launched so far. */
int gev_synchronize(gev_ctx *ctx);
void *gev_stream(gev_ctx *ctx);
int64_t gev_kernel_launches(const gev_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
