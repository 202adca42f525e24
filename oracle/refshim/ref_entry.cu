// ref_entry.cu -- compiles gevolution-2.0's own hot-path sources (gevolution.hpp,
// background.hpp, tools.hpp, metadata.hpp, Particles_gevolution.hpp, taken from
// the reference tree where they lie) against the single-rank LATfield2 stand-in
// in this directory, and exposes their host-side arithmetic -- and, for the
// lightcone output, their CUDA kernels -- through plain C entry points.
//
// TEST INFRASTRUCTURE ONLY: the result (oracle/_ref/libgevref.so) pins the oracle
// restatement (oracle/oracle.c) to the reference's own code, and serves as the
// reference CPU arm of bench.py.  Nothing here is part of the product path.
//
// Every entry point takes the same arguments as its orc_* twin in oracle.h.
// ref_step composes them into one cycle of main.cu's loop; LATfield2's FFT
// (PlanFFT, cuFFT/FFTW inside, not part of the reference tree) is stood in for
// by the oracle's FFT (orc_r2c / orc_c2r, linked from ../liboracle.so) or by
// the pair of transforms given to ref_set_fft.
#include <cstdint>
#include <omp.h>
#include <nvtx3/nvToolsExt.h>
#include "LATfield2.hpp"
#include "cuda_staging.hpp"
#include "metadata.hpp"
#include "tools.hpp"
#include "background.hpp"
#include "gevolution.hpp"
#include "Particles_gevolution.hpp"
#include "ic_basic.hpp"

#include <cstdint>
#include <functional>
#include <vector>

#include "../oracle.h"

using namespace LATfield2;

// the transforms of ref_step and PlanFFT (ref_set_fft)
typedef void (*ref_fft_fn)(int N, const double * in, double * out);
static ref_fft_fn g_r2c = orc_r2c, g_c2r = orc_c2r;

namespace
{

struct ParticleSet
{
	Lattice lat;
	std::vector<part_simple> parts;
	perfParticles<part_simple, part_simple_info> pcls;

	ParticleSet(int N, int64_t np, const double * pos, const double * q, double mass) : lat(N, false), parts(np)
	{
		for (int64_t p = 0; p < np; p++)
		{
			for (int i = 0; i < 3; i++)
			{
				parts[p].pos[i] = pos[3 * p + i];
				parts[p].vel[i] = q ? q[3 * p + i] : 0.;
			}
			parts[p].ID = p;
		}
		part_simple_info info{};
		info.mass = mass;
		pcls.attach(&lat, parts.data(), np, info);
	}
};

void site_loop(int N, const std::function<void(int, int, int)> & body)
{
#pragma omp parallel for collapse(2) schedule(static)
	for (int z = 0; z < N; z++)
		for (int y = 0; y < N; y++)
			for (int x = 0; x < N; x++) body(x, y, z);
}

cosmology make_cosmo(double Om, double OL, double Orad)
{
	cosmology c;
	std::memset(&c, 0, sizeof(c));
	c.Omega_cdm = Om;
	c.Omega_b = 0.;
	c.Omega_m = Om;
	c.Omega_Lambda = OL;
	c.Omega_rad = Orad;
	c.num_ncdm = 0;
	return c;
}

} // namespace

extern "C" {

// projection_T00_project (gevolution.hpp:1887) through particle_T00_project's host branch
void ref_project_T00(int N, int64_t np, const double * pos, const double * q, double mass, const double * phi, double a, double coeff, double * T00)
{
	ParticleSet ps(N, np, pos, q, mass);
	Field<Real> fT00(ps.lat, T00, 1), fphi(ps.lat, const_cast<double *>(phi), 1);
	Field<Real> * fields[2] = {&fT00, phi ? &fphi : nullptr};
	double params[2] = {a, coeff};
	ps.pcls.projectParticles(particle_T00_project_functor(), fields, phi ? 2 : 1, params);
}

// projection_Tij_project (gevolution.hpp:2999) through particle_Tij_project's host branch
void ref_project_Tij(int N, int64_t np, const double * pos, const double * q, double mass, const double * phi, double a, double coeff, double * Tij)
{
	ParticleSet ps(N, np, pos, q, mass);
	Field<Real> fT(ps.lat, Tij, 6, symmetric), fphi(ps.lat, const_cast<double *>(phi), 1);
	Field<Real> * fields[2] = {&fT, phi ? &fphi : nullptr};
	double params[7] = {a, coeff, 0, 0, 0, 0, 0};
	ps.pcls.projectParticles(particle_Tij_project_functor(), fields, phi ? 2 : 1, params);
}

// projection_T0i_project (gevolution.hpp:2232) through particle_T0i_project's host branch
void ref_project_T0i(int N, int64_t np, const double * pos, const double * q, double mass, const double * phi, double coeff, double * T0i)
{
	ParticleSet ps(N, np, pos, q, mass);
	Field<Real> fT(ps.lat, T0i, 3), fphi(ps.lat, const_cast<double *>(phi), 1);
	Field<Real> * fields[2] = {&fT, phi ? &fphi : nullptr};
	ps.pcls.projectParticles(particle_T0i_project_functor(), fields, phi ? 2 : 1, &coeff);
}

// scalarProjectionCIC_project (gevolution.hpp:1902)
void ref_project_cic(int N, int64_t np, const double * pos, double mass, double * rho)
{
	ParticleSet ps(N, np, pos, nullptr, mass);
	Field<Real> f(ps.lat, rho, 1);
	scalarProjectionCIC_project(&ps.pcls, &f);
}

// prepareFTsource_T00 (gevolution.hpp:160-171), applied site by site; returns the sum of source
double ref_prepare_T00(int N, const double * phi, const double * chi, const double * source, double bgmodel, double coeff, double coeff2, double coeff3, double * result)
{
	Lattice lat(N, false);
	std::vector<double> src(source, source + (size_t) N * N * N);
	Field<Real> fres(lat, result, 1), fsrc(lat, src.data(), 1), fphi(lat, const_cast<double *>(phi), 1), fchi(lat, const_cast<double *>(chi), 1);
	Field<Real> * fields[4] = {&fres, &fsrc, &fphi, &fchi};
	double params[4] = {bgmodel, coeff, coeff2, coeff3};
	double sum = 0.;
#pragma omp parallel for collapse(2) reduction(+ : sum) schedule(static)
	for (int z = 0; z < N; z++)
		for (int y = 0; y < N; y++)
			for (int x = 0; x < N; x++)
			{
				Site s(lat, x, y, z);
				Site sites[4] = {s, s, s, s};
				double out[1];
				prepareFTsource_T00(fields, sites, 4, params, out);
				sum += out[0];
			}
	return sum;
}

// prepareFTsource_Tij (gevolution.hpp:64-107), applied site by site
void ref_prepare_Tij(int N, const double * phi, const double * Tij, double coeff, double * Sij)
{
	Lattice lat(N, false);
	std::vector<double> tij(Tij, Tij + 6 * (size_t) N * N * N);
	Field<Real> fS(lat, Sij, 6, symmetric), fT(lat, tij.data(), 6, symmetric), fphi(lat, const_cast<double *>(phi), 1);
	Field<Real> * fields[3] = {&fS, &fT, &fphi};
	double params = coeff;
	site_loop(N, [&](int x, int y, int z) {
		Site s(lat, x, y, z);
		Site sites[3] = {s, s, s};
		prepareFTsource_Tij(fields, sites, 3, &params, nullptr);
	});
}

// Fourier-space solvers, called unchanged (gevolution.hpp:251-852)
void ref_solve_poisson(int N, const double * srcFT, double * potFT, double coeff, double modif)
{
	Lattice lat(N, true);
	size_t m = (size_t) (N / 2 + 1) * N * N;
	std::vector<Imag> src((const Imag *) srcFT, (const Imag *) srcFT + m);
	Field<Imag> fs(lat, src.data(), 1), fp(lat, (Imag *) potFT, 1);
	solveModifiedPoissonFT(fs, fp, coeff, modif);
}

void ref_project_scalar(int N, const double * SijFT, double * chiFT, int add)
{
	Lattice lat(N, true);
	Field<Imag> fS(lat, (Imag *) SijFT, 6, symmetric), fc(lat, (Imag *) chiFT, 1);
	projectFTscalar(fS, fc, add);
}

void ref_project_vector(int N, const double * SiFT, double * BiFT, double coeff, double modif)
{
	Lattice lat(N, true);
	size_t m = (size_t) (N / 2 + 1) * N * N;
	std::vector<Imag> s((const Imag *) SiFT, (const Imag *) SiFT + 3 * m);
	Field<Imag> fS(lat, s.data(), 3), fB(lat, (Imag *) BiFT, 3);
	projectFTvector(fS, fB, coeff, modif);
}

void ref_evolve_vector(int N, const double * SijFT, double * BiFT, double a2dtau)
{
	Lattice lat(N, true);
	Field<Imag> fS(lat, (Imag *) SijFT, 6, symmetric), fB(lat, (Imag *) BiFT, 3);
	evolveFTvector(fS, fB, a2dtau);
}

void ref_project_tensor(int N, const double * SijFT, double * hijFT)
{
	Lattice lat(N, true);
	Field<Imag> fS(lat, (Imag *) SijFT, 6, symmetric), fh(lat, (Imag *) hijFT, 6, symmetric);
	projectFTtensor(fS, fh);
}

void ref_evolve_tensor(int N, double * SijFT, double * hijFT, double * hijprimeFT, double hubble, double dtau, double dtau_old)
{
	Lattice lat(N, true);
	Field<Imag> fS(lat, (Imag *) SijFT, 6, symmetric), fh(lat, (Imag *) hijFT, 6, symmetric), fhp(lat, (Imag *) hijprimeFT, 6, symmetric);
	evolveFTtensor(fS, fh, fhp, hubble, dtau, dtau_old);
}

// update_q (gevolution.hpp:888-1011) through perfParticles::updateVel; returns sqrt(max q^2/a^2)
double ref_update_q(int N, int64_t np, const double * pos, double * q, const double * phi, const double * chi, const double * Bi, int nfield, double dtau, double a, double bcoeff)
{
	ParticleSet ps(N, np, pos, q, 0.);
	Field<Real> fphi(ps.lat, const_cast<double *>(phi), 1), fchi(ps.lat, const_cast<double *>(chi), 1), fB(ps.lat, const_cast<double *>(Bi), 3);
	Field<Real> * fields[3] = {&fphi, chi ? &fchi : nullptr, Bi ? &fB : nullptr};
	double params[7] = {a, bcoeff, 0, 0, 0, 0, 0};
	double vmax = ps.pcls.updateVel(update_q_functor(), dtau, fields, nfield, params);
	for (int64_t p = 0; p < np; p++)
		for (int i = 0; i < 3; i++) q[3 * p + i] = ps.parts[p].vel[i];
	return vmax;
}

// update_pos (gevolution.hpp:1162-1232) through perfParticles::moveParticles
void ref_update_pos(int N, int64_t np, double * pos, const double * q, const double * phi, const double * chi, const double * Bi, int nfield, double dtau, double a, double bcoeff)
{
	ParticleSet ps(N, np, pos, q, 0.);
	Field<Real> fphi(ps.lat, const_cast<double *>(phi), 1), fchi(ps.lat, const_cast<double *>(chi), 1), fB(ps.lat, const_cast<double *>(Bi), 3);
	Field<Real> * fields[3] = {&fphi, &fchi, &fB};
	double params[7] = {a, bcoeff, 0, 0, 0, 0, 0};
	ps.pcls.moveParticles(update_pos_functor(), dtau, fields, nfield, params);
	for (int64_t p = 0; p < np; p++)
		for (int i = 0; i < 3; i++) pos[3 * p + i] = ps.parts[p].pos[i];
}

// update_q_Newton (gevolution.hpp:1051-1118) through perfParticles::updateVel
double ref_update_q_newton(int N, int64_t np, const double * pos, double * q, const double * psi, double dtau, double a)
{
	ParticleSet ps(N, np, pos, q, 0.);
	Field<Real> fpsi(ps.lat, const_cast<double *>(psi), 1);
	Field<Real> * fields[2] = {&fpsi, nullptr};
	double params[7] = {a, 0, 0, 0, 0, 0, 0};
	double vmax = ps.pcls.updateVel(update_q_Newton_functor(), dtau, fields, 1, params);
	for (int64_t p = 0; p < np; p++)
		for (int i = 0; i < 3; i++) q[3 * p + i] = ps.parts[p].vel[i];
	return vmax;
}

// update_pos_Newton (gevolution.hpp:1270-1273) through perfParticles::moveParticles
void ref_update_pos_newton(int N, int64_t np, double * pos, const double * q, double dtau, double a)
{
	ParticleSet ps(N, np, pos, q, 0.);
	double params[7] = {a, 0, 0, 0, 0, 0, 0};
	ps.pcls.moveParticles(update_pos_Newton_functor(), dtau, nullptr, 0, params);
	for (int64_t p = 0; p < np; p++)
		for (int i = 0; i < 3; i++) pos[3 * p + i] = ps.parts[p].pos[i];
}

// background.hpp:200-291
double ref_hconf(double a, double fourpiG, double Om, double OL, double Orad)
{
	return Hconf(a, fourpiG, make_cosmo(Om, OL, Orad));
}

double ref_rk4bg(double a, double fourpiG, double Om, double OL, double Orad, double dtau)
{
	rungekutta4bg(a, fourpiG, make_cosmo(Om, OL, Orad), dtau);
	return a;
}

double ref_particle_horizon(double a, double fourpiG, double Om, double OL, double Orad)
{
	cosmology c = make_cosmo(Om, OL, Orad);
	return particleHorizon(a, fourpiG, c);
}

// extractPowerSpectrum (tools.hpp:339 -> :65-314), deconvolved, linear k
void ref_power_spectrum(int N, const double * fieldFT, int numbins, double * kbin, double * power, double * kscatter, double * pscatter, int * occupation)
{
	Lattice lat(N, true);
	Field<Imag> f(lat, (Imag *) const_cast<double *>(fieldFT), 1);
	extractPowerSpectrum(f, kbin, power, kscatter, pscatter, occupation, numbins, true, KTYPE_LINEAR);
}

// findIntersectingLightcones (tools.hpp:637-886); vertex_out holds MAX_INTERSECTS*3 doubles
int ref_find_intersecting(const double * lc_vertex, const double * lc_direction, double opening, double outer, double inner, const double * domain, double * vertex_out)
{
	lightcone_geometry lc;
	std::memset(&lc, 0, sizeof(lc));
	for (int i = 0; i < 3; i++) { lc.vertex[i] = lc_vertex[i]; lc.direction[i] = lc_direction[i]; }
	lc.opening = opening;
	double dom[6];
	for (int i = 0; i < 6; i++) dom[i] = domain[i];
	double vtx[MAX_INTERSECTS][3];
	int n = findIntersectingLightcones(lc, outer, inner, dom, vtx);
	for (int v = 0; v < n && v < MAX_INTERSECTS; v++)
		for (int i = 0; i < 3; i++) vertex_out[3 * v + i] = vtx[v][i];
	return n;
}

int ref_max_intersects(void) { return MAX_INTERSECTS; }

// perfParticles_gevolution::saveExpress (Particles_gevolution.hpp:2641-2767)
// of np particles (pos, q box units, ids) on an N^3 lattice, one rank; hdr is
// the 256-byte gadget2_header.  Particle arrays in managed memory (the writer
// copies them from the device), so the call needs a GPU.  0, or -1.
int ref_express_write(const char * filename, int N, int64_t np, const double * pos, const double * q, const int64_t * ids,
                      const void * hdr)
{
	typedef perfParticles_gevolution<part_simple, part_simple_info> PG;
	PG pcl;
	Real * mp = nullptr, * mq = nullptr;
	long * mid = nullptr;
	if (cudaMallocManaged(&mp, sizeof(Real) * 3 * (np + 1)) != cudaSuccess ||
	    cudaMallocManaged(&mq, sizeof(Real) * 3 * (np + 1)) != cudaSuccess ||
	    cudaMallocManaged(&mid, sizeof(long) * (np + 1)) != cudaSuccess)
		return -1;
	for (int64_t i = 0; i < 3 * np; i++) { mp[i] = pos[i]; mq[i] = q[i]; }
	for (int64_t i = 0; i < np; i++) mid[i] = ids[i];
	pcl.p = mp; pcl.q = mq; pcl.other = mid;
	pcl.num_particles_ = np;
	pcl.total_capacity_ = np;
	for (int i = 0; i < 3; i++) { pcl.lat_size_[i] = N; pcl.lat_size_local_[i] = N; }
	gadget2_header h;
	std::memcpy(&h, hdr, sizeof(h));
	int rc = 0;
	try { pcl.saveExpress(filename, h); } catch (...) { rc = -1; }
	cudaFree(mp); cudaFree(mq); cudaFree(mid);
	return rc;
}

// perfParticles_gevolution::loadExpress (:2769-2902) into arrays of capacity
// cap; n receives the count, hdr the 256-byte gadget2_header.  0, or -1 if the
// reader rejects the file.
int ref_express_read(const char * filename, int N, int64_t cap, double * pos, double * q, int64_t * ids, int64_t * n,
                     void * hdr)
{
	typedef perfParticles_gevolution<part_simple, part_simple_info> PG;
	PG pcl;
	Real * mp = nullptr, * mq = nullptr;
	long * mid = nullptr;
	if (cudaMallocManaged(&mp, sizeof(Real) * 3 * (cap + 1)) != cudaSuccess ||
	    cudaMallocManaged(&mq, sizeof(Real) * 3 * (cap + 1)) != cudaSuccess ||
	    cudaMallocManaged(&mid, sizeof(long) * (cap + 1)) != cudaSuccess)
		return -1;
	pcl.p = mp; pcl.q = mq; pcl.other = mid;
	pcl.total_capacity_ = cap;
	for (int i = 0; i < 3; i++) { pcl.lat_size_[i] = N; pcl.lat_size_local_[i] = N; }
	gadget2_header h;
	int rc = 0;
	try { pcl.loadExpress(filename, h); } catch (...) { rc = -1; }
	if (rc == 0)
	{
		*n = pcl.num_particles_;
		for (int64_t i = 0; i < 3 * pcl.num_particles_; i++) { pos[i] = mp[i]; q[i] = mq[i]; }
		for (int64_t i = 0; i < pcl.num_particles_; i++) ids[i] = mid[i];
		std::memcpy(hdr, &h, sizeof(h));
	}
	cudaFree(mp); cudaFree(mq); cudaFree(mid);
	return rc;
}

// the natural cubic spline of the GSL stand-in (gsl_spline_init, gsl_spline_eval)
// through (x, y), n knots, at m points v
void ref_spline_eval(const double * x, const double * y, int n, const double * v, int m, double * out)
{
	gsl_spline * s = gsl_spline_alloc(gsl_interp_cspline, n);
	gsl_spline_init(s, x, y, n);
	for (int i = 0; i < m; i++) out[i] = gsl_spline_eval(s, v[i], nullptr);
	gsl_spline_free(s);
}

// n words of sitmo::prng_engine (prng_engine.hpp) after seed(seed) and
// discard(start): the random stream of generateDisplacementField
void ref_sitmo_words(uint32_t seed, uint64_t start, int64_t n, uint32_t * out)
{
	sitmo::prng_engine e;
	e.seed(seed);
	if (start) e.discard(start);
	for (int64_t i = 0; i < n; i++) out[i] = e();
}

// The reference's initial-condition generator for a tabulated power spectrum:
// generateIC_basic (ic_basic.hpp:1834-2509), CDM only (baryon treatment
// "ignore", no ncdm), composed like ref_step from the reference's own
// functions in its order.  The spectrum and the particle template are
// written to temporary files that the reference's loadPowerSpectrum and
// loadHomogeneousTemplate read; generateCICKernel, generateDisplacementField,
// initializeParticlePositions, the displacement and velocity functors, the
// CIC projection and the Fourier solvers are called unchanged.  The
// driver-level wrappers that stage their parameters on the GPU
// (projection_T0i_project, projection_Tij_project, prepareFTsource) are
// replaced by their functors applied on the host, as in ref_step.  The
// oracle's FFT (or ref_set_fft's) stands behind PlanFFT; thrust's device
// system is OpenMP in this build (oracle/Makefile), so generateCICKernel's
// thrust::fill_n runs on the host.
// Outputs: the n_tmpl numtile^3 particles in ID order (pos, q box units; ids),
// phi, chi (N^3) and B_i (3 N^3), maxvel[0] (:2433).  Returns 0, -1 on a file
// error.
int ref_ics_basic(int N, double boxsize, double a, double fourpiG, double Om, double OL, double Orad, const double * pk_k,
                  const double * pk_p, int n_pk, uint32_t seed, int ksphere, int correct, int gr, int numtile,
                  const float * tmpl, int64_t ntmpl, double * pos, double * q, int64_t * ids, double * phi, double * chi,
                  double * Bi, double * maxvel)
{
	// the input files
	char pkname[] = "/tmp/gev_ref_pk_XXXXXX", pclname[] = "/tmp/gev_ref_pcl_XXXXXX";
	int fd1 = mkstemp(pkname), fd2 = mkstemp(pclname);
	if (fd1 < 0 || fd2 < 0) return -1;
	{
		FILE * f = fdopen(fd1, "w");
		for (int i = 0; i < n_pk; i++) fprintf(f, "%.17g %.17g\n", pk_k[i], pk_p[i]);
		fclose(f);
		gadget2_header hdr;
		std::memset(&hdr, 0, sizeof(hdr));
		hdr.npart[1] = (uint32_t) ntmpl;
		hdr.npartTotal[1] = (uint32_t) ntmpl;
		hdr.num_files = 1;
		hdr.BoxSize = 1.0;
		FILE * g = fdopen(fd2, "wb");
		uint32_t b = sizeof(hdr);
		fwrite(&b, 4, 1, g); fwrite(&hdr, sizeof(hdr), 1, g); fwrite(&b, 4, 1, g);
		b = (uint32_t) (12 * ntmpl);
		fwrite(&b, 4, 1, g); fwrite(tmpl, sizeof(float), 3 * ntmpl, g); fwrite(&b, 4, 1, g);
		fclose(g);
	}
	const cosmology cosmo = make_cosmo(Om, OL, Orad);
	const int64_t n3 = (int64_t) N * N * N, nk = (int64_t) (N / 2 + 1) * N * N;
	const double dx = 1. / N;
	std::vector<double> vsrc(n3, 0.), vSij(6 * n3, 0.);
	std::vector<Imag> vscalar(nk), vBiFT(3 * nk), vSijFT(6 * nk);
	Lattice lat(N, false), klat(N, true);
	Field<Real> fphi(lat, phi, 1), fchi(lat, chi, 1), fsource(lat, vsrc.data(), 1), fBi(lat, Bi, 3), fSij(lat, vSij.data(), 6, symmetric);
	Field<Imag> fscalar(klat, vscalar.data(), 1), fBiFT(klat, vBiFT.data(), 3), fSijFT(klat, vSijFT.data(), 6, symmetric);
	gev_shim_r2c = g_r2c;
	gev_shim_c2r = g_c2r;
	PlanFFT<Imag> plan_phi(&fphi, &fscalar), plan_chi(&fchi, &fscalar), plan_source(&fsource, &fscalar);
	PlanFFT<Imag> plan_Bi(&fBi, &fBiFT, 3), plan_Sij(&fSij, &fSijFT, 6);
	const double H = Hconf(a, fourpiG, cosmo);

	// template (:1873), kernel and its transform (:1892-1899)
	long numpcl = 0;
	float * pcldata = nullptr;
	loadHomogeneousTemplate(pclname, numpcl, pcldata);
	if (correct) generateCICKernel(fsource, numpcl, pcldata, numtile);
	else generateCICKernel(fsource);
	plan_source.execute(FFT_FORWARD);
	// spectrum (:1903-1920) and displacement potential (:1922, :2190)
	gsl_spline * pkspline = nullptr;
	loadPowerSpectrum(pkname, pkspline, boxsize);
	{
		std::vector<double> x(pkspline->x, pkspline->x + pkspline->size), y(pkspline->size);
		for (size_t i = 0; i < pkspline->size; i++) y[i] = pkspline->y[i] / boxsize / boxsize;
		const size_t size = pkspline->size;
		gsl_spline_free(pkspline);
		pkspline = gsl_spline_alloc(gsl_interp_cspline, size);
		gsl_spline_init(pkspline, x.data(), y.data(), size);
	}
	generateDisplacementField(fscalar, gr * H * H, pkspline, seed, ksphere ? ICFLAG_KSPHERE : 0);
	plan_chi.execute(FFT_BACKWARD);
	// particles (:2198-2219)
	perfParticles<part_simple, part_simple_info> pcls_cdm;
	part_simple_info info;
	std::memset(&info, 0, sizeof(info));
	info.mass = cosmo.Omega_cdm / (Real) (numpcl * (long) numtile * (long) numtile * (long) numtile);
	Real boxSize[3] = {1., 1., 1.};
	const long capacity = 16L * numpcl * numtile * numtile * numtile / 15L;
	pcls_cdm.initialize(info, &lat, boxSize, capacity + PCL_EXTRA_CAPACITY, PCL_EXTRA_CAPACITY);
	initializeParticlePositions(numpcl, pcldata, numtile, pcls_cdm);
	{
		Field<Real> * f[1] = {&fchi};
		double maxdisp = 0.;
		int op = MAX;
		pcls_cdm.moveParticles(displace_pcls_ic_basic_functor(), 1., f, 1, nullptr, &maxdisp, &op, 1);
	}
	free(pcldata);
	// phi from the CIC density (:2407-2425)
	std::fill(vsrc.begin(), vsrc.end(), 0.);
	scalarProjectionCIC_project(&pcls_cdm, &fsource);
	plan_source.execute(FFT_FORWARD);
	vscalar[0] = Imag(0., 0.);
	solveModifiedPoissonFT(fscalar, fscalar, fourpiG / a, 3. * gr * (H * H + fourpiG * cosmo.Omega_m / a));
	plan_phi.execute(FFT_BACKWARD);
	// momenta (:2429-2434)
	{
		const double rescale = a / H / (1.5 * Omega_m(a, cosmo) + 2. * Omega_rad(a, cosmo));
		Field<Real> * f[1] = {&fphi};
		*maxvel = pcls_cdm.updateVel(initialize_q_ic_basic_functor(), rescale, f, 1) / a;
	}
	// B_i (:2469-2477): projection_T0i_project(pcls, Bi, phi) through its functor
	std::fill(Bi, Bi + 3 * n3, 0.);
	{
		Field<Real> * f[2] = {&fBi, &fphi};
		double coeff = 1.;
		pcls_cdm.projectParticles(particle_T0i_project_functor(), f, 2, &coeff);
	}
	plan_Bi.execute(FFT_FORWARD);
	projectFTvector(fBiFT, fBiFT, fourpiG / (double) N / (double) N);
	plan_Bi.execute(FFT_BACKWARD);
	// chi (:2481-2491): projection_Tij_project(pcls, Sij, a, phi) and
	// prepareFTsource(phi, Sij, Sij, 2 fourpiG / a / N^2) through their functors
	std::fill(vSij.begin(), vSij.end(), 0.);
	{
		Field<Real> * f[2] = {&fSij, &fphi};
		double params[7] = {a, 1., 0., 0., 0., 0., 0.};
		pcls_cdm.projectParticles(particle_Tij_project_functor(), f, 2, params);
	}
	{
		Field<Real> * f[3] = {&fSij, &fSij, &fphi};
		double coeff = 2. * fourpiG / a / (double) N / (double) N;
		site_loop(N, [&](int x, int y, int z) {
			Site st(lat, x, y, z);
			Site sites[3] = {st, st, st};
			prepareFTsource_Tij(f, sites, 3, &coeff, nullptr);
		});
	}
	plan_Sij.execute(FFT_FORWARD);
	projectFTscalar(fSijFT, fscalar);
	plan_chi.execute(FFT_BACKWARD);
	gsl_spline_free(pkspline);
	std::remove(pkname);
	std::remove(pclname);
	(void) dx;

	const long np = pcls_cdm.num_particles();
	const part_simple * pp = pcls_cdm.particles();
	for (long i = 0; i < np; i++)
	{
		for (int k = 0; k < 3; k++) { pos[3 * i + k] = pp[i].pos[k]; q[3 * i + k] = pp[i].vel[k]; }
		ids[i] = pp[i].ID;
	}
	return 0;
}

// The particle lightcone shell of one cycle as the reference writes it
// (writeLightcones, output.hpp:2093-2135 -> perfParticles_gevolution::
// saveGadget2, Particles_gevolution.hpp:1567-2160), run on the GPU with the
// reference's own kernels: count_tracer_particles, buffer_tracer_IDs and
// count_lightcone_duplicate_ids (the check-zone count), buffer_tracer_particles
// with bufferTracerParticle (selection and EXACT_OUTPUT_REDSHIFTS
// interpolation), mark_lightcone_kept_particles and
// gather_lightcone_kept_particles (de-duplication against the ID backlog),
// count/fill_lightcone_prelog_bins (the IDs logged for the next cycle's
// backlog).  One rank, all rows in one chunk, no file: the caller gets the
// buffers saveGadget2 would write.
//   pos, q: np x 3 box units; id: np; phi: N^3 (or NULL); vertex, direction,
//   opening: the lightcone geometry; dist = d - tau; backlog: the IDs logged
//   in the previous cycle (any order; sorted and made unique here, as
//   LightconeIDBacklog::finalize does); idlog_scatter selects the 9-bin ID log
//   (saveGadget2<1>, output.hpp:1180).
// Outputs: the kept particles (pos in boxsize units, vel, ids) in the order
// the reference leaves them, n_out; n_header = the header's particle count
// (selected minus check-zone duplicates); prelog: the IDs logged, bin by bin.
// Returns 0, -1 on a CUDA error, -2 if capacity is too small (n_out holds the
// count needed).
int ref_lightcone_shell(int N, int64_t np, const double * pos, const double * q, const int64_t * id, const double * phi,
                        const double * lc_vertex, const double * lc_direction, double opening, double dist, double dtau,
                        double dtau_old, double a, double dadtau, double boxsize, int tracer_factor, int idlog_scatter,
                        const int64_t * backlog, int64_t nbacklog, int64_t capacity, float * out_pos, float * out_vel,
                        int64_t * out_id, int64_t * n_out, int64_t * n_header, int64_t * prelog, int64_t * n_prelog)
{
	typedef perfParticles_gevolution<part_simple, part_simple_info> PG;
	typedef PG::RowBuffer Row;
	std::vector<void *> allocs;
	bool failed = false;
	auto managed = [&](size_t bytes) -> void *
	{
		void * m = nullptr;
		if (cudaMallocManaged(&m, bytes > 0 ? bytes : 1) != cudaSuccess) { failed = true; return nullptr; }
		allocs.push_back(m);
		return m;
	};
	auto release = [&](int rc) { cudaDeviceSynchronize(); for (void * m : allocs) cudaFree(m); return rc; };
	auto sync = [&]() { return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess; };

	// vertices: output.hpp:1175-1190 (the whole box on one rank) and :2095
	lightcone_geometry lc;
	std::memset(&lc, 0, sizeof(lc));
	for (int i = 0; i < 3; i++) { lc.vertex[i] = lc_vertex[i]; lc.direction[i] = lc_direction[i]; }
	lc.opening = opening;
	double domain[6];
	for (int i = 0; i < 3; i++) { domain[i] = -0.5 / N; domain[i + 3] = (N + 0.5) / N; }
	double vertex[MAX_INTERSECTS][3];
	const int vertexcount = findIntersectingLightcones(lc, dist + (0.5 + LIGHTCONE_IDCHECK_ZONE) * dtau_old, dist - 0.5 * dtau, domain, vertex);
	const Real inner = dist - 0.5 * dtau;                                     // Particles_gevolution.hpp:1602-1603
	const Real outer = dist + (0.5 + LIGHTCONE_IDCHECK_ZONE) * dtau_old;

	// particles into row buffers, one per (y, z) row of cells, in input order
	const int nrows = N * N;
	std::vector<int> rowcount(nrows, 0), rowof(np);
	for (int64_t p = 0; p < np; p++)
	{
		int c[3];
		for (int i = 0; i < 3; i++) c[i] = (((int) std::floor(pos[3 * p + i] * N)) % N + N) % N;
		rowof[p] = c[1] + N * c[2];
		rowcount[rowof[p]]++;
	}
	Real * pp = (Real *) managed(sizeof(Real) * 3 * np);
	Real * pq = (Real *) managed(sizeof(Real) * 3 * np);
	long * pid = (long *) managed(sizeof(long) * np);
	Row * rows = (Row *) managed(sizeof(Row) * nrows);
	PG * pcl = (PG *) managed(sizeof(PG));
	double (*d_vertex)[3] = (double (*)[3]) managed(sizeof(double) * 3 * MAX_INTERSECTS);
	Real * d_domain = (Real *) managed(sizeof(Real) * 4);
	long * d_npart = (long *) managed(sizeof(long));
	int * d_npart_row = (int *) managed(sizeof(int) * nrows);
	int * d_npart_check_row = (int *) managed(sizeof(int) * nrows);
	unsigned long long * counters = (unsigned long long *) managed(sizeof(unsigned long long) * 4);
	if (failed) return release(-1);
	{
		std::vector<long> start(nrows + 1, 0);
		for (int r = 0; r < nrows; r++) start[r + 1] = start[r] + rowcount[r];
		std::vector<long> fill(start.begin(), start.end() - 1);
		for (int64_t p = 0; p < np; p++)
		{
			const long k = fill[rowof[p]]++;
			for (int i = 0; i < 3; i++) { pp[3 * k + i] = pos[3 * p + i]; pq[3 * k + i] = q[3 * p + i]; }
			pid[k] = id ? (long) id[p] : (long) p;
		}
		for (int r = 0; r < nrows; r++) rows[r] = Row{rowcount[r], pp + 3 * start[r], pq + 3 * start[r], pid + start[r]};
	}
	new (pcl) PG();
	pcl->row_buffers_ = rows;
	pcl->num_row_buffers_ = nrows;
	for (int i = 0; i < 3; i++) { pcl->lat_size_[i] = N; pcl->lat_size_local_[i] = N; pcl->boxSize_[i] = 1; }
	for (int v = 0; v < vertexcount; v++)
		for (int i = 0; i < 3; i++) d_vertex[v][i] = vertex[v][i];
	// the rank's domain in box units (Particles_gevolution.hpp:1634-1637)
	d_domain[0] = 0; d_domain[1] = 1; d_domain[2] = 0; d_domain[3] = 1;
	Field<Real> * fphi = nullptr;
	if (phi)
	{
		Lattice * lat = (Lattice *) managed(sizeof(Lattice));
		Real * data = (Real *) managed(sizeof(Real) * (size_t) N * N * N);
		fphi = (Field<Real> *) managed(sizeof(Field<Real>));
		if (failed) return release(-1);
		new (lat) Lattice(N, false);
		for (long i = 0; i < (long) N * N * N; i++) data[i] = phi[i];
		new (fphi) Field<Real>(*lat, data, 1);
	}

	// count (Particles_gevolution.hpp:1670)
	*d_npart = 0;
	for (int r = 0; r < nrows; r++) { d_npart_row[r] = 0; d_npart_check_row[r] = 0; }
	count_tracer_particles<part_simple, part_simple_info><<<nrows, 128>>>(pcl, tracer_factor, lc, inner, outer, dtau_old, d_vertex, vertexcount, d_npart, d_npart_row, d_npart_check_row);
	if (!sync()) return release(-1);
	long total = 0, check = 0;
	for (int r = 0; r < nrows; r++) { total += d_npart_row[r]; check += d_npart_check_row[r]; }

	std::vector<long> bl(backlog, backlog + nbacklog);
	std::sort(bl.begin(), bl.end());
	bl.erase(std::unique(bl.begin(), bl.end()), bl.end());
	long * d_backlog = (long *) managed(sizeof(long) * bl.size());
	float * posdata = (float *) managed(sizeof(float) * 3 * total);
	float * veldata = (float *) managed(sizeof(float) * 3 * total);
	long * ids = (long *) managed(sizeof(long) * total);
	unsigned char * loginfo = (unsigned char *) managed(total);
	long * check_ids = (long *) managed(sizeof(long) * check);
	if (failed) return release(-1);
	for (size_t i = 0; i < bl.size(); i++) d_backlog[i] = bl[i];

	// check-zone IDs against the backlog: the header count (:1806-1856)
	long reject = 0;
	counters[0] = 0;
	buffer_tracer_IDs<part_simple, part_simple_info><<<nrows, 128>>>(pcl, tracer_factor, lc, inner, outer, dtau_old, d_vertex, vertexcount, check_ids, 0, counters);
	if (!sync()) return release(-1);
	if (counters[0] > 0 && !bl.empty())
	{
		counters[1] = 0;
		const int blocks = std::min<long>((counters[0] + 255) / 256, 65535);
		count_lightcone_duplicate_ids<<<blocks, 256>>>(check_ids, counters[0], d_backlog, (long) bl.size(), counters + 1);
		if (!sync()) return release(-1);
		reject = (long) counters[1];
	}
	*n_header = total - reject;

	// buffer the particles: check zone first, the rest after it (:2000-2056)
	counters[0] = 0;
	counters[1] = (unsigned long long) check;
	if (idlog_scatter)
		buffer_tracer_particles<part_simple, part_simple_info, 1><<<nrows, 128>>>(pcl, tracer_factor, lc, (Real) dist, inner, outer, dtau, dtau_old, a, dadtau, boxsize, d_domain, fphi, d_vertex, vertexcount, posdata, veldata, ids, loginfo, 0, counters, counters + 1);
	else
		buffer_tracer_particles<part_simple, part_simple_info, 0><<<nrows, 128>>>(pcl, tracer_factor, lc, (Real) dist, inner, outer, dtau, dtau_old, a, dadtau, boxsize, d_domain, fphi, d_vertex, vertexcount, posdata, veldata, ids, loginfo, 0, counters, counters + 1);
	if (!sync()) return release(-1);
	long count = total;

	// drop the check-zone particles logged in the previous cycle (:2065-2114);
	// the flagged selection is stable, as cub::DeviceSelect::Flagged is
	if (counters[0] > 0 && !bl.empty() && total > 0)
	{
		unsigned char * keep = (unsigned char *) managed(total);
		unsigned long long * selected = (unsigned long long *) managed(sizeof(unsigned long long) * total);
		float * cpos = (float *) managed(sizeof(float) * 3 * total);
		float * cvel = (float *) managed(sizeof(float) * 3 * total);
		long * cids = (long *) managed(sizeof(long) * total);
		unsigned char * clog = (unsigned char *) managed(total);
		if (failed) return release(-1);
		int blocks = std::min<long>((total + 255) / 256, 65535);
		mark_lightcone_kept_particles<<<blocks, 256>>>(ids, total, counters[0], d_backlog, (long) bl.size(), keep);
		if (!sync()) return release(-1);
		long kept = 0;
		for (long i = 0; i < total; i++)
			if (keep[i]) selected[kept++] = (unsigned long long) i;
		if (kept < total)
		{
			if (kept > 0)
			{
				blocks = std::min<long>((kept + 255) / 256, 65535);
				gather_lightcone_kept_particles<<<blocks, 256>>>(posdata, veldata, ids, loginfo, cpos, cvel, cids, clog, selected, kept);
				if (!sync()) return release(-1);
			}
			posdata = cpos; veldata = cvel; ids = cids; loginfo = clog;
			count = kept;
		}
	}
	*n_out = count;

	// the ID log for the next cycle, bin by bin (:2118-2165)
	long nlog = 0;
	if (count > 0)
	{
		const int log_bins = idlog_scatter ? 9 : 1;
		unsigned long long * bins = (unsigned long long *) managed(sizeof(unsigned long long) * 27);
		long * logged = (long *) managed(sizeof(long) * count);
		if (failed) return release(-1);
		for (int b = 0; b < 27; b++) bins[b] = 0;
		const int blocks = std::min<long>((count + 255) / 256, 65535);
		count_lightcone_prelog_bins<<<blocks, 256>>>(loginfo, count, log_bins, bins);
		if (!sync()) return release(-1);
		for (int b = 0; b < log_bins; b++) { bins[9 + b] = (unsigned long long) nlog; nlog += (long) bins[b]; }
		if (nlog > 0)
		{
			fill_lightcone_prelog_bins<<<blocks, 256>>>(ids, loginfo, count, log_bins, bins + 9, bins + 18, logged);
			if (!sync()) return release(-1);
		}
		if (nlog <= capacity)
			for (long i = 0; i < nlog; i++) prelog[i] = logged[i];
	}
	*n_prelog = nlog;
	if (count > capacity || nlog > capacity) return release(-2);
	for (long i = 0; i < count; i++)
	{
		for (int k = 0; k < 3; k++) { out_pos[3 * i + k] = posdata[3 * i + k]; out_vel[3 * i + k] = veldata[3 * i + k]; }
		out_id[i] = ids[i];
	}
	return release(0);
}

// One cycle of main.cu's loop (main.cu:608-1317) for CDM in the weak-field GR
// gauge with the elliptic vector method, no radiation, ncdm, baryons or
// output, composed from the reference's own functors and functions:
//   T00, Tij projections with the previous phi   main.cu:616-623, :750-756
//   prepareFTsource (T00) + FFT + solveModifiedPoissonFT + FFT^-1
//                                                 main.cu:719-809
//   prepareFTsource (Tij) + 6 FFTs + projectFTscalar + FFT^-1
//                                                 main.cu:811-903
//   T0i projection with the new phi + 3 FFTs + projectFTvector + 3 FFT^-1
//                                                 main.cu:836-955
//   updateVel(update_q), rungekutta4bg, moveParticles(update_pos),
//   rungekutta4bg, maxvel, step control          main.cu:1225-1310
// sim and st have the layouts of orc_sim and orc_state (oracle.h); pos and q
// are advanced in place (particle p has ID p), phi, chi and Bi are the
// persistent fields.

// transforms used by ref_step, with the conventions of orc_r2c / orc_c2r
// (unnormalised, half spectrum kx + (N/2+1)(ky + N kz)); null restores those
void ref_set_fft(ref_fft_fn r2c, ref_fft_fn c2r)
{
	g_r2c = r2c ? r2c : orc_r2c;
	g_c2r = c2r ? c2r : orc_c2r;
}

void ref_step(const orc_sim * sim, orc_state * st, int64_t np, double * pos, double * q, double * phi, double * chi, double * Bi)
{
	const int N = sim->N;
	const int64_t n3 = (int64_t) N * N * N, nk = (int64_t) (N / 2 + 1) * N * N;
	const double dx = 1. / N;
	const double fourpiG = sim->fourpiG;
	const cosmology cosmo = make_cosmo(sim->cosmo.Omega_m, sim->cosmo.Omega_Lambda, sim->cosmo.Omega_rad);
	double a = st->a;

	ParticleSet ps(N, np, pos, q, sim->mass);
	Lattice klat(N, true);
	std::vector<double> source(n3, 0.), Sij(6 * n3, 0.);
	std::vector<Imag> FT(6 * nk);
	Field<Real> fsource(ps.lat, source.data(), 1), fphi(ps.lat, phi, 1), fchi(ps.lat, chi, 1);
	Field<Real> fSij(ps.lat, Sij.data(), 6, symmetric), fBi(ps.lat, Bi, 3);
	Field<Imag> fscalar(klat, FT.data(), 1), fSijFT(klat, FT.data(), 6, symmetric), fBiFT(klat, FT.data(), 3);
	double * ft = reinterpret_cast<double *>(FT.data());

	// stress-energy: projection_T00_project(&pcls_cdm, &source, a, &phi) and
	// projection_Tij_project_Async with f_params {a, 1}
	{
		Field<Real> * f[2] = {&fsource, &fphi};
		double params[2] = {a, 1.};
		ps.pcls.projectParticles(particle_T00_project_functor(), f, 2, params);
	}
	{
		Field<Real> * f[2] = {&fSij, &fphi};
		double params[7] = {a, 1., 0., 0., 0., 0., 0.};
		ps.pcls.projectParticles(particle_Tij_project_functor(), f, 2, params);
	}

	// phi update
	if (st->dtau_old > 0.)
	{
		const double H = Hconf(a, fourpiG, cosmo);
		Field<Real> * f[4] = {&fsource, &fsource, &fphi, &fchi};
		double params[4] = {cosmo.Omega_cdm + cosmo.Omega_b, 3. * H * dx * dx / st->dtau_old, fourpiG * dx * dx / a, 3. * H * H * dx * dx};
		double sum = 0.;
#pragma omp parallel for collapse(2) reduction(+ : sum) schedule(static)
		for (int z = 0; z < N; z++)
			for (int y = 0; y < N; y++)
				for (int x = 0; x < N; x++)
				{
					Site s(ps.lat, x, y, z);
					Site sites[4] = {s, s, s, s};
					double out[1];
					prepareFTsource_T00(f, sites, 4, params, out);
					sum += out[0];
				}
		st->T00hom = sum / (double) n3;
		g_r2c(N, source.data(), ft);
		solveModifiedPoissonFT(fscalar, fscalar, 1. / (dx * dx), 3. * H / st->dtau_old);
		st->phi_hom = ft[0];
		g_c2r(N, ft, phi);
	}

	// chi: prepareFTsource(phi, Sij, Sij, 2 fourpiG dx^2 / a), projectFTscalar
	{
		Field<Real> * f[3] = {&fSij, &fSij, &fphi};
		double coeff = 2. * fourpiG * dx * dx / a;
		site_loop(N, [&](int x, int y, int z) {
			Site s(ps.lat, x, y, z);
			Site sites[3] = {s, s, s};
			prepareFTsource_Tij(f, sites, 3, &coeff, nullptr);
		});
		for (int c = 0; c < 6; c++) g_r2c(N, Sij.data() + c * n3, ft + 2 * c * nk);
		std::vector<Imag> chiFT(nk);
		Field<Imag> fchiFT(klat, chiFT.data(), 1);
		projectFTscalar(fSijFT, fchiFT);
		g_c2r(N, reinterpret_cast<double *>(chiFT.data()), chi);
	}

	// B_i, elliptic: projection_T0i_project_Async with the new phi, projectFTvector
	if (sim->with_B)
	{
		std::fill(Bi, Bi + 3 * n3, 0.);
		Field<Real> * f[2] = {&fBi, &fphi};
		double coeff = 1.;
		ps.pcls.projectParticles(particle_T0i_project_functor(), f, 2, &coeff);
		for (int c = 0; c < 3; c++) g_r2c(N, Bi + c * n3, ft + 2 * c * nk);
		projectFTvector(fBiFT, fBiFT, fourpiG * dx * dx);
		for (int c = 0; c < 3; c++) g_c2r(N, ft + 2 * c * nk, Bi + c * n3);
	}

	// particle update and background
	{
		Field<Real> * f[3] = {&fphi, &fchi, &fBi};
		double params[7] = {a, a * a * N, 0., 0., 0., 0., 0.};
		double mv = ps.pcls.updateVel(update_q_functor(), (st->dtau + st->dtau_old) / 2., f, (1. / a < sim->z_relax + 1. ? 3 : 2), params);
		rungekutta4bg(a, fourpiG, cosmo, 0.5 * st->dtau);
		params[0] = a;
		params[1] = a * a * N;
		ps.pcls.moveParticles(update_pos_functor(), st->dtau, f, (1. / a < sim->z_relax + 1. ? 3 : 0), params);
		rungekutta4bg(a, fourpiG, cosmo, 0.5 * st->dtau);
		st->maxvel = mv / sqrt(mv * mv + 1.0);
	}
	for (int64_t p = 0; p < np; p++)
		for (int i = 0; i < 3; i++)
		{
			pos[3 * p + i] = ps.parts[p].pos[i];
			q[3 * p + i] = ps.parts[p].vel[i];
		}

	// step control
	st->tau += st->dtau;
	st->dtau_old = st->dtau;
	const double Hn = Hconf(a, fourpiG, cosmo);
	st->dtau = (sim->Cf * dx < sim->steplimit / Hn) ? sim->Cf * dx : sim->steplimit / Hn;
	st->a = a;
	st->cycle++;
}

} // extern "C"
