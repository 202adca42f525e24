// Cycles of gevolution-2.0's main loop written with the reference's per-cycle
// calls (include/gev_latfield.hpp: projection_*_project, prepareFTsource,
// PlanFFT::execute, solveModifiedPoissonFT, projectFTscalar / projectFTvector
// / evolveFTvector, projectFTtensor / evolveFTtensor, updateVel,
// moveParticles, Hconf, rungekutta4bg), in main.cu's order, against the same
// cycles run by gev_step on a second box.  Two configurations: FP64 with the
// elliptic vector method, and mixed precision with the parabolic method and the
// tensor state.  Exit status 0 when the particles and fields agree.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unistd.h>
#include <random>
#include <vector>

#include "gev_latfield.hpp"

namespace {

// the fields of the reference's cosmology struct that the background reads
struct Cosmology {
    double Omega_cdm, Omega_b, Omega_m, Omega_Lambda, Omega_fld, w0_fld, wa_fld, Omega_rad;
    int num_ncdm;
};

double maxrel(const std::vector<double> &x, const std::vector<double> &y)
{
    double m = 0., s = 1e-300;
    for (size_t i = 0; i < x.size(); i++) {
        m = std::fmax(m, std::fabs(x[i] - y[i]));
        s = std::fmax(s, std::fabs(y[i]));
    }
    return m / s;
}

// tol_hom: the zero mode phi_hom is the mean of the prepared source over
// N^3 points, which nearly cancels (the background model is subtracted); in
// FP32 its relative rounding is far above that of the fields
int run(bool mixed, bool elliptic, bool tensor, double tol_pos, double tol_field, double tol_hom)
{
    const int N = 32, ncycles = 3;
    const int64_t n = (int64_t)N * N * N;
    const double boxsize = 160.0, dx = 1.0 / N;
    const double fourpiG = 1.5 * boxsize * boxsize / (2997.92458 * 2997.92458);
    Cosmology cosmo{0.27, 0.05, 0.32, 0.68, 0., -1., 0., 0., 0};
    const double z_relax = 100.;

    std::mt19937_64 rng(11);
    std::uniform_real_distribution<double> u(-0.3, 0.3);
    std::vector<double> pos(3 * n), q(3 * n);
    std::vector<int64_t> id(n);
    for (int64_t i = 0; i < n; i++) {
        const int64_t c[3] = {i % N, (i / N) % N, i / ((int64_t)N * N)};
        for (int k = 0; k < 3; k++) {
            pos[3 * i + k] = (c[k] + 0.5 + u(rng)) / N;
            q[3 * i + k] = 2e-4 * u(rng);
        }
        id[i] = i;
    }
    const double mass = cosmo.Omega_m / n;

    // the reference's objects, on a box of the library
    gev_b200::Box box(N, boxsize, n, mixed, elliptic, tensor);
    Field<Real> phi(box, GEV_FIELD_PHI), chi(box, GEV_FIELD_CHI), source(box, GEV_FIELD_SOURCE), Sij(box, GEV_FIELD_SIJ),
        Bi(box, GEV_FIELD_BI);
    Field<Imag> scalarFT(box, FT_SCALAR), SijFT(box, FT_SIJ), BiFT(box, FT_BI), hijFT(box, FT_HIJ), hijprimeFT(box, FT_HIJPRIME);
    PlanFFT<Imag> plan_source(&source, &scalarFT), plan_phi(&phi, &scalarFT), plan_chi(&chi, &scalarFT), plan_Sij(&Sij, &SijFT),
        plan_Bi(&Bi, &BiFT);
    perfParticles_gevolution<part_simple, part_simple_info> pcls_cdm(box);
    pcls_cdm.initialize(pos.data(), q.data(), id.data(), n, mass);
    Field<Real> *project_Tij_fields[2] = {&Sij, &phi};
    Field<Real> *project_T0i_fields[2] = {&Bi, &phi};
    Field<Real> *update_cdm_fields[3] = {&phi, &chi, &Bi};
    double f_params[7] = {0., 0., 0., 0., 0., 0., 0.};
    DeviceStagingBuffer<double> d_f_params(7);
    rKSite kFT;

    // the library's own cycle on a second box
    gev_b200::Cycle ref(N, boxsize, n, mixed, elliptic, tensor);
    gev_b200::particles_set(ref, pos.data(), q.data(), id.data(), n, mass);
    const gev_cosmo gc{cosmo.Omega_cdm + cosmo.Omega_b, cosmo.Omega_Lambda, cosmo.Omega_rad, fourpiG, 48.0, 0.04, z_relax, boxsize};

    double a = 1.0 / 51.0, tau = particleHorizon(a, fourpiG, cosmo), dtau_old = 0.;
    double dtau = std::fmin(48.0 * dx, 0.04 / Hconf(a, fourpiG, cosmo));
    gev_state st{a, tau, dtau, 0., 0, 0., 0., 0.};
    double T00hom = 0., maxvel = 0.;
    Real phi_hom = 0.;
    for (int cycle = 0; cycle < ncycles; cycle++) {
        // stress-energy with the previous phi
        projection_T00_project(&pcls_cdm, &source, a, &phi);
        projection_T00_comm(&source);
        // phi
        if (dtau_old > 0.) {
            T00hom = prepareFTsource(phi, chi, source, cosmo.Omega_cdm + cosmo.Omega_b, source,
                                     3. * Hconf(a, fourpiG, cosmo) * dx * dx / dtau_old, fourpiG * dx * dx / a,
                                     3. * Hconf(a, fourpiG, cosmo) * Hconf(a, fourpiG, cosmo) * dx * dx);
            T00hom /= (double)n;
            plan_source.execute(FFT_FORWARD);
        }
        f_params[0] = a;
        f_params[1] = 1.;
        d_f_params.copy_from_host(f_params, 7);
        projection_Tij_project_Async(&pcls_cdm, project_Tij_fields, 2, d_f_params.data());
        if (dtau_old > 0.) solveModifiedPoissonFT(scalarFT, scalarFT, 1. / (dx * dx), 3. * Hconf(a, fourpiG, cosmo) / dtau_old);
        projection_Tij_comm(&Sij);
        if (dtau_old > 0.) {
            plan_phi.execute(FFT_BACKWARD);
            phi.updateHalo();
            if (kFT.setCoord(0, 0, 0)) phi_hom = scalarFT(kFT).real();
        }
        // chi and the T0i projection with the new phi
        prepareFTsource(phi, Sij, Sij, 2. * fourpiG * dx * dx / a);
        plan_Sij.execute(FFT_FORWARD);
        if (elliptic) {
            f_params[0] = 1.;
            d_f_params.copy_from_host(f_params, 1);
            projection_T0i_project_Async(&pcls_cdm, project_T0i_fields, 2, d_f_params.data());
        }
        projectFTscalar(SijFT, scalarFT);
        if (elliptic) projection_T0i_comm(&Bi);
        plan_chi.execute(FFT_BACKWARD);
        chi.updateHalo();
        // B
        if (elliptic) {
            plan_Bi.execute(FFT_FORWARD);
            projectFTvector(BiFT, BiFT, fourpiG * dx * dx);
        } else {
            evolveFTvector(SijFT, BiFT, a * a * dtau_old);
        }
        plan_Bi.execute(FFT_BACKWARD);
        Bi.updateHalo();
        if (tensor) {
            if (cycle == 0) projectFTtensor(SijFT, hijFT);
            else evolveFTtensor(SijFT, hijFT, hijprimeFT, Hconf(a, fourpiG, cosmo), dtau, dtau_old);
        }
        // particle update
        f_params[0] = a;
        f_params[1] = a * a * N;
        d_f_params.copy_from_host(f_params, 7);
        maxvel = pcls_cdm.updateVel(update_q_functor(), (dtau + dtau_old) / 2., update_cdm_fields, (1. / a < z_relax + 1. ? 3 : 2),
                                    d_f_params.data());
        rungekutta4bg(a, fourpiG, cosmo, 0.5 * dtau);
        f_params[0] = a;
        f_params[1] = a * a * N;
        d_f_params.copy_from_host(f_params, 7);
        pcls_cdm.moveParticles(update_pos_functor(), dtau, update_cdm_fields, (1. / a < z_relax + 1. ? 3 : 0), d_f_params.data());
        rungekutta4bg(a, fourpiG, cosmo, 0.5 * dtau);
        maxvel /= std::sqrt(maxvel * maxvel + 1.0);
        tau += dtau;
        dtau_old = dtau;
        dtau = std::fmin(48.0 * dx, 0.04 / Hconf(a, fourpiG, cosmo));

        gev_b200::check(ref.ctx(), gev_step(ref.ctx(), &gc, &st));
    }

    // the particles through an express file (saveExpress / loadExpress) and back
    {
        gev_gadget2_header hdr;
        std::memset(&hdr, 0, sizeof hdr);
        hdr.num_files = 1;
        hdr.time = a;
        char name[] = "/tmp/gev_latfield_express_XXXXXX";
        const int fd = mkstemp(name);
        if (fd < 0) throw std::runtime_error("mkstemp");
        close(fd);
        pcls_cdm.saveExpress(name, hdr);
        gev_gadget2_header back;
        pcls_cdm.loadExpress(name, back);
        std::remove(name);
        std::remove((std::string(name) + ".0").c_str());
        if (back.time != a || back.npartTotal[1] != (uint32_t)n) throw std::runtime_error("express header mismatch");
    }

    std::vector<double> p1(3 * n), q1(3 * n), p2(3 * n), q2(3 * n);
    std::vector<int64_t> i1(n), i2(n);
    int64_t got = 0;
    gev_b200::check(box.ctx(), gev_particles_get(box.ctx(), p1.data(), q1.data(), i1.data(), n, &got));
    gev_b200::check(ref.ctx(), gev_particles_get(ref.ctx(), p2.data(), q2.data(), i2.data(), n, &got));
    std::vector<double> ps(3 * n), qs(3 * n), pr(3 * n), qr(3 * n);
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            ps[3 * i1[i] + k] = p1[3 * i + k];
            qs[3 * i1[i] + k] = q1[3 * i + k];
            pr[3 * i2[i] + k] = p2[3 * i + k];
            qr[3 * i2[i] + k] = q2[3 * i + k];
        }
    double dp = 0.;
    for (int64_t i = 0; i < 3 * n; i++) {
        double d = ps[i] - pr[i];
        d -= std::round(d);
        dp = std::fmax(dp, std::fabs(d) * N);
    }
    std::vector<double> f1(n), f2(n), c1(n), c2(n), b1(3 * n), b2(3 * n);
    phi.copy_to_host(f1.data());
    chi.copy_to_host(c1.data());
    Bi.copy_to_host(b1.data());
    gev_b200::check(ref.ctx(), gev_field_get(ref.ctx(), GEV_FIELD_PHI, f2.data()));
    gev_b200::check(ref.ctx(), gev_field_get(ref.ctx(), GEV_FIELD_CHI, c2.data()));
    gev_b200::check(ref.ctx(), gev_field_get(ref.ctx(), GEV_FIELD_BI, b2.data()));
    double dh = 0.;
    if (tensor) {
        const int64_t nk = (int64_t)(N / 2 + 1) * N * N;
        std::vector<double> h1(12 * nk), h2(12 * nk);
        gev_b200::check(box.ctx(), gev_field_get(box.ctx(), GEV_FIELD_HIJP_FT, h1.data()));
        gev_b200::check(ref.ctx(), gev_field_get(ref.ctx(), GEV_FIELD_HIJP_FT, h2.data()));
        dh = maxrel(h1, h2);
    }
    const double dq = maxrel(qs, qr), dphi = maxrel(f1, f2), dchi = maxrel(c1, c2), dB = maxrel(b1, b2);
    const double da = std::fabs(a / st.a - 1.), dv = std::fabs(maxvel / st.maxvel - 1.), dT = std::fabs(T00hom / st.T00hom - 1.);
    const double dph = std::fabs(phi_hom - st.phi_hom) / std::fmax(std::fabs(st.phi_hom), 1e-300);
    std::printf("%s %s%s: pos %.2e q %.2e phi %.2e chi %.2e B %.2e h' %.2e a %.1e maxvel %.1e T00hom %.1e phi_hom %.1e\n",
                mixed ? "mixed" : "fp64", elliptic ? "elliptic" : "parabolic", tensor ? " tensor" : "", dp, dq, dphi, dchi, dB,
                dh, da, dv, dT, dph);
    const bool ok = dp < tol_pos && dq < tol_field && dphi < tol_field && dchi < tol_field && dB < tol_field && dh < tol_field &&
                    da < 1e-14 && dv < tol_field && dT < tol_field && dph < tol_hom;
    return ok ? 0 : 1;
}

}  // namespace

int main()
{
    try {
        int rc = run(false, true, false, 1e-10, 1e-10, 1e-9);
        rc |= run(true, false, true, 1e-5, 1e-4, 1e-2);
        return rc;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
}
