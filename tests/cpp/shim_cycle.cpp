// Two PM cycles written in main.cu's call order against include/gev_shim.hpp,
// compared with the same cycles run by gev_step on a second context.
// Prints the largest relative differences; exit status 0 when they are within
// the FP64 tolerance.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "gev_shim.hpp"

namespace b = gev_b200;

static double maxrel(const std::vector<double> &x, const std::vector<double> &y)
{
    double m = 0., s = 1e-300;
    for (size_t i = 0; i < x.size(); i++) { m = std::fmax(m, std::fabs(x[i] - y[i])); s = std::fmax(s, std::fabs(y[i])); }
    return m / s;
}

int main()
{
    const int N = 32;
    const int64_t n = (int64_t)N * N * N;
    const double box = 160.0, Om = 0.32, fourpiG = 1.5 * box * box / (2997.92458 * 2997.92458);
    gev_cosmo cosmo{Om, 1.0 - Om, 0.0, fourpiG, 48.0, 0.04, 100.0, box};
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> u(-0.3, 0.3);
    std::vector<double> pos(3 * n), q(3 * n);
    std::vector<int64_t> id(n);
    for (int64_t i = 0; i < n; i++) {
        const int64_t c[3] = {i % N, (i / N) % N, i / ((int64_t)N * N)};
        for (int k = 0; k < 3; k++) {
            pos[3 * i + k] = (c[k] + 0.5 + u(rng)) / N;
            q[3 * i + k] = 1e-4 * u(rng);
        }
        id[i] = i;
    }
    const double mass = Om / n;
    try {
        b::Cycle shim(N, box, n, false, true), ref(N, box, n, false, true);
        b::particles_set(shim, pos.data(), q.data(), id.data(), n, mass);
        b::particles_set(ref, pos.data(), q.data(), id.data(), n, mass);
        const double a0 = 1.0 / 101.0, dx = 1.0 / N;
        gev_state st{a0, gev_particle_horizon(a0, fourpiG, &cosmo), 0., 0., 0, 0., 0., 0.};
        st.dtau = std::fmin(cosmo.Cf * dx, cosmo.steplimit / b::Hconf(a0, fourpiG, cosmo));
        double a = st.a, dtau = st.dtau, dtau_old = 0.;
        for (int cycle = 0; cycle < 2; cycle++) {
            // the shim, in main.cu's order
            b::projection_T00_Tij_project(shim, a, true);
            const double H = b::Hconf(a, fourpiG, cosmo);
            if (dtau_old > 0.)
                b::phi_update(shim, true, Om, 3. * H * dx * dx / dtau_old, fourpiG * dx * dx / a, 3. * H * H * dx * dx,
                              1. / (dx * dx), 3. * H / dtau_old);
            b::chi_update(shim, 2. * fourpiG * dx * dx / a, cycle == 0, H, dtau, dtau_old, a * a * dtau_old);
            b::projection_T0i_project(shim, true);
            b::B_update(shim, fourpiG * dx * dx);
            const int nk = (1. / a < cosmo.z_relax + 1.) ? 3 : 2;
            b::updateVel(shim, 0.5 * (dtau + dtau_old), nk, a, a * a * N);
            b::rungekutta4bg(a, fourpiG, cosmo, 0.5 * dtau);
            const int nd = (1. / a < cosmo.z_relax + 1.) ? 3 : 0;
            b::moveParticles(shim, dtau, nd, a, a * a * N);
            b::rungekutta4bg(a, fourpiG, cosmo, 0.5 * dtau);
            dtau_old = dtau;
            dtau = std::fmin(cosmo.Cf * dx, cosmo.steplimit / b::Hconf(a, fourpiG, cosmo));
            // the library's own cycle
            b::check(ref.ctx(), gev_step(ref.ctx(), &cosmo, &st));
        }
        std::vector<double> p1(3 * n), q1(3 * n), p2(3 * n), q2(3 * n), f1(n), f2(n);
        std::vector<int64_t> i1(n), i2(n);
        int64_t got = 0;
        b::check(shim.ctx(), gev_particles_get(shim.ctx(), p1.data(), q1.data(), i1.data(), n, &got));
        b::check(ref.ctx(), gev_particles_get(ref.ctx(), p2.data(), q2.data(), i2.data(), n, &got));
        // both sets come back in bucket order; compare by ID
        std::vector<double> ps(3 * n), qs(3 * n), pr(3 * n), qr(3 * n);
        for (int64_t i = 0; i < n; i++)
            for (int k = 0; k < 3; k++) {
                ps[3 * i1[i] + k] = p1[3 * i + k]; qs[3 * i1[i] + k] = q1[3 * i + k];
                pr[3 * i2[i] + k] = p2[3 * i + k]; qr[3 * i2[i] + k] = q2[3 * i + k];
            }
        b::check(shim.ctx(), gev_field_get(shim.ctx(), GEV_FIELD_PHI, f1.data()));
        b::check(ref.ctx(), gev_field_get(ref.ctx(), GEV_FIELD_PHI, f2.data()));
        const double dp = maxrel(ps, pr), dq = maxrel(qs, qr), dphi = maxrel(f1, f2), da = std::fabs(a / st.a - 1.);
        std::printf("shim vs gev_step after 2 cycles: pos %.3e  q %.3e  phi %.3e  a %.3e\n", dp, dq, dphi, da);
        return (dp < 1e-12 && dq < 1e-10 && dphi < 1e-10 && da < 1e-14) ? 0 : 1;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
}
