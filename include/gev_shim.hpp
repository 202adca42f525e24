// gev_shim.hpp -- C++ binding of include/gev.h with gevolution-2.0's per-cycle
// call names and argument order, for a host code built like main.cu.  Every
// function forwards to one C ABI entry point; a failed call throws
// std::runtime_error with the library's message, the way the reference's CUDA
// checks do (main.cu:778-782).
#ifndef GEV_B200_SHIM_HPP
#define GEV_B200_SHIM_HPP

#include <cstdint>
#include <stdexcept>
#include <string>

#include "gev.h"

namespace gev_b200 {

inline void check(const gev_ctx *c, int rc)
{
    if (rc != GEV_OK) throw std::runtime_error(std::string("libgevb200: ") + gev_last_error(c));
}

// the fields, Fourier workspace, FFT plans and particle container of main.cu:298-385
class Cycle {
public:
    Cycle(int N, double boxsize, int64_t numpcl, bool mixed, bool elliptic, bool tensor = false, int device = 0)
    {
        gev_config cfg{};
        cfg.N = N;
        cfg.precision = mixed ? GEV_MIXED : GEV_FP64;
        cfg.capacity = numpcl;
        cfg.boxsize = boxsize;
        cfg.vector_method = elliptic ? GEV_VECTOR_ELLIPTIC : GEV_VECTOR_PARABOLIC;
        cfg.tensor = tensor ? 1 : 0;
        cfg.device = device;
        check(nullptr, gev_ctx_create(&cfg, &ctx_));
    }
    ~Cycle() { gev_ctx_destroy(ctx_); }
    Cycle(const Cycle &) = delete;
    Cycle &operator=(const Cycle &) = delete;
    gev_ctx *ctx() const { return ctx_; }

private:
    gev_ctx *ctx_ = nullptr;
};

// perfParticles::initialize + addParticle_global + updateRowBuffers (ic_basic.hpp:2206-2211)
inline void particles_set(Cycle &c, const double *pos, const double *q, const int64_t *id, int64_t n, double mass)
{
    check(c.ctx(), gev_particles_set(c.ctx(), pos, q, id, n, mass));
}

// projection_T00_project + projection_Tij_project(_Async) + comm (gevolution.hpp:1887, :2999, :3030; main.cu:616-700)
inline void projection_T00_Tij_project(Cycle &c, double a, bool with_phi, double coeff = 1.)
{
    check(c.ctx(), gev_project(c.ctx(), GEV_PROJ_T00 | GEV_PROJ_TIJ, a, coeff, with_phi ? 1 : 0, 0));
}

// projection_T0i_project + comm (gevolution.hpp:2232; main.cu:836-887)
inline void projection_T0i_project(Cycle &c, bool with_phi, double coeff = 1.)
{
    check(c.ctx(), gev_project(c.ctx(), GEV_PROJ_T0I, 1., coeff, with_phi ? 1 : 0, 0));
}

// scalarProjectionCIC_project (gevolution.hpp:1902)
inline void scalarProjectionCIC_project(Cycle &c, double coeff = 1.)
{
    check(c.ctx(), gev_project(c.ctx(), GEV_PROJ_CIC, 1., coeff, 0, 0));
}

// prepareFTsource (gevolution.hpp:183) + FFT + solveModifiedPoissonFT (:806) + FFT^-1 (main.cu:719-809);
// returns the sum of T00 (prepareFTsource's return value)
inline double phi_update(Cycle &c, bool prepare, double bgmodel, double coeff, double coeff2, double coeff3,
                         double poisson_coeff, double modif, double *phi_hom = nullptr)
{
    double sum = 0., ph = 0.;
    check(c.ctx(), gev_solve_phi(c.ctx(), prepare ? 1 : 0, bgmodel, coeff, coeff2, coeff3, poisson_coeff, modif, &sum, &ph));
    if (phi_hom) *phi_hom = ph;
    return sum;
}

// prepareFTsource(phi, Sij, Sij, coeff) (:119) + FFTs + projectFTscalar (:251) (+ tensor, parabolic B) (main.cu:811-966)
inline void chi_update(Cycle &c, double coeff, bool cycle0, double hubble, double dtau, double dtau_old, double a2dtau)
{
    check(c.ctx(), gev_solve_chi(c.ctx(), coeff, cycle0 ? 1 : 0, hubble, dtau, dtau_old, a2dtau));
}

// FFT + projectFTvector (:449) + FFT^-1 (main.cu:918-955)
inline void B_update(Cycle &c, double coeff, double modif = 0.)
{
    check(c.ctx(), gev_solve_B(c.ctx(), coeff, modif));
}

// perfParticles::updateVel(update_q_functor, dtau, fields, nfield, {a, a^2 N}) (main.cu:1230-1235); returns maxvel
inline double updateVel(Cycle &c, double dtau, int nfield, double a, double a2N)
{
    double maxvel = 0.;
    check(c.ctx(), gev_kick(c.ctx(), dtau, a, a2N, nfield, &maxvel));
    return maxvel;
}

// perfParticles::moveParticles(update_pos_functor, dtau, fields, nfield, {a, a^2 N}) (main.cu:1256-1262)
inline void moveParticles(Cycle &c, double dtau, int nfield, double a, double a2N)
{
    check(c.ctx(), gev_drift(c.ctx(), dtau, a, a2N, nfield));
}

// Hconf / rungekutta4bg (background.hpp:200-244)
inline double Hconf(double a, double fourpiG, const gev_cosmo &cosmo) { return gev_hconf(a, fourpiG, &cosmo); }
inline void rungekutta4bg(double &a, double fourpiG, const gev_cosmo &cosmo, double dtau)
{
    gev_rungekutta4bg(&a, fourpiG, &cosmo, dtau);
}

}  // namespace gev_b200

#endif
