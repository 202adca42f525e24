// gev_latfield.hpp -- gevolution-2.0's per-cycle interface on libgevb200.
//
// The types (Field, PlanFFT, rKSite, perfParticles, DeviceStagingBuffer) and
// free functions that the reference's main loop calls (main.cu:608-1317), with
// the reference's names, argument lists and defaults:
//
//   projection_T00_project(perfParticles*, Field<Real>* T00, double a = 1., Field<Real>* phi = nullptr, double coeff = 1.)
//                                                           gevolution.hpp:1887
//   projection_T0i_project(perfParticles*, Field<Real>* T0i, Field<Real>* phi = nullptr, double coeff = 1.)     :2232
//   projection_T0i_project_Async(perfParticles*, Field<Real>** fields, int nfield, double* params)             :2242
//   projection_Tij_project(perfParticles*, Field<Real>* Tij, double a = 1., Field<Real>* phi = nullptr,
//                          double coeff = 1., Real* hij_hom = nullptr)                                        :2999
//   projection_Tij_project_Async(perfParticles*, Field<Real>** fields, int nfield, double* params)             :3030
//   projection_T00_comm / projection_T0i_comm / projection_Tij_comm(Field<Real>*)                 :1726, :2028, :2573
//   scalarProjectionCIC_project(perfParticles*, Field<Real>*)                                                 :1902
//   prepareFTsource(Field<Real>& phi, Field<Real>& Tij, Field<Real>& Sij, double coeff)                        :119
//   double prepareFTsource(Field<Real>& phi, Field<Real>& chi, Field<Real>& source, double bgmodel,
//                          Field<Real>& result, double coeff, double coeff2, double coeff3)                    :183
//   solveModifiedPoissonFT(Field<Imag>& src, Field<Imag>& pot, Real coeff, Real modif = 0)                     :806
//   projectFTscalar(Field<Imag>& SijFT, Field<Imag>& chiFT, int add = 0)                                       :251
//   projectFTvector(Field<Imag>& SiFT, Field<Imag>& BiFT, Real coeff = 1, Real modif = 0)                       :449
//   evolveFTvector(Field<Imag>& SijFT, Field<Imag>& BiFT, Real a2dtau)                                         :359
//   projectFTtensor(Field<Imag>& SijFT, Field<Imag>& hijFT)                                                    :693
//   evolveFTtensor(Field<Imag>& SijFT, Field<Imag>& hijFT, Field<Imag>& hijprimeFT, double hubble,
//                  double dtau, double dtau_old)                                                               :537
//   perfParticles::updateVel(update_q_functor(), dtau, fields, nfield, params) -> max velocity        main.cu:1232
//   perfParticles::moveParticles(update_pos_functor(), dtau, fields, nfield, params)                   main.cu:1258
//   perfParticles_gevolution::saveGadget2 (snapshot and lightcone forms), loadGadget2,
//   saveExpress, loadExpress
//                                                                                  Particles_gevolution.hpp:180-183
//   PlanFFT<Imag>::execute(FFT_FORWARD | FFT_BACKWARD), Field<Real>::updateHalo()
//   Hconf, rungekutta4bg, particleHorizon                                          background.hpp:200, :235, :268
//
// How the calls map onto the library.  The library fuses each Fourier solve
// (source preparation, forward transform, k-space solver, backward transform)
// into one call on fields that live on the GPU, so a Box records what the
// reference's sequence asks for and runs the fused solve when its result is
// needed:
//   - prepareFTsource (T00 form) runs at once (it returns the sum of T00):
//     gev_prepare_T00;
//   - plan_source.execute(FFT_FORWARD), solveModifiedPoissonFT(scalarFT, ...)
//     are recorded, plan_phi.execute(FFT_BACKWARD) runs gev_solve_phi, and
//     scalarFT(kFT) at k = 0 returns the zero mode (main.cu:808-809);
//   - prepareFTsource (Tij form), plan_Sij.execute(FFT_FORWARD),
//     projectFTscalar are recorded; plan_chi.execute(FFT_BACKWARD) runs
//     gev_solve_chi -- for the parabolic vector method or a box with the
//     tensor state, that runs at evolveFTvector / projectFTtensor /
//     evolveFTtensor, which supply its remaining parameters, or at the next
//     particle update;
//   - plan_Bi.execute(FFT_FORWARD) and projectFTvector are recorded,
//     plan_Bi.execute(FFT_BACKWARD) runs gev_solve_B;
//   - a projection overwrites its target field on the first projection of a
//     cycle (after the particle update, after a solve consumed the field, or
//     after zero(field)) and adds to it afterwards -- the reference zeroes the
//     targets with thrust::fill_n before projecting (main.cu:616, :681, :840),
//     which this header replaces;
//   - updateHalo and projection_*_comm do nothing: neighbours on one GPU come
//     from periodic indexing;
//   - DeviceStagingBuffer keeps its values in host memory; the functions above
//     read their params from it on the host.
// Only cold dark matter in the weak-field GR gauge is supported (one particle
// species; Hconf and friends refuse ncdm and fluid components); a request
// outside that (a Newtonian functor, projectFTscalar with add != 0, hij_hom,
// redshift-interpolated snapshots) throws std::runtime_error.
#ifndef GEV_B200_LATFIELD_HPP
#define GEV_B200_LATFIELD_HPP

#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "gev_shim.hpp"

#ifndef GEV_LATFIELD_REAL
#define GEV_LATFIELD_REAL double
#endif
typedef GEV_LATFIELD_REAL Real;

constexpr int FFT_FORWARD = 0;
constexpr int FFT_BACKWARD = 1;

class Imag {
public:
    Imag() = default;
    Imag(double re, double im) : re_(re), im_(im) {}
    double real() const { return re_; }
    double imag() const { return im_; }

private:
    double re_ = 0., im_ = 0.;
};

namespace gev_b200 {

// One simulation box: the library context plus the Fourier-space work that
// the reference's unfused call sequence has announced but not yet asked for.
class Box {
public:
    Box(int N, double boxsize, int64_t capacity, bool mixed, bool elliptic, bool tensor = false, int device = 0)
        : cycle_(N, boxsize, capacity, mixed, elliptic, tensor, device), N_(N), elliptic_(elliptic), tensor_(tensor)
    {
    }
    gev_ctx *ctx() const { return cycle_.ctx(); }
    int N() const { return N_; }
    bool elliptic() const { return elliptic_; }
    bool tensor() const { return tensor_; }

    // ---- phi ----
    void prepared_source() { src_prepared_ = true; }
    void source_forward() { src_forward_ = true; }
    void poisson(double coeff, double modif)
    {
        poisson_set_ = true;
        pc_ = coeff;
        modif_ = modif;
    }
    void phi_backward()
    {
        if (!src_forward_ || !poisson_set_)
            throw std::runtime_error("gev_latfield: phi backward transform without a forward transform and solveModifiedPoissonFT");
        double sum = 0., ph = 0.;
        check(ctx(), gev_solve_phi(ctx(), 0, 0., 0., 0., 0., pc_, modif_, &sum, &ph));
        phi_hom_ = ph;
        have_phi_hom_ = true;
        src_forward_ = poisson_set_ = src_prepared_ = false;
        consumed(GEV_FIELD_SOURCE);
    }
    double phi_hom() const
    {
        if (!have_phi_hom_) throw std::runtime_error("gev_latfield: the zero mode is known only after the phi update");
        return phi_hom_;
    }

    // ---- chi (and parabolic B, tensor) ----
    void tij_prepare(double coeff)
    {
        tij_coeff_ = coeff;
        tij_prepare_ = true;
    }
    void sij_forward() { sij_forward_ = true; }
    void scalar_projection() { chi_project_ = true; }
    void chi_backward()
    {
        chi_requested_ = true;
        if (elliptic_ && !tensor_) run_chi(false, 0., 0., 0.);
    }
    void vector_evolution(double a2dtau)
    {
        a2dtau_ = a2dtau;
        have_a2dtau_ = true;
        if (!tensor_ && chi_requested_) run_chi(false, 0., 0., 0.);
    }
    void tensor_step(bool cycle0, double hubble, double dtau, double dtau_old)
    {
        if (!tensor_) throw std::runtime_error("gev_latfield: the box was created without the tensor state");
        if (!chi_requested_) throw std::runtime_error("gev_latfield: projectFTtensor / evolveFTtensor before the Sij transform");
        run_chi(cycle0, hubble, dtau, dtau_old);
    }
    // a deferred chi solve runs before anything reads chi or B_i
    void flush()
    {
        if (chi_requested_) run_chi(false, 0., 0., 0.);
    }

    // ---- B_i (elliptic) ----
    void bi_forward() { bi_forward_ = true; }
    void vector_projection(double coeff, double modif)
    {
        vec_set_ = true;
        vc_ = coeff;
        vmodif_ = modif;
    }
    void bi_backward()
    {
        // parabolic: B_i comes out of the (possibly still deferred) chi solve;
        // elliptic: an independent solve, which leaves a deferred chi solve pending
        if (!elliptic_) return;
        if (!bi_forward_ || !vec_set_)
            throw std::runtime_error("gev_latfield: B backward transform without a forward transform and projectFTvector");
        check(ctx(), gev_solve_B(ctx(), vc_, vmodif_));
        bi_forward_ = vec_set_ = false;
        consumed(GEV_FIELD_BI);
    }

    // ---- projections ----
    // accumulate flag of the next projection into `field`
    int accumulate_into(int field)
    {
        const int acc = fresh_[field] ? 1 : 0;
        fresh_[field] = true;
        return acc;
    }
    void consumed(int field) { fresh_[field] = false; }
    // the particle update ends a cycle: the next cycle's projections start
    // from zero, as main.cu zeroes their targets at the top of its loop
    void cycle_end()
    {
        consumed(GEV_FIELD_SOURCE);
        consumed(GEV_FIELD_SIJ);
        consumed(GEV_FIELD_BI);
    }

    // backlog slot of a caller-side ID log (lightcone shells)
    int shell_of(const void *idlog)
    {
        auto it = shells_.find(idlog);
        if (it != shells_.end()) return it->second;
        const int s = (int)shells_.size();
        if (s >= 8) throw std::runtime_error("gev_latfield: at most 8 lightcone ID logs");
        shells_[idlog] = s;
        return s;
    }

private:
    void run_chi(bool cycle0, double hubble, double dtau, double dtau_old)
    {
        if (!tij_prepare_ || !sij_forward_ || !chi_project_)
            throw std::runtime_error("gev_latfield: chi transform without prepareFTsource, the Sij transform and projectFTscalar");
        if (!elliptic_ && !have_a2dtau_)
            throw std::runtime_error("gev_latfield: parabolic vector method without evolveFTvector");
        check(ctx(), gev_solve_chi(ctx(), tij_coeff_, cycle0 ? 1 : 0, hubble, dtau, dtau_old, have_a2dtau_ ? a2dtau_ : 0.));
        tij_prepare_ = sij_forward_ = chi_project_ = chi_requested_ = have_a2dtau_ = false;
        consumed(GEV_FIELD_SIJ);
        if (!elliptic_) consumed(GEV_FIELD_BI);
    }

    Cycle cycle_;
    int N_;
    bool elliptic_, tensor_;
    bool src_prepared_ = false, src_forward_ = false, poisson_set_ = false, have_phi_hom_ = false;
    double pc_ = 0., modif_ = 0., phi_hom_ = 0.;
    bool tij_prepare_ = false, sij_forward_ = false, chi_project_ = false, chi_requested_ = false, have_a2dtau_ = false;
    double tij_coeff_ = 0., a2dtau_ = 0.;
    bool bi_forward_ = false, vec_set_ = false;
    double vc_ = 0., vmodif_ = 0.;
    bool fresh_[8] = {false, false, false, false, false, false, false, false};
    std::map<const void *, int> shells_;
};

}  // namespace gev_b200

class Lattice {
public:
    explicit Lattice(int N = 0) : N_(N) {}
    long sitesLocalGross() const { return (long)N_ * N_ * N_; }
    int size(int) const { return N_; }

private:
    int N_;
};

// a wavenumber site; on one rank every coordinate is local
class rKSite {
public:
    bool setCoord(int kx, int ky, int kz)
    {
        k_[0] = kx;
        k_[1] = ky;
        k_[2] = kz;
        return true;
    }
    int coord(int i) const { return k_[i]; }

private:
    int k_[3] = {0, 0, 0};
};

template <class T> class Field;

// a real field of a Box: GEV_FIELD_PHI, _CHI, _SOURCE, _SIJ or _BI
template <> class Field<Real> {
public:
    Field(gev_b200::Box &box, int field) : box_(&box), id_(field), lat_(box.N()) {}
    gev_b200::Box &box() const { return *box_; }
    int id() const { return id_; }
    void updateHalo() {}
    const Lattice &lattice() const { return lat_; }
    int components() const { return gev_field_components(id_); }
    // copies between this field and host memory (components() planes of N^3 values)
    void copy_to_host(double *host) const { box_->flush(); gev_b200::check(box_->ctx(), gev_field_get(box_->ctx(), id_, host)); }
    void copy_from_host(const double *host)
    {
        gev_b200::check(box_->ctx(), gev_field_set(box_->ctx(), id_, host));
        box_->consumed(id_);
    }

private:
    gev_b200::Box *box_;
    int id_;
    Lattice lat_;
};

// the role of a Fourier field in main.cu: scalarFT, SijFT, BiFT, hijFT, hijprimeFT
enum FourierRole { FT_SCALAR, FT_SIJ, FT_BI, FT_HIJ, FT_HIJPRIME };

template <> class Field<Imag> {
public:
    Field(gev_b200::Box &box, FourierRole role) : box_(&box), role_(role) {}
    gev_b200::Box &box() const { return *box_; }
    FourierRole role() const { return role_; }
    // only the k = 0 mode of scalarFT after the phi update is addressable
    Imag operator()(const rKSite &k) const
    {
        if (role_ != FT_SCALAR || k.coord(0) || k.coord(1) || k.coord(2))
            throw std::runtime_error("gev_latfield: Fourier modes live on the GPU; only scalarFT at k = 0 is readable");
        return Imag(box_->phi_hom(), 0.);
    }

private:
    gev_b200::Box *box_;
    FourierRole role_;
};

template <class T> class PlanFFT;

template <> class PlanFFT<Imag> {
public:
    PlanFFT(Field<Real> *rfield, Field<Imag> *kfield) : r_(rfield), k_(kfield) {}
    void execute(int direction)
    {
        gev_b200::Box &b = r_->box();
        const int f = r_->id();
        if (direction == FFT_FORWARD) {
            if (f == GEV_FIELD_SOURCE && k_->role() == FT_SCALAR) b.source_forward();
            else if (f == GEV_FIELD_SIJ && k_->role() == FT_SIJ) b.sij_forward();
            else if (f == GEV_FIELD_BI && k_->role() == FT_BI) b.bi_forward();
            else throw std::runtime_error("gev_latfield: forward transform of an unsupported field pair");
        } else {
            if (f == GEV_FIELD_PHI && k_->role() == FT_SCALAR) b.phi_backward();
            else if (f == GEV_FIELD_CHI && k_->role() == FT_SCALAR) b.chi_backward();
            else if (f == GEV_FIELD_BI && k_->role() == FT_BI) b.bi_backward();
            else throw std::runtime_error("gev_latfield: backward transform of an unsupported field pair");
        }
    }

private:
    Field<Real> *r_;
    Field<Imag> *k_;
};

// parameters of a particle operation; kept in host memory
template <class T> class DeviceStagingBuffer {
public:
    explicit DeviceStagingBuffer(size_t n) : v_(n) {}
    DeviceStagingBuffer(const T *host, size_t n) : v_(host, host + n) {}
    void copy_from_host(const T *host, size_t n)
    {
        if (n > v_.size()) v_.resize(n);
        std::memcpy(v_.data(), host, n * sizeof(T));
    }
    T *data() { return v_.data(); }

private:
    std::vector<T> v_;
};

struct part_simple {
    Real pos[3];
    Real vel[3];
    long ID;
};
struct part_simple_info {
    double mass;
    int relativistic;
    char type_name[64];
};

// particle functors: tags selecting the library's kernels
struct update_q_functor {};
struct update_pos_functor {};
struct update_q_Newton_functor {};
struct update_pos_Newton_functor {};

template <class part, class part_info> class perfParticles {
public:
    perfParticles() = default;
    explicit perfParticles(gev_b200::Box &box) : box_(&box) {}
    void attach(gev_b200::Box &box) { box_ = &box; }
    gev_b200::Box &box() const
    {
        if (!box_) throw std::runtime_error("gev_latfield: particle container without a box");
        return *box_;
    }
    // the particles of the box (box units, momentum per unit mass; IDs may be null)
    void initialize(const double *pos, const double *q, const int64_t *ids, int64_t n, double mass)
    {
        mass_ = mass;
        gev_b200::check(box().ctx(), gev_particles_set(box().ctx(), pos, q, ids, n, mass));
    }
    // part_simple_info.mass of the particles loaded from files (the reference sets it after
    // loadGadget2, ic_read.hpp)
    void set_mass(double mass) { mass_ = mass; }
    double mass() const { return mass_; }
    long num_particles() const
    {
        int64_t n = 0;
        gev_b200::check(box().ctx(), gev_particles_count(box().ctx(), &n));
        return (long)n;
    }
    // updateVel(update_q_functor(), dtau, {phi, chi, Bi}, nfield, {a, a^2 N}): returns the maximum velocity
    Real updateVel(update_q_functor, double dtau, Field<Real> **, int nfield, double *params)
    {
        box().flush();
        box().cycle_end();
        double maxvel = 0.;
        gev_b200::check(box().ctx(), gev_kick(box().ctx(), dtau, params[0], params[1], nfield, &maxvel));
        return (Real)maxvel;
    }
    void moveParticles(update_pos_functor, double dtau, Field<Real> **, int nfield, double *params)
    {
        box().flush();
        box().cycle_end();
        gev_b200::check(box().ctx(), gev_drift(box().ctx(), dtau, params[0], params[1], nfield));
    }
    Real updateVel(update_q_Newton_functor, double, Field<Real> **, int, double *)
    {
        throw std::runtime_error("gev_latfield: the Newtonian particle update is not part of the GR cycle");
    }
    void moveParticles(update_pos_Newton_functor, double, Field<Real> **, int, double *)
    {
        throw std::runtime_error("gev_latfield: the Newtonian particle update is not part of the GR cycle");
    }

private:
    gev_b200::Box *box_ = nullptr;
    double mass_ = 0.;
};

template <class part, class part_info> class perfParticles_gevolution : public perfParticles<part, part_info> {
public:
    using perfParticles<part, part_info>::perfParticles;

    // particle file (Particles_gevolution.hpp:183): every particle of one
    // Gadget-2 file, with the mass given by set_mass / initialize
    template <class Header> void loadGadget2(std::string filename, Header &hdr)
    {
        gev_gadget2_header h;
        gev_b200::check(this->box().ctx(), gev_particles_load_gadget2(this->box().ctx(), filename.c_str(), this->mass(), &h));
        static_assert(sizeof(Header) == sizeof(gev_gadget2_header), "gadget2_header is 256 bytes (metadata.hpp:159-178)");
        std::memcpy(&hdr, &h, sizeof h);
    }

    // express files (Particles_gevolution.hpp:185-186): the reference's rank-file
    // naming and layout, one rank; the file's Real is the caller's Real
    template <class Header> void saveExpress(std::string filename, Header &hdr)
    {
        const gev_gadget2_header h = to_header(hdr);
        gev_b200::check(this->box().ctx(), gev_express_write(this->box().ctx(), filename.c_str(), &h, (int32_t)sizeof(Real)));
    }
    template <class Header> void loadExpress(std::string filename, Header &hdr)
    {
        gev_gadget2_header h;
        gev_b200::check(this->box().ctx(), gev_express_read(this->box().ctx(), filename.c_str(), this->mass(), &h));
        static_assert(sizeof(Header) == sizeof(gev_gadget2_header), "gadget2_header is 256 bytes (metadata.hpp:159-178)");
        std::memcpy(&hdr, &h, sizeof h);
    }

    // snapshot (Particles_gevolution.hpp:180): particles whose ID is a multiple
    // of tracer_factor, positions x BoxSize, velocities q / a^1.5 with a =
    // hdr.time; the redshift interpolation (dtau_pos, dtau_vel) is not applied
    template <class Header>
    void saveGadget2(std::string filename, Header &hdr, const int tracer_factor = 1, double dtau_pos = 0., double dtau_vel = 0.,
                     Field<Real> *phi = nullptr)
    {
        (void)phi;
        if (dtau_pos != 0. || dtau_vel != 0.)
            throw std::runtime_error("gev_latfield: redshift-interpolated snapshots are not supported");
        const gev_gadget2_header h = to_header(hdr);
        gev_b200::check(this->box().ctx(), gev_snapshot_gadget2(this->box().ctx(), filename.c_str(), &h, tracer_factor));
    }

    // lightcone shell (Particles_gevolution.hpp:181): the library finds the
    // vertex images itself (findIntersectingLightcones, up to 64 of them) and
    // keeps the ID logs of each shell on the GPU, one per caller-side backlog
    // object; vertex, vertexcount and IDprelog are not read.  a = hdr.time.
    template <int IDlog_scatter = 0, class Header, class Geometry, class Backlog, class Prelog>
    void saveGadget2(std::string filename, Header &hdr, Geometry &lightcone, double dist, double dtau, double dtau_old,
                     double dadtau, double (*vertex)[3], const int vertexcount, Backlog &IDbacklog, Prelog *IDprelog,
                     Field<Real> *phi, const int tracer_factor = 1)
    {
        (void)vertex; (void)vertexcount; (void)IDprelog; (void)phi;
        gev_b200::Box &b = this->box();
        b.flush();
        gev_lightcone_args lc{};
        for (int i = 0; i < 3; i++) {
            lc.vertex[i] = lightcone.vertex[i];
            lc.direction[i] = lightcone.direction[i];
        }
        lc.opening = lightcone.opening;
        lc.distance[0] = lightcone.distance[0];
        lc.distance[1] = lightcone.distance[1];
        lc.d = dist;   // with tau = 0 below, the crossing distance is dist
        lc.tracer_factor = tracer_factor;
        lc.shell = b.shell_of(&IDbacklog);
        int64_t n = 0, cap = 0;
        gev_b200::check(b.ctx(), gev_particles_count(b.ctx(), &cap));
        gev_b200::check(b.ctx(), gev_lightcone(b.ctx(), &lc, 0., dtau, dtau_old, hdr.time, dadtau, cap, nullptr, nullptr,
                                               nullptr, &n));
        std::vector<float> pos(3 * (size_t)n), vel(3 * (size_t)n);
        std::vector<int64_t> ids((size_t)n);
        gev_b200::check(b.ctx(), gev_lightcone_fetch(b.ctx(), n, pos.data(), vel.data(), ids.data(), &n));
        const gev_gadget2_header h = to_header(hdr);
        gev_b200::check(b.ctx(), gev_gadget2_write(filename.c_str(), &h, pos.data(), vel.data(), ids.data(), n));
    }

private:
    template <class Header> static gev_gadget2_header to_header(const Header &hdr)
    {
        static_assert(sizeof(Header) == sizeof(gev_gadget2_header), "gadget2_header is 256 bytes (metadata.hpp:159-178)");
        gev_gadget2_header h;
        std::memcpy(&h, &hdr, sizeof h);
        return h;
    }
};

// ---- projections (gevolution.hpp) ----
template <class part, class info>
inline void projection_T00_project(perfParticles<part, info> *pcls, Field<Real> *T00, double a = 1., Field<Real> *phi = nullptr,
                                   double coeff = 1.)
{
    gev_b200::Box &b = pcls->box();
    if (T00->id() != GEV_FIELD_SOURCE) throw std::runtime_error("gev_latfield: T00 projects into the source field");
    gev_b200::check(b.ctx(), gev_project(b.ctx(), GEV_PROJ_T00, a, coeff, phi ? 1 : 0, b.accumulate_into(GEV_FIELD_SOURCE)));
}

template <class part, class info>
inline void projection_Tij_project(perfParticles<part, info> *pcls, Field<Real> *Tij, double a = 1., Field<Real> *phi = nullptr,
                                   double coeff = 1., Real *hij_hom = nullptr)
{
    if (hij_hom) throw std::runtime_error("gev_latfield: anisotropic expansion (hij_hom) is not supported");
    gev_b200::Box &b = pcls->box();
    if (Tij->id() != GEV_FIELD_SIJ) throw std::runtime_error("gev_latfield: Tij projects into the Sij field");
    gev_b200::check(b.ctx(), gev_project(b.ctx(), GEV_PROJ_TIJ, a, coeff, phi ? 1 : 0, b.accumulate_into(GEV_FIELD_SIJ)));
}

// fields = {Tij, phi}, params = {a, coeff, hij_hom[0..4]}
template <class part, class info>
inline void projection_Tij_project_Async(perfParticles<part, info> *pcls, Field<Real> **fields, int nfield, double *params)
{
    projection_Tij_project(pcls, fields[0], params[0], nfield > 1 ? fields[1] : nullptr, params[1]);
}

template <class part, class info>
inline void projection_T0i_project(perfParticles<part, info> *pcls, Field<Real> *T0i, Field<Real> *phi = nullptr, double coeff = 1.)
{
    gev_b200::Box &b = pcls->box();
    if (T0i->id() != GEV_FIELD_BI) throw std::runtime_error("gev_latfield: T0i projects into the Bi field");
    gev_b200::check(b.ctx(), gev_project(b.ctx(), GEV_PROJ_T0I, 1., coeff, phi ? 1 : 0, b.accumulate_into(GEV_FIELD_BI)));
}

// fields = {T0i, phi}, params = {coeff}
template <class part, class info>
inline void projection_T0i_project_Async(perfParticles<part, info> *pcls, Field<Real> **fields, int nfield, double *params)
{
    projection_T0i_project(pcls, fields[0], nfield > 1 ? fields[1] : nullptr, params[0]);
}

template <class part, class info>
inline void scalarProjectionCIC_project(perfParticles<part, info> *pcls, Field<Real> *field)
{
    gev_b200::Box &b = pcls->box();
    if (field->id() != GEV_FIELD_SOURCE) throw std::runtime_error("gev_latfield: the CIC density projects into the source field");
    gev_b200::check(b.ctx(), gev_project(b.ctx(), GEV_PROJ_CIC, 1., 1., 0, b.accumulate_into(GEV_FIELD_SOURCE)));
}

// the halo folds of the reference (projection_comm1 etc.): nothing to fold on one GPU
inline void projection_T00_comm(Field<Real> *) {}
inline void projection_T0i_comm(Field<Real> *) {}
inline void projection_Tij_comm(Field<Real> *) {}

// the replacement of main.cu's thrust::fill_n on a projection target: the next projection overwrites
inline void zero(Field<Real> &field) { field.box().consumed(field.id()); }

// ---- source preparation and Fourier-space solvers (gevolution.hpp) ----
inline double prepareFTsource(Field<Real> &phi, Field<Real> &chi, Field<Real> &source, double bgmodel, Field<Real> &result,
                              double coeff, double coeff2, double coeff3)
{
    if (phi.id() != GEV_FIELD_PHI || chi.id() != GEV_FIELD_CHI || source.id() != GEV_FIELD_SOURCE || result.id() != GEV_FIELD_SOURCE)
        throw std::runtime_error("gev_latfield: prepareFTsource(phi, chi, source, bg, source, ...) is the supported T00 form");
    gev_b200::Box &b = source.box();
    b.flush();
    double sum = 0.;
    gev_b200::check(b.ctx(), gev_prepare_T00(b.ctx(), bgmodel, coeff, coeff2, coeff3, &sum));
    b.prepared_source();
    return sum;
}

inline void prepareFTsource(Field<Real> &phi, Field<Real> &Tij, Field<Real> &Sij, double coeff)
{
    if (phi.id() != GEV_FIELD_PHI || Tij.id() != GEV_FIELD_SIJ || Sij.id() != GEV_FIELD_SIJ)
        throw std::runtime_error("gev_latfield: prepareFTsource(phi, Sij, Sij, coeff) is the supported Tij form");
    Sij.box().tij_prepare(coeff);
}

inline void solveModifiedPoissonFT(Field<Imag> &src, Field<Imag> &pot, Real coeff, Real modif = 0)
{
    if (src.role() != FT_SCALAR || pot.role() != FT_SCALAR)
        throw std::runtime_error("gev_latfield: solveModifiedPoissonFT(scalarFT, scalarFT, ...) is the supported form");
    src.box().poisson(coeff, modif);
}

inline void projectFTscalar(Field<Imag> &SijFT, Field<Imag> &chiFT, int add = 0)
{
    if (add || SijFT.role() != FT_SIJ || chiFT.role() != FT_SCALAR)
        throw std::runtime_error("gev_latfield: projectFTscalar(SijFT, scalarFT) without add is the supported form");
    SijFT.box().scalar_projection();
}

inline void projectFTvector(Field<Imag> &SiFT, Field<Imag> &BiFT, Real coeff = 1, Real modif = 0)
{
    if (SiFT.role() != FT_BI || BiFT.role() != FT_BI)
        throw std::runtime_error("gev_latfield: projectFTvector(BiFT, BiFT, ...) is the supported form");
    BiFT.box().vector_projection(coeff, modif);
}

inline void evolveFTvector(Field<Imag> &SijFT, Field<Imag> &BiFT, Real a2dtau)
{
    if (SijFT.role() != FT_SIJ || BiFT.role() != FT_BI) throw std::runtime_error("gev_latfield: evolveFTvector(SijFT, BiFT, ...)");
    BiFT.box().vector_evolution(a2dtau);
}

inline void projectFTtensor(Field<Imag> &SijFT, Field<Imag> &hijFT)
{
    if (SijFT.role() != FT_SIJ || hijFT.role() != FT_HIJ) throw std::runtime_error("gev_latfield: projectFTtensor(SijFT, hijFT)");
    SijFT.box().tensor_step(true, 0., 0., 0.);
}

inline void evolveFTtensor(Field<Imag> &SijFT, Field<Imag> &hijFT, Field<Imag> &hijprimeFT, double hubble, double dtau,
                           double dtau_old)
{
    if (SijFT.role() != FT_SIJ || hijFT.role() != FT_HIJ || hijprimeFT.role() != FT_HIJPRIME)
        throw std::runtime_error("gev_latfield: evolveFTtensor(SijFT, hijFT, hijprimeFT, ...)");
    SijFT.box().tensor_step(false, hubble, dtau, dtau_old);
}

// ---- background (background.hpp), for the reference's cosmology struct ----
template <class Cosmology> inline gev_cosmo gev_background_of(const Cosmology &c)
{
    if (c.num_ncdm > 0 || c.Omega_fld != 0.)
        throw std::runtime_error("gev_latfield: the background supports CDM, baryons, Lambda and radiation only");
    gev_cosmo g{};
    g.Omega_m = c.Omega_cdm + c.Omega_b;
    g.Omega_Lambda = c.Omega_Lambda;
    g.Omega_rad = c.Omega_rad;
    return g;
}

template <class Cosmology> inline double Hconf(const double a, const double fourpiG, const Cosmology &cosmo)
{
    const gev_cosmo g = gev_background_of(cosmo);
    return gev_hconf(a, fourpiG, &g);
}

template <class Cosmology> inline void rungekutta4bg(double &a, const double fourpiG, const Cosmology &cosmo, const double dtau)
{
    const gev_cosmo g = gev_background_of(cosmo);
    gev_rungekutta4bg(&a, fourpiG, &g, dtau);
}

template <class Cosmology> inline double particleHorizon(const double a, const double fourpiG, Cosmology &cosmo)
{
    const gev_cosmo g = gev_background_of(cosmo);
    return gev_particle_horizon(a, fourpiG, &g);
}

#endif
