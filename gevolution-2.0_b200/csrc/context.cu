// context.cu -- the C ABI (include/gev.h): context, device memory, call
// sequencing of the kernels, background integrator and step driver.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gev.h"
#include "kernels.h"

namespace gev {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ArgError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct DeviceError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CapacityError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct NoMemError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

static void ck(cudaError_t e, const char *what)
{
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        throw NoMemError(std::string(what) + ": " + cudaGetErrorString(e));
    }
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T> struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    void alloc(size_t count, const char *what)
    {
        free();
        if (count == 0) return;
        ck(cudaMalloc((void **)&p, count * sizeof(T)), what);
        n = count;
    }
    void free()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DBuf() { free(); }
};

// rows of `width` values between arrays with row pitches sp and dp
template <class A, class B>
__global__ void k_convert_rows(const A *src, int sp, B *dst, int dp, int width, int64_t rows)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= rows * width) return;
    const int64_t r = i / width, c = i - r * width;
    dst[r * dp + c] = (B)src[r * sp + c];
}

template <class A, class B>
__global__ void k_convert(const A *src, B *dst, int64_t n)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (B)src[i];
}

// ---------------------------------------------------------------------------
// findIntersectingLightcones (tools.hpp:637-886), one domain = the whole box.
// Up to 64 periodic images are kept (the reference keeps MAX_INTERSECTS = 12 and
// warns that data is lost beyond that, tools.hpp:877-882).
// ---------------------------------------------------------------------------
static int find_intersecting(const double *lcv, const double *dir, double opening, double outer, double inner,
                             const double *domain, double vtx[64][3])
{
    int range = (int)std::ceil(outer) + 1, n = 0;
    double cen[3], rdom = 0.0;
    for (int i = 0; i < 3; i++) {
        cen[i] = 0.5 * domain[i] + 0.5 * domain[i + 3];
        rdom += (domain[i + 3] - domain[i]) * (domain[i + 3] - domain[i]);
    }
    rdom = 0.5 * std::sqrt(rdom);
    for (int u = -range; u <= range; u++)
        for (int v = -range; v <= range; v++)
            for (int w = -range; w <= range; w++) {
                const double x[3] = {lcv[0] + u, lcv[1] + v, lcv[2] + w};
                double dd = 0.0;   // distance from the image to the domain box
                for (int i = 0; i < 3; i++) {
                    double e = x[i] < domain[i] ? domain[i] - x[i] : (x[i] > domain[i + 3] ? x[i] - domain[i + 3] : 0.0);
                    dd += e * e;
                }
                if (std::sqrt(dd) > outer) continue;
                bool inside = true;   // domain entirely within the inner sphere
                for (int c = 0; c < 8 && inside; c++) {
                    double cc[3] = {domain[(c & 1) ? 3 : 0], domain[(c & 2) ? 4 : 1], domain[(c & 4) ? 5 : 2]};
                    double r = std::sqrt((cc[0] - x[0]) * (cc[0] - x[0]) + (cc[1] - x[1]) * (cc[1] - x[1]) + (cc[2] - x[2]) * (cc[2] - x[2]));
                    if (!(r < inner)) inside = false;
                }
                if (inside) continue;
                double dist = std::sqrt((cen[0] - x[0]) * (cen[0] - x[0]) + (cen[1] - x[1]) * (cen[1] - x[1]) + (cen[2] - x[2]) * (cen[2] - x[2]));
                bool take = dist <= rdom;
                if (!take) {
                    double ca = ((cen[0] - x[0]) * dir[0] + (cen[1] - x[1]) * dir[1] + (cen[2] - x[2]) * dir[2]) / dist;
                    if (ca >= opening) take = true;
                    else if (dist > outer && std::acos(ca) - std::acos(opening) <= std::acos((outer * outer + dist * dist - rdom * rdom) / (2. * outer * dist))) take = true;
                    else if (dist <= outer && std::acos(ca) - std::acos(opening) <= std::asin(rdom / dist)) take = true;
                }
                if (take) {
                    if (n < 64)
                        for (int i = 0; i < 3; i++) vtx[n][i] = x[i];
                    n++;
                }
            }
    return n < 64 ? n : 64;
}

// ---------------------------------------------------------------------------
// background.hpp:200-207, :235-244, :268-291 (CDM + Lambda + radiation)
// ---------------------------------------------------------------------------
static double hconf(double a, double fourpiG, const gev_cosmo &c)
{
    return std::sqrt((2. * fourpiG / 3.) * ((c.Omega_m / a) + (c.Omega_Lambda * a * a) + (c.Omega_rad / a / a)));
}

static void rk4bg(double &a, double fourpiG, const gev_cosmo &c, double dtau)
{
    double k1a = a * hconf(a, fourpiG, c);
    double k2a = (a + k1a * dtau / 2.) * hconf(a + k1a * dtau / 2., fourpiG, c);
    double k3a = (a + k2a * dtau / 2.) * hconf(a + k2a * dtau / 2., fourpiG, c);
    double k4a = (a + k3a * dtau) * hconf(a + k3a * dtau, fourpiG, c);
    a += dtau * (k1a + 2. * k2a + 2. * k3a + k4a) / 6.;
}

static double horizon_integrand(double s, const gev_cosmo &c) { return 2. / (s * hconf(s * s, 1., c)); }

static double simpson(double lo, double hi, double flo, double fmid, double fhi, double whole, double tol, int depth,
                      const gev_cosmo &c)
{
    double mid = 0.5 * (lo + hi), lm = 0.5 * (lo + mid), rm = 0.5 * (mid + hi);
    double flm = horizon_integrand(lm, c), frm = horizon_integrand(rm, c);
    double left = (mid - lo) / 6. * (flo + 4 * flm + fmid), right = (hi - mid) / 6. * (fmid + 4 * frm + fhi);
    if (depth <= 0 || std::fabs(left + right - whole) <= 15 * tol) return left + right + (left + right - whole) / 15.;
    return simpson(lo, mid, flo, flm, fmid, left, tol / 2, depth - 1, c) + simpson(mid, hi, fmid, frm, fhi, right, tol / 2, depth - 1, c);
}

static double particle_horizon(double a, double fourpiG, const gev_cosmo &c)
{
    double lo = std::sqrt(a) * 1.0e-7, hi = std::sqrt(a);
    double flo = horizon_integrand(lo, c), fhi = horizon_integrand(hi, c), fm = horizon_integrand(0.5 * (lo + hi), c);
    double whole = (hi - lo) / 6. * (flo + 4 * fm + fhi);
    return simpson(lo, hi, flo, fm, fhi, whole, 1e-13, 60, c) / std::sqrt(fourpiG);
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct CtxBase {
    gev_config cfg{};
    std::string err;
    virtual ~CtxBase() {}
    virtual void particles_set(const double *pos, const double *q, const int64_t *id, int64_t n, double mass) = 0;
    virtual void particles_get(double *pos, double *q, int64_t *id, int64_t cap, int64_t *n_out) = 0;
    virtual void particles_exchange(double *pos_out, double *q_out, int64_t *id_out, int64_t cap, int64_t *n_out,
                                    const double *pos_in, const double *q_in, const int64_t *id_in, int64_t n_in,
                                    double mass) = 0;
    virtual int64_t particles_count() const = 0;
    virtual double particle_mass() const = 0;
    virtual void field_get(int f, double *host) = 0;
    virtual void field_set(int f, const double *host) = 0;
    virtual void project(uint32_t which, double a, double coeff, int use_phi, int accumulate) = 0;
    virtual void solve_phi(int prepare, double bg, double c, double c2, double c3, double pc, double modif, double *sum, double *phom) = 0;
    virtual double prepare_t00(double bg, double c, double c2, double c3) = 0;
    virtual void prepare_tij(double coeff) = 0;
    virtual void solve_chi(double coeff, int cycle0, double hubble, double dtau, double dtau_old, double a2dtau) = 0;
    virtual void solve_B(double coeff, double modif) = 0;
    virtual double kick_drift(const KickDriftParams &kp) = 0;
    virtual void power_spectrum(int nb, double kmax, double *kb, double *pw, double *ks, double *ps, int32_t *occ) = 0;
    virtual void lightcone(const gev_lightcone_args &lc, double tau, double dtau, double dtau_old, double a, double dadtau,
                           int64_t cap, float *pos, float *vel, int64_t *ids, int64_t *n_out) = 0;
    virtual void fetch_lightcone(int64_t cap, float *pos, float *vel, int64_t *ids, int64_t *n_out) = 0;
    virtual void ics_zeldovich(const gev_ics_params &ip) = 0;
    virtual void ics_basic(const gev_ics_basic_params &ip) = 0;
    virtual void sync() = 0;
    virtual cudaStream_t stream() = 0;
    virtual int64_t kernel_launches() const = 0;
};

template <class R> struct Ctx final : CtxBase {
    using C = typename CT<R>::C;
    Geom g{};
    cudaStream_t st = nullptr;
    DBuf<R> phi, chi, source, Sij, Bi;
    DBuf<C> W, hij, hijp, bstate;
    DBuf<C> tw_full, tw_half;
    DBuf<double> k2;
    DBuf<double2> ks;
    DBuf<uint32_t> cellA, cellB, bucket, rank, inv, counts, bstart, bsums, depwork;
    DBuf<double> offA, offB;
    DBuf<R> qA, qB;
    DBuf<int64_t> idA, idB;
    DBuf<double> partial, scal;          // scal: [0] sum, [1] phi_hom
    DBuf<unsigned long long> u64;        // [0] vmax bits, [1] lc count, [2] prelog count
    DBuf<int> derr;
    DBuf<double> bins;
    DBuf<unsigned long long> occ;
    DBuf<double> rho64;                  // mixed precision: FP64 density of the spectrum measurement
    DBuf<double2> tw64_full, tw64_half;  // mixed precision: FP64 twiddles of that measurement
    DBuf<double> stage;                  // particle / field transfer staging
    DBuf<int64_t> stage_id;
    // particles_exchange: download and upload streams, four staging slots
    // (two per direction), and the events that order them
    cudaStream_t sdn = nullptr, sup = nullptr;
    cudaEvent_t ev_start = nullptr, ev_dn[2] = {nullptr, nullptr}, ev_dn_end = nullptr, ev_up_end = nullptr;
    DBuf<double> xstage;
    DBuf<int64_t> xstage_id;
    static constexpr int64_t XCHUNK = 1 << 21;
    DBuf<float> lc_pos, lc_vel;
    DBuf<int64_t> lc_id;
    DBuf<unsigned long long> idset[8][2];   // per shell: ID logs of the previous and current cycle
    int idset_cur[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool backlog_valid[8] = {false, false, false, false, false, false, false, false};
    int64_t idset_cap = 0;
    int64_t lc_last = 0;
    bool cur_is_A = true;
    bool bi_sums = false;       // Bi holds the potential-free T0i sums of project_step
    bool t0i_pending = false;   // FP64 T0I_SUMS: solve_B deposits T0i first (with t0i_coeff)
    double t0i_coeff = 1.0;
    int64_t launch_count = 0;
    int64_t np = 0;
    double mass = 0.0;
    bool have_particles = false;
    static constexpr int64_t CHUNK = 1 << 22;

    explicit Ctx(const gev_config &c)
    {
        cfg = c;
        const int N = c.N;
        g.N = N;
        g.P = N / 2 + 1;
        g.nt = N / 8;
        g.n3 = (int64_t)N * N * N;
        g.PP = N / 2 + 2;
        g.nk = (int64_t)g.PP * N * N;
        g.ntiles = (int64_t)g.nt * g.nt * g.nt;
        ck(cudaSetDevice(c.device), "cudaSetDevice");
        ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        phi.alloc(g.n3, "phi");
        chi.alloc(g.n3, "chi");
        source.alloc(g.n3, "source");
        Sij.alloc(6 * g.n3, "Sij");
        Bi.alloc(3 * g.n3, "Bi");
        W.alloc(6 * g.nk, "Fourier workspace");
        if (c.tensor) { hij.alloc(6 * g.nk, "hij"); hijp.alloc(6 * g.nk, "hij'"); }
        if (c.vector_method == GEV_VECTOR_PARABOLIC) bstate.alloc(3 * g.nk, "B state");
        for (auto *b : {&phi, &chi, &source}) ck(cudaMemsetAsync(b->p, 0, b->n * sizeof(R), st), "memset");
        ck(cudaMemsetAsync(Sij.p, 0, Sij.n * sizeof(R), st), "memset");
        ck(cudaMemsetAsync(Bi.p, 0, Bi.n * sizeof(R), st), "memset");
        if (hij.p) { ck(cudaMemsetAsync(hij.p, 0, hij.n * sizeof(C), st), "memset"); ck(cudaMemsetAsync(hijp.p, 0, hijp.n * sizeof(C), st), "memset"); }
        if (bstate.p) ck(cudaMemsetAsync(bstate.p, 0, bstate.n * sizeof(C), st), "memset");
        make_tables();
        const int64_t cap = c.capacity;
        cellA.alloc(cap, "particles"); cellB.alloc(cap, "particles");
        offA.alloc(3 * cap, "particles"); offB.alloc(3 * cap, "particles");
        qA.alloc(3 * cap, "particles"); qB.alloc(3 * cap, "particles");
        idA.alloc(cap, "particles"); idB.alloc(cap, "particles");
        bucket.alloc(cap, "buckets"); rank.alloc(cap, "buckets"); inv.alloc(cap, "buckets");
        const int64_t nb = g.ntiles * 8;
        counts.alloc(nb, "bucket counts");
        bstart.alloc(nb + 1, "bucket starts");
        bsums.alloc((nb + 1023) / 1024 + 1, "scan");
        depwork.alloc(g.ntiles + 2, "deposit work list");
        ck(cudaMemsetAsync(bstart.p, 0, (nb + 1) * sizeof(uint32_t), st), "memset");
        partial.alloc((int64_t)N * N, "partials");
        scal.alloc(4, "scalars");
        u64.alloc(4, "scalars");
        derr.alloc(1, "error word");
        ck(cudaMemsetAsync(derr.p, 0, sizeof(int), st), "memset");
        ck(cudaStreamSynchronize(st), "init");
    }

    ~Ctx() override
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        for (cudaStream_t s : {sdn, sup})
            if (s) {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
        for (cudaEvent_t e : {ev_start, ev_dn[0], ev_dn[1], ev_dn_end, ev_up_end})
            if (e) cudaEventDestroy(e);
    }

    cudaStream_t stream() override { return st; }

    void make_tables()
    {
        const int N = g.N;
        std::vector<C> tf(N), th(N / 2);
        for (int k = 0; k < N; k++) {
            double ang = -2.0 * M_PI * (double)k / N;
            tf[k].x = (R)std::cos(ang);
            tf[k].y = (R)std::sin(ang);
        }
        for (int k = 0; k < N / 2; k++) {
            double ang = -2.0 * M_PI * (double)k / (N / 2);
            th[k].x = (R)std::cos(ang);
            th[k].y = (R)std::sin(ang);
        }
        // gevolution.hpp:269-275
        std::vector<double> hk2(N);
        std::vector<double2> hks(N);
        for (int i = 0; i < N; i++) {
            double gk = 2.0 * (double)N * std::sin(M_PI * (double)i / (double)N);
            hks[i] = make_double2(gk * std::cos(M_PI * (double)i / (double)N), -gk * std::sin(M_PI * (double)i / (double)N));
            hk2[i] = gk * gk;
        }
        tw_full.alloc(N, "twiddles"); tw_half.alloc(N / 2, "twiddles");
        k2.alloc(N, "k tables"); ks.alloc(N, "k tables");
        ck(cudaMemcpy(tw_full.p, tf.data(), N * sizeof(C), cudaMemcpyHostToDevice), "tables");
        ck(cudaMemcpy(tw_half.p, th.data(), (N / 2) * sizeof(C), cudaMemcpyHostToDevice), "tables");
        ck(cudaMemcpy(k2.p, hk2.data(), N * sizeof(double), cudaMemcpyHostToDevice), "tables");
        ck(cudaMemcpy(ks.p, hks.data(), N * sizeof(double2), cudaMemcpyHostToDevice), "tables");
    }

    FftTables<R> tables() const { return FftTables<R>{tw_full.p, tw_half.p, k2.p, ks.p}; }

    void make_tables64()
    {
        const int N = g.N;
        std::vector<double2> tf(N), th(N / 2);
        for (int k = 0; k < N; k++) tf[k] = make_double2(std::cos(-2.0 * M_PI * (double)k / N), std::sin(-2.0 * M_PI * (double)k / N));
        for (int k = 0; k < N / 2; k++)
            th[k] = make_double2(std::cos(-2.0 * M_PI * (double)k / (N / 2)), std::sin(-2.0 * M_PI * (double)k / (N / 2)));
        tw64_full.alloc(N, "twiddles");
        tw64_half.alloc(N / 2, "twiddles");
        ck(cudaMemcpy(tw64_full.p, tf.data(), N * sizeof(double2), cudaMemcpyHostToDevice), "tables");
        ck(cudaMemcpy(tw64_half.p, th.data(), (N / 2) * sizeof(double2), cudaMemcpyHostToDevice), "tables");
    }

    PView<R> view(bool A) const
    {
        PView<R> v;
        v.cell = A ? cellA.p : cellB.p;
        v.off = A ? offA.p : offB.p;
        v.q = A ? qA.p : qB.p;
        v.id = A ? idA.p : idB.p;
        v.cap = cfg.capacity;
        v.n = np;
        return v;
    }
    PView<R> cur() const { return view(cur_is_A); }

    // every kernel launch of the library goes through here (count = kernels launched)
    void launched(const char *what, int kernels = 1)
    {
        ck(cudaGetLastError(), what);
        launch_count += kernels;
    }

    // a tile deposit: the tile launch and the dense-tile launch
    void deposit(int kind, bool use_phi, const DepOut<R> &o, double a, double m00, double mij, double m0i, int accumulate,
                 const char *what)
    {
        ck(cudaMemsetAsync(depwork.p, 0, 2 * sizeof(uint32_t), st), "memset");
        launch_deposit<R>(kind, use_phi, cur(), bstart.p, g.N, phi.p, o, a, m00, mij, m0i, accumulate, depwork.p, derr.p,
                          st);
        launched(what, 2);
    }
    int64_t kernel_launches() const override { return launch_count; }

    void check_device_error()
    {
        int e = 0;
        ck(cudaMemcpyAsync(&e, derr.p, sizeof(int), cudaMemcpyDeviceToHost, st), "error word");
        ck(cudaStreamSynchronize(st), "synchronize");
        if (e) {
            ck(cudaMemsetAsync(derr.p, 0, sizeof(int), st), "memset");
            char buf[224];
            snprintf(buf, sizeof buf, "device error word 0x%x (%s%s%s%s%s)", e, (e & ERR_NONFINITE) ? "non-finite particle coordinate " : "",
                     (e & ERR_LC_OVERFLOW) ? "lightcone buffer overflow " : "", (e & ERR_BAD_CELL) ? "cell index out of range " : "",
                     (e & ERR_TMA_TIMEOUT) ? "bulk tensor copy timed out " : "", (e & ERR_BAD_ORDER) ? "bucket order not sorted by cell" : "");
            throw DeviceError(buf);
        }
    }

    void sync() override
    {
        ck(cudaStreamSynchronize(st), "synchronize");
        check_device_error();
    }

    void ensure_stage(int64_t doubles, int64_t ids)
    {
        if ((int64_t)stage.n < doubles) stage.alloc(doubles, "staging");
        if ((int64_t)stage_id.n < ids) stage_id.alloc(ids, "staging");
    }

    // bucket order from the current cell indices
    void rebin_from_cells()
    {
        const int64_t nb = g.ntiles * 8;
        ck(cudaMemsetAsync(counts.p, 0, nb * sizeof(uint32_t), st), "memset");
        launch_bin_count<R>(cur(), g.N, counts.p, bucket.p, rank.p, st);
        launched("bin_count");
        finish_rebin();
    }

    void finish_rebin()
    {
        const int64_t nb = g.ntiles * 8;
        launch_scan(counts.p, bstart.p, nb, bsums.p, st);
        launched("scan", 3);
        launch_rebin<R>(cur(), view(!cur_is_A), bstart.p, bucket.p, rank.p, inv.p, g.N, derr.p, st);
        launched("rebin", 2);
        cur_is_A = !cur_is_A;
    }

    void particles_set(const double *pos, const double *q, const int64_t *id, int64_t n, double m) override
    {
        if (n < 0 || n > cfg.capacity) throw ArgError("particle count exceeds the context capacity");
        if (n > 0 && (!pos || !q)) throw ArgError("null particle array");
        if (n >= (int64_t)UINT32_MAX) throw ArgError("particle count exceeds 2^32 - 1");
        np = n;
        mass = m;
        const int64_t ch = std::min<int64_t>(std::max<int64_t>(n, 1), CHUNK);
        ensure_stage(6 * ch, ch);
        PView<R> v = view(true);
        for (int64_t o = 0; o < n; o += ch) {
            int64_t c = std::min(ch, n - o);
            ck(cudaMemcpyAsync(stage.p, pos + 3 * o, 3 * c * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
            ck(cudaMemcpyAsync(stage.p + 3 * ch, q + 3 * o, 3 * c * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
            if (id) ck(cudaMemcpyAsync(stage_id.p, id + o, c * sizeof(int64_t), cudaMemcpyHostToDevice, st), "H2D");
            PView<R> vo = v;
            vo.cell += o; vo.off += o; vo.q += o; vo.id += o;
            launch_load_particles<R>(vo, stage.p, stage.p + 3 * ch, id ? stage_id.p : nullptr, c, g.N, derr.p, st);
            launched("load_particles");
            if (!id) {
                // default IDs: the particle's index in the caller's array
                std::vector<int64_t> ids(c);
                for (int64_t k = 0; k < c; k++) ids[k] = o + k;
                ck(cudaMemcpyAsync(vo.id, ids.data(), c * sizeof(int64_t), cudaMemcpyHostToDevice, st), "H2D");
                ck(cudaStreamSynchronize(st), "synchronize");
            }
            ck(cudaStreamSynchronize(st), "synchronize");
        }
        cur_is_A = true;
        rebin_from_cells();
        have_particles = true;
        sync();
    }

    void ics_zeldovich(const gev_ics_params &ip) override
    {
        const int N = g.N;
        if (cfg.capacity < g.n3) throw ArgError("the context capacity is below N^3 particles");
        if (ip.boxsize <= 0.0 || ip.a <= 0.0 || ip.fourpiG <= 0.0) throw ArgError("boxsize, a and fourpiG must be positive");
        if (ip.n_pk < 2 || !ip.pk_k || !ip.pk_p) throw ArgError("the power spectrum table needs at least two points");
        std::vector<double> tab(2 * (size_t)ip.n_pk);
        for (int i = 0; i < ip.n_pk; i++) {
            if (!(ip.pk_k[i] > 0.0) || !(ip.pk_p[i] > 0.0) || (i > 0 && !(ip.pk_k[i] > ip.pk_k[i - 1])))
                throw ArgError("power spectrum table: k must increase and k, P must be positive");
            tab[i] = std::log(ip.pk_k[i]);
            tab[ip.n_pk + i] = std::log(ip.pk_p[i]);
        }
        DBuf<double> dtab;
        dtab.alloc(tab.size(), "P(k) table");
        ck(cudaMemcpyAsync(dtab.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
        // 1. white noise
        if (ip.noise) field_set(GEV_FIELD_SOURCE, ip.noise);
        else {
            launch_ics_noise<R>(source.p, g.n3, ip.seed, st);
            launched("ics noise");
        }
        if (ip.noise_out) field_get(GEV_FIELD_SOURCE, ip.noise_out);
        // 2. displacement field into the B_i planes
        const FftTables<R> tb = tables();
        fx_forward<R>(N, FX_COPY, source.p, g.n3, 1, 0, nullptr, nullptr, 0, 0, 0, 0, W.p, g.nk, nullptr, tb, st);
        fy_pass<R>(N, -1, W.p, g.nk, 1, derr.p, tb, st);
        FzParams fz{};
        fz.op = OP_ZELD;
        fz.p0 = ip.boxsize;
        fz.p1 = ip.ksphere ? 1.0 : 0.0;
        fz.tab = dtab.p;
        fz.ntab = ip.n_pk;
        fz.err = derr.p;
        fz_pass<R>(N, fz, W.p, g.nk, nullptr, nullptr, nullptr, tb, st);
        fy_pass<R>(N, 1, W.p, g.nk, 3, derr.p, tb, st);
        fx_inverse<R>(N, W.p, g.nk, Bi.p, g.n3, 3, tb, st);
        launched("ics displacement", 5);
        // 3. the displaced lattice (part_simple_info.mass = Omega_m / Np, ic_basic.hpp:2198-2201)
        np = g.n3;
        mass = ip.Omega_m / (double)g.n3;
        cur_is_A = true;
        launch_ics_lattice<R>(view(true), Bi.p, N, st);
        bi_sums = false;
        launched("ics lattice");
        rebin_from_cells();
        have_particles = true;
        // 4-5. phi and the momenta
        ics_phi_and_momenta(ip.a, ip.fourpiG, ip.Omega_m, ip.Omega_Lambda, ip.Omega_rad, ip.boxsize, ip.gr);
        sync();
    }

    // phi from the CIC density of the particles (ic_basic.hpp:2404-2427) and
    // the momenta from phi (:2431-2437; Omega_m(a), Omega_rad(a):
    // background.hpp:211-213)
    void ics_phi_and_momenta(double a, double fourpiG, double Om, double OL, double Orad, double boxsize, int gr)
    {
        const int N = g.N;
        const FftTables<R> tb = tables();
        project(GEV_PROJ_CIC, 1.0, 1.0, 0, 0);
        gev_cosmo cm{Om, OL, Orad, fourpiG, 0.0, 0.0, 0.0, boxsize};
        const double H = hconf(a, fourpiG, cm);
        fx_forward<R>(N, FX_COPY, source.p, g.n3, 1, 0, nullptr, nullptr, 0, 0, 0, 0, W.p, g.nk, nullptr, tb, st);
        fy_pass<R>(N, -1, W.p, g.nk, 1, derr.p, tb, st);
        FzParams fp{};
        fp.op = OP_POISSON;
        fp.p0 = (fourpiG / a) / -((double)N * (double)N * (double)N);
        fp.p1 = gr ? 3.0 * (H * H + fourpiG * Om / a) : 0.0;
        fp.p2 = 1.0;   // remove the k = 0 mode
        fp.err = derr.p;
        fz_pass<R>(N, fp, W.p, g.nk, nullptr, nullptr, nullptr, tb, st);
        fy_pass<R>(N, 1, W.p, g.nk, 1, derr.p, tb, st);
        fx_inverse<R>(N, W.p, g.nk, phi.p, g.n3, 1, tb, st);
        launched("ics phi", 5);
        const double den = Om + OL * a * a * a + Orad / a;
        const double om_a = Om / den;
        const double orad_a = Orad / (Om * a + OL * a * a * a * a + Orad);
        launch_ics_velocity<R>(cur(), phi.p, N, a / H / (1.5 * om_a + 2.0 * orad_a), st);
        launched("ics velocity");
    }

    void ics_basic(const gev_ics_basic_params &ip) override
    {
        const int N = g.N;
        const double L = ip.boxsize;
        if (!(L > 0.0) || !(ip.a > 0.0) || !(ip.fourpiG > 0.0)) throw ArgError("boxsize, a and fourpiG must be positive");
        if (ip.numtile < 1 || ip.template_n < 1 || !ip.template_pos) throw ArgError("the particle template is empty");
        for (int64_t i = 0; i < 3 * ip.template_n; i++)   // ic_basic.hpp:325-333
            if (!(ip.template_pos[i] >= 0.0f && ip.template_pos[i] <= 1.0f))
                throw ArgError("template positions must lie in [0, 1]");
        const int64_t T = ip.numtile;
        if (ip.template_n > (int64_t)1 << 40 || T > 4096) throw ArgError("template or tiling factor too large");
        const int64_t npart = ip.template_n * T * T * T;
        if (npart > cfg.capacity) throw ArgError("the particle count n numtile^3 exceeds the context capacity");
        if (npart > (int64_t)UINT32_MAX) throw ArgError("too many particles");
        if (ip.n_pk < 3 || !ip.pk_k || !ip.pk_p) throw ArgError("the power spectrum table needs at least three points");
        // loadPowerSpectrum's table (k L, sqrt(P L / 2)), ic_basic.hpp:431-432, and the
        // 1 / L^2 of :1905-1913, as a natural cubic spline
        std::vector<double> x(ip.n_pk), y(ip.n_pk), sb, sc, sd;
        for (int i = 0; i < ip.n_pk; i++) {
            if (!(ip.pk_k[i] >= 0.0) || !(ip.pk_p[i] >= 0.0)) throw ArgError("negative k or P(k) in the power spectrum table");
            x[i] = ip.pk_k[i] * L;
            if (i > 0 && !(x[i - 1] < x[i])) throw ArgError("power spectrum table: k must increase");
            y[i] = std::sqrt(0.5 * ip.pk_p[i] * L) / L / L;
        }
        ics_natural_spline(x, y, sb, sc, sd);
        // the table must cover every |2 pi n| a non-zero mode evaluates (GSL's
        // spline fails outside it): |n|^2 from 1 to 3 (N/2 - 2)^2, below (N/2 - 1)^2 with ksphere
        {
            const int kmax = N / 2 - 1;
            const double fp2 = (4.0 * 3.14159265358979323846) * 3.14159265358979323846;
            auto xk = [&](long m) { return (double)std::sqrt((float)((double)(float)m * fp2)); };
            const long mhi = ip.ksphere ? (long)kmax * kmax - 1 : 3L * (kmax - 1) * (kmax - 1);
            if (kmax >= 2 && (x.front() > xk(1) || x.back() < xk(mhi)))
                throw ArgError("the power spectrum table does not cover 2 pi / L <= k <= 2 pi sqrt(3) (N/2 - 2) / L");
        }
        gev_cosmo cm{ip.Omega_m, ip.Omega_Lambda, ip.Omega_rad, ip.fourpiG, 0.0, 0.0, 0.0, L};
        const double H = hconf(ip.a, ip.fourpiG, cm);
        const FftTables<R> tb = tables();
        // 1. the convolution kernel in the source field
        std::vector<std::pair<int64_t, R>> ker;
        ics_cic_kernel<R>(N, ip.correct_displacement ? ip.template_n : 0, ip.correct_displacement ? ip.template_pos : nullptr,
                          ip.numtile, ker);
        ck(cudaMemsetAsync(source.p, 0, g.n3 * sizeof(R), st), "memset");
        for (const auto &e : ker) ck(cudaMemcpyAsync(source.p + e.first, &e.second, sizeof(R), cudaMemcpyHostToDevice, st), "H2D");
        ck(cudaStreamSynchronize(st), "synchronize");
        // 2. the modes' numerators, line by line from the reference's stream
        const int nspl = ip.n_pk;
        DBuf<double> spl;
        spl.alloc(5 * (int64_t)nspl, "P(k) spline");
        std::vector<double> packed;
        for (const auto *v : {&x, &y, &sb, &sc, &sd}) packed.insert(packed.end(), v->begin(), v->end());
        ck(cudaMemcpyAsync(spl.p, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
        DBuf<double2> modes;
        modes.alloc((int64_t)(N / 2 + 1) * N * N, "IC modes");
        const IcsSpline sp{spl.p, spl.p + nspl, spl.p + 2 * nspl, spl.p + 3 * nspl, spl.p + 4 * nspl, nspl};
        launch_ics_modes(modes.p, N, ip.seed, ip.ksphere, (float)(ip.gr ? H * H : 0.0), sp, derr.p, st);
        launched("ics modes");
        // 3. kernel transform, numerator / kernel, backward transform: the displacement potential in chi
        fx_forward<R>(N, FX_COPY, source.p, g.n3, 1, 0, nullptr, nullptr, 0, 0, 0, 0, W.p, g.nk, nullptr, tb, st);
        fy_pass<R>(N, -1, W.p, g.nk, 1, derr.p, tb, st);
        FzParams fz{};
        fz.op = OP_ICS;
        fz.modes = modes.p;
        fz.err = derr.p;
        fz_pass<R>(N, fz, W.p, g.nk, nullptr, nullptr, nullptr, tb, st);
        fy_pass<R>(N, 1, W.p, g.nk, 1, derr.p, tb, st);
        fx_inverse<R>(N, W.p, g.nk, chi.p, g.n3, 1, tb, st);
        launched("ics displacement potential", 5);
        // 4. the tiled, displaced template
        DBuf<float> tmpl;
        tmpl.alloc(3 * ip.template_n, "particle template");
        ck(cudaMemcpyAsync(tmpl.p, ip.template_pos, 3 * ip.template_n * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
        np = npart;
        mass = ip.Omega_m / (double)npart;
        cur_is_A = true;
        launch_ics_template<R>(view(true), chi.p, tmpl.p, ip.template_n, ip.numtile, N, npart, st);
        launched("ics template");
        bi_sums = false;
        t0i_pending = false;
        rebin_from_cells();
        have_particles = true;
        // 5. phi and the momenta
        ics_phi_and_momenta(ip.a, ip.fourpiG, ip.Omega_m, ip.Omega_Lambda, ip.Omega_rad, L, ip.gr);
        // 6. B_i: T0i with phi, projectFTvector(fourpiG / N^2) (ic_basic.hpp:2468-2477)
        project(GEV_PROJ_T0I, 1.0, 1.0, 1, 0);
        solve_B(ip.fourpiG / (double)N / (double)N, 0.0);
        // 7. chi: Tij with phi, prepareFTsource(2 fourpiG / a / N^2), projectFTscalar (:2479-2489)
        project(GEV_PROJ_TIJ, ip.a, 1.0, 1, 0);
        chi_pass(2.0 * ip.fourpiG / ip.a / (double)N / (double)N, 0, 0.0, 0.0, 0.0, 0.0);
        sync();
    }

    void particles_get(double *pos, double *q, int64_t *id, int64_t cap, int64_t *n_out) override
    {
        if (n_out) *n_out = np;
        if (cap < np) throw CapacityError("host arrays smaller than the particle count");
        const int64_t ch = std::min<int64_t>(std::max<int64_t>(np, 1), CHUNK);
        ensure_stage(6 * ch, ch);
        PView<R> v = cur();
        for (int64_t o = 0; o < np; o += ch) {
            int64_t c = std::min(ch, np - o);
            PView<R> vo = v;
            vo.cell += o; vo.off += o; vo.q += o; vo.id += o;
            launch_store_particles<R>(vo, pos ? stage.p : nullptr, q ? stage.p + 3 * ch : nullptr, id ? stage_id.p : nullptr, c, g.N, st);
            launched("store_particles");
            if (pos) ck(cudaMemcpyAsync(pos + 3 * o, stage.p, 3 * c * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
            if (q) ck(cudaMemcpyAsync(q + 3 * o, stage.p + 3 * ch, 3 * c * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
            if (id) ck(cudaMemcpyAsync(id + o, stage_id.p, c * sizeof(int64_t), cudaMemcpyDeviceToHost, st), "D2H");
            ck(cudaStreamSynchronize(st), "synchronize");
        }
    }

    // particles_get followed by particles_set, with the downloads on one copy
    // stream and the uploads on another so that the two directions of the host
    // link run at once, chunk by chunk.  The uploads fill the other particle
    // buffer, so the device sides never conflict; on the host, an input array
    // that is the matching output array waits chunk by chunk for its download,
    // any other overlap of an input with an output waits for all downloads.
    void particles_exchange(double *pos_out, double *q_out, int64_t *id_out, int64_t cap, int64_t *n_out,
                            const double *pos_in, const double *q_in, const int64_t *id_in, int64_t n_in,
                            double m) override
    {
        if (n_out) *n_out = np;
        if (cap < np) throw CapacityError("host arrays smaller than the particle count");
        if (np > 0 && (!pos_out || !q_out || !id_out)) throw ArgError("null particle array");
        if (n_in < 0 || n_in > cfg.capacity) throw ArgError("particle count exceeds the context capacity");
        if (n_in > 0 && (!pos_in || !q_in || !id_in)) throw ArgError("null particle array");
        if (n_in >= (int64_t)UINT32_MAX) throw ArgError("particle count exceeds 2^32 - 1");
        const int64_t nout = np;
        struct Span { uintptr_t lo, hi; };
        auto span = [](const void *p, int64_t bytes) { return Span{(uintptr_t)p, (uintptr_t)p + (uintptr_t)bytes}; };
        const Span outs[3] = {span(pos_out, 24 * nout), span(q_out, 24 * nout), span(id_out, 8 * nout)};
        const Span ins[3] = {span(pos_in, 24 * n_in), span(q_in, 24 * n_in), span(id_in, 8 * n_in)};
        bool overlap = false;
        for (const Span &i : ins)
            for (const Span &o : outs) overlap |= i.lo < i.hi && o.lo < o.hi && i.lo < o.hi && o.lo < i.hi;
        const bool same = pos_in == pos_out && q_in == q_out && id_in == id_out;
        const bool chunkwise = !overlap || same;

        if (!sdn) {
            ck(cudaStreamCreateWithFlags(&sdn, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaStreamCreateWithFlags(&sup, cudaStreamNonBlocking), "cudaStreamCreate");
            for (cudaEvent_t *e : {&ev_start, &ev_dn[0], &ev_dn[1], &ev_dn_end, &ev_up_end})
                ck(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
        }
        if ((int64_t)xstage.n < 4 * 6 * XCHUNK) xstage.alloc(4 * 6 * XCHUNK, "exchange staging");
        if ((int64_t)xstage_id.n < 4 * XCHUNK) xstage_id.alloc(4 * XCHUNK, "exchange staging");
        ck(cudaEventRecord(ev_start, st), "cudaEventRecord");
        ck(cudaStreamWaitEvent(sdn, ev_start, 0), "cudaStreamWaitEvent");
        ck(cudaStreamWaitEvent(sup, ev_start, 0), "cudaStreamWaitEvent");
        const PView<R> src = cur(), dst = view(!cur_is_A);
        const int64_t ndn = (nout + XCHUNK - 1) / XCHUNK, nup = (n_in + XCHUNK - 1) / XCHUNK;
        auto down = [&](int64_t i) {
            const int64_t o = i * XCHUNK, c = std::min(XCHUNK, nout - o);
            double *sp = xstage.p + (i & 1) * 6 * XCHUNK;
            int64_t *si = xstage_id.p + (i & 1) * XCHUNK;
            PView<R> vo = src;
            vo.cell += o; vo.off += o; vo.q += o; vo.id += o;
            launch_store_particles<R>(vo, sp, sp + 3 * XCHUNK, si, c, g.N, sdn);
            launched("store_particles");
            ck(cudaMemcpyAsync(pos_out + 3 * o, sp, 3 * c * sizeof(double), cudaMemcpyDeviceToHost, sdn), "D2H");
            ck(cudaMemcpyAsync(q_out + 3 * o, sp + 3 * XCHUNK, 3 * c * sizeof(double), cudaMemcpyDeviceToHost, sdn), "D2H");
            ck(cudaMemcpyAsync(id_out + o, si, c * sizeof(int64_t), cudaMemcpyDeviceToHost, sdn), "D2H");
            ck(cudaEventRecord(ev_dn[i & 1], sdn), "cudaEventRecord");
        };
        auto up = [&](int64_t i) {
            const int64_t o = i * XCHUNK, c = std::min(XCHUNK, n_in - o);
            double *sp = xstage.p + (2 + (i & 1)) * 6 * XCHUNK;
            int64_t *si = xstage_id.p + (2 + (i & 1)) * XCHUNK;
            if (chunkwise && same && i < ndn) ck(cudaStreamWaitEvent(sup, ev_dn[i & 1], 0), "cudaStreamWaitEvent");
            ck(cudaMemcpyAsync(sp, pos_in + 3 * o, 3 * c * sizeof(double), cudaMemcpyHostToDevice, sup), "H2D");
            ck(cudaMemcpyAsync(sp + 3 * XCHUNK, q_in + 3 * o, 3 * c * sizeof(double), cudaMemcpyHostToDevice, sup), "H2D");
            ck(cudaMemcpyAsync(si, id_in + o, c * sizeof(int64_t), cudaMemcpyHostToDevice, sup), "H2D");
            PView<R> vo = dst;
            vo.cell += o; vo.off += o; vo.q += o; vo.id += o;
            launch_load_particles<R>(vo, sp, sp + 3 * XCHUNK, si, c, g.N, derr.p, sup);
            launched("load_particles");
        };
        for (int64_t i = 0; i < std::max(ndn, nup); i++) {
            if (i < ndn) down(i);
            if (chunkwise && i < nup) up(i);
        }
        ck(cudaEventRecord(ev_dn_end, sdn), "cudaEventRecord");
        if (!chunkwise) {
            ck(cudaStreamWaitEvent(sup, ev_dn_end, 0), "cudaStreamWaitEvent");
            for (int64_t i = 0; i < nup; i++) up(i);
        }
        ck(cudaEventRecord(ev_up_end, sup), "cudaEventRecord");
        ck(cudaStreamWaitEvent(st, ev_dn_end, 0), "cudaStreamWaitEvent");
        ck(cudaStreamWaitEvent(st, ev_up_end, 0), "cudaStreamWaitEvent");
        np = n_in;
        mass = m;
        cur_is_A = !cur_is_A;
        rebin_from_cells();
        have_particles = true;
        sync();
    }

    int64_t particles_count() const override { return np; }
    double particle_mass() const override { return mass; }

    // (device pointer, number of planes, complex?) of a field
    void field_ref(int f, void **p, int *planes, bool *cplx)
    {
        *cplx = false;
        switch (f) {
        case GEV_FIELD_PHI: *p = phi.p; *planes = 1; break;
        case GEV_FIELD_CHI: *p = chi.p; *planes = 1; break;
        case GEV_FIELD_SOURCE: *p = source.p; *planes = 1; break;
        case GEV_FIELD_SIJ: *p = Sij.p; *planes = 6; break;
        case GEV_FIELD_BI: *p = Bi.p; *planes = 3; break;
        case GEV_FIELD_HIJ_FT: *p = hij.p; *planes = 6; *cplx = true; break;
        case GEV_FIELD_HIJP_FT: *p = hijp.p; *planes = 6; *cplx = true; break;
        case GEV_FIELD_BI_FT: *p = bstate.p; *planes = 3; *cplx = true; break;
        default: throw ArgError("unknown field id");
        }
        if (!*p) throw StateError("field not allocated in this configuration");
    }

    void field_get(int f, double *host) override
    {
        void *p; int planes; bool cplx;
        field_ref(f, &p, &planes, &cplx);
        if (!host) throw ArgError("null host pointer");
        // host planes are dense (Fourier rows of P complex values); device
        // Fourier rows have the pitch PP
        const int64_t n = cplx ? 2 * (int64_t)g.P * g.N * g.N : g.n3;
        const int64_t dn = cplx ? 2 * g.nk : g.n3;
        const int w = cplx ? 2 * g.P : (int)g.n3, dw = cplx ? 2 * g.PP : (int)g.n3;
        const int64_t rows = cplx ? (int64_t)g.N * g.N : 1;
        ensure_stage(n, 0);
        for (int c = 0; c < planes; c++) {
            const R *src = (const R *)p + (int64_t)c * dn;
            k_convert_rows<R, double><<<cdiv(n, 256), 256, 0, st>>>(src, dw, stage.p, w, w, rows);
            launched("convert");
            ck(cudaMemcpyAsync(host + (int64_t)c * n, stage.p, n * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
            ck(cudaStreamSynchronize(st), "synchronize");
        }
    }

    void field_set(int f, const double *host) override
    {
        void *p; int planes; bool cplx;
        field_ref(f, &p, &planes, &cplx);
        if (!host) throw ArgError("null host pointer");
        const int64_t n = cplx ? 2 * (int64_t)g.P * g.N * g.N : g.n3;
        const int64_t dn = cplx ? 2 * g.nk : g.n3;
        const int w = cplx ? 2 * g.P : (int)g.n3, dw = cplx ? 2 * g.PP : (int)g.n3;
        const int64_t rows = cplx ? (int64_t)g.N * g.N : 1;
        if (f == GEV_FIELD_BI) bi_sums = t0i_pending = false;
        ensure_stage(n, 0);
        for (int c = 0; c < planes; c++) {
            ck(cudaMemcpyAsync(stage.p, host + (int64_t)c * n, n * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
            k_convert_rows<double, R><<<cdiv(n, 256), 256, 0, st>>>(stage.p, w, (R *)p + (int64_t)c * dn, dw, w, rows);
            launched("convert");
            ck(cudaStreamSynchronize(st), "synchronize");
        }
    }

    void need_particles() const
    {
        if (!have_particles) throw StateError("no particles loaded");
    }

    void project(uint32_t which, double a, double coeff, int use_phi, int accumulate) override
    {
        need_particles();
        if (which & ~(GEV_PROJ_T00 | GEV_PROJ_TIJ | GEV_PROJ_T0I | GEV_PROJ_CIC | GEV_PROJ_T0I_SUMS))
            throw ArgError("unknown projection");
        if (which & GEV_PROJ_T0I_SUMS) {
            if (which != (GEV_PROJ_T00 | GEV_PROJ_TIJ | GEV_PROJ_T0I_SUMS) || !use_phi || accumulate)
                throw ArgError("GEV_PROJ_T0I_SUMS goes with T00 | TIJ, use_phi and no accumulate");
            project_t0i_sums(a, coeff);
            return;
        }
        if ((which & GEV_PROJ_CIC) && (which & GEV_PROJ_T00)) throw ArgError("CIC and T00 both target the source field");
        if (use_phi && a <= 0.0 && (which & (GEV_PROJ_T00 | GEV_PROJ_TIJ))) throw ArgError("scale factor must be positive");
        const double n3 = (double)g.n3;   // 1/dx^3
        if ((which & GEV_PROJ_T00) || (which & GEV_PROJ_TIJ)) {
            double m00 = mass * coeff * n3;
            if (use_phi) m00 /= a;                       // gevolution.hpp:1731, :1750
            double mij = mass * coeff * n3 / a;          // gevolution.hpp:2584
            DepOut<R> o{};
            int kind;
            if ((which & GEV_PROJ_T00) && (which & GEV_PROJ_TIJ)) {
                kind = DEP_T00_TIJ;
                o.p[0] = source.p;
                for (int c = 0; c < 6; c++) o.p[1 + c] = Sij.p + c * g.n3;
            } else if (which & GEV_PROJ_T00) {
                kind = DEP_T00;
                o.p[0] = source.p;
            } else {
                kind = DEP_TIJ;
                for (int c = 0; c < 6; c++) o.p[c] = Sij.p + c * g.n3;
            }
            deposit(kind, use_phi != 0, o, a, m00, mij, 0.0, accumulate, "deposit T00/Tij");
        }
        if (which & GEV_PROJ_CIC) {
            DepOut<R> o{};
            o.p[0] = source.p;
            deposit(DEP_T00, false, o, 1.0, mass * coeff * n3, 0.0, 0.0, accumulate, "deposit CIC");
        }
        if (which & GEV_PROJ_T0I) {
            DepOut<R> o{};
            for (int c = 0; c < 3; c++) o.p[c] = Bi.p + c * g.n3;
            deposit(DEP_T0I, use_phi != 0, o, 1.0, mass * coeff * n3, 0.0, 0.0, accumulate, "deposit T0i");
            bi_sums = false;
            t0i_pending = false;
        }
    }

    // One deposit for the cycle's three projections.  T0i's potential enters
    // only as the per-vertex factor 1 + phi(x) + phi(x + e_i)
    // (particle_T0i_project, gevolution.hpp:2031-2201) and the particles do
    // not move between main.cu's T00/Tij and T0i projections, so the
    // potential-free sums S_i are deposited here with T00 and Tij (previous
    // phi), and solve_B's x pass multiplies them by the factor with the phi of
    // its call (the new phi, as main.cu:836-955 uses).
    void project_t0i_sums(double a, double coeff)
    {
        need_particles();
        if (a <= 0.0) throw ArgError("scale factor must be positive");
        if constexpr (sizeof(R) == 8) {
            // FP64: 16-value records would leave one CTA per SM; the T0i
            // deposit runs on its own at the start of solve_B instead
            project(GEV_PROJ_T00 | GEV_PROJ_TIJ, a, coeff, 1, 0);
            t0i_pending = true;
            t0i_coeff = coeff;
            return;
        }
        const double n3 = (double)g.n3 * coeff;
        DepOut<R> o{};
        o.p[0] = source.p;
        for (int c = 0; c < 6; c++) o.p[1 + c] = Sij.p + c * g.n3;
        for (int c = 0; c < 3; c++) o.p[7 + c] = Bi.p + c * g.n3;
        // gevolution.hpp:1731, :1750, :2584; T0i mass * coeff / dx^3
        deposit(DEP_T00_TIJ_S0I, true, o, a, mass * n3 / a, mass * n3 / a, mass * n3, 0, "deposit T00/Tij/T0i sums");
        bi_sums = true;
    }

    void solve_phi(int prepare, double bg, double c, double c2, double c3, double pc, double modif, double *sum,
                   double *phom) override
    {
        const int N = g.N;
        const FftTables<R> tb = tables();
        fx_forward<R>(N, prepare ? FX_PREP_T00 : FX_COPY, source.p, g.n3, 1, 0, phi.p, chi.p, bg, c, c2, c3, W.p, g.nk,
                      partial.p, tb, st);
        launched("fx forward (phi)");
        if (prepare) {
            launch_reduce_sum(partial.p, (int64_t)(N / fx_rows_per_block(N, sizeof(R) == 8)) * N, scal.p, st);
            launched("reduce");
        }
        fy_pass<R>(N, -1, W.p, g.nk, 1, derr.p, tb, st);
        launched("fy forward (phi)");
        FzParams fp{};
        fp.err = derr.p;
        fp.op = OP_POISSON;
        fp.p0 = pc / -((double)N * (double)N * (double)N);
        fp.p1 = modif;
        fp.phi_hom = scal.p + 1;
        fz_pass<R>(N, fp, W.p, g.nk, nullptr, nullptr, nullptr, tb, st);
        launched("fz Poisson");
        fy_pass<R>(N, 1, W.p, g.nk, 1, derr.p, tb, st);
        launched("fy inverse (phi)");
        fx_inverse<R>(N, W.p, g.nk, phi.p, g.n3, 1, tb, st);
        launched("fx inverse (phi)");
        if (sum || phom) {
            double h[2] = {0.0, 0.0};
            ck(cudaMemcpyAsync(h, scal.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
            sync();
            if (sum) *sum = prepare ? h[0] : 0.0;
            if (phom) *phom = h[1];
        }
    }

    // prepareFTsource on its own, in place (main.cu:725, :822): the T00 form
    // returns the sum of the source field before the preparation
    double prepare_t00(double bg, double c, double c2, double c3) override
    {
        const int N = g.N;
        prep_t00_pass<R>(N, source.p, phi.p, chi.p, bg, c, c2, c3, partial.p, st);
        launched("prepare T00");
        launch_reduce_sum(partial.p, (int64_t)N * N, scal.p, st);
        launched("reduce");
        double h = 0.0;
        ck(cudaMemcpyAsync(&h, scal.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        sync();
        return h;
    }

    void prepare_tij(double coeff) override
    {
        prep_tij_pass<R>(g.N, Sij.p, phi.p, coeff, st);
        launched("prepare Tij");
    }

    void solve_chi(double coeff, int cycle0, double hubble, double dtau, double dtau_old, double a2dtau) override
    {
        int extra = 0;
        if (cfg.tensor) extra |= cycle0 ? EXTRA_TENSOR_PROJECT : EXTRA_TENSOR_EVOLVE;
        if (cfg.vector_method == GEV_VECTOR_PARABOLIC) extra |= EXTRA_VECTOR_EVOLVE;
        chi_pass(coeff, extra, hubble, dtau, dtau_old, a2dtau);
    }

    // prepareFTsource(phi, Sij, Sij, coeff), the six forward FFTs,
    // projectFTscalar with the given extras, the backward FFT(s)
    void chi_pass(double coeff, int extra, double hubble, double dtau, double dtau_old, double a2dtau)
    {
        const int N = g.N;
        const FftTables<R> tb = tables();
        fx_forward<R>(N, FX_PREP_TIJ, Sij.p, g.n3, 6, 0, phi.p, chi.p, 0, coeff, 0, 0, W.p, g.nk, nullptr, tb, st);
        launched("fx forward (Sij)");
        fy_pass<R>(N, -1, W.p, g.nk, 6, derr.p, tb, st);
        launched("fy forward (Sij)");
        FzParams fp{};
        fp.err = derr.p;
        fp.op = OP_SCALAR;
        fp.extra = extra;
        const bool parab = (extra & EXTRA_VECTOR_EVOLVE) != 0;
        fp.p0 = hubble; fp.p1 = dtau; fp.p2 = dtau_old; fp.p3 = a2dtau;
        fz_pass<R>(N, fp, W.p, g.nk, hij.p, hijp.p, bstate.p, tb, st);
        launched("fz scalar projection");
        const int nout = parab ? 4 : 1;
        fy_pass<R>(N, 1, W.p, g.nk, nout, derr.p, tb, st);
        launched("fy inverse (chi)");
        fx_inverse<R>(N, W.p, g.nk, chi.p, g.n3, 1, tb, st);
        launched("fx inverse (chi)");
        if (parab) {
            fx_inverse<R>(N, W.p + g.nk, g.nk, Bi.p, g.n3, 3, tb, st);
            launched("fx inverse (B)");
            bi_sums = false;
        }
    }

    void solve_B(double coeff, double modif) override
    {
        const int N = g.N;
        const FftTables<R> tb = tables();
        // T0i straight from project(T0I), or completed from project_step's sums with the current phi
        if (t0i_pending) project(GEV_PROJ_T0I, 1.0, t0i_coeff, 1, 0);
        t0i_pending = false;
        fx_forward<R>(N, bi_sums ? FX_PREP_T0I : FX_COPY, Bi.p, g.n3, 3, 0, phi.p, nullptr, 0, 0, 0, 0, W.p, g.nk,
                      nullptr, tb, st);
        launched("fx forward (T0i)");
        bi_sums = false;
        fy_pass<R>(N, -1, W.p, g.nk, 3, derr.p, tb, st);
        launched("fy forward (T0i)");
        FzParams fp{};
        fp.err = derr.p;
        fp.op = OP_VECTOR;
        fp.p0 = coeff;
        fp.p1 = modif;
        fz_pass<R>(N, fp, W.p, g.nk, nullptr, nullptr, nullptr, tb, st);
        launched("fz vector projection");
        fy_pass<R>(N, 1, W.p, g.nk, 3, derr.p, tb, st);
        launched("fy inverse (B)");
        fx_inverse<R>(N, W.p, g.nk, Bi.p, g.n3, 3, tb, st);
        launched("fx inverse (B)");
    }

    double kick_drift(const KickDriftParams &kp) override
    {
        need_particles();
        const int64_t nb = g.ntiles * 8;
        if (kp.do_bin) ck(cudaMemsetAsync(counts.p, 0, nb * sizeof(uint32_t), st), "memset");
        ck(cudaMemsetAsync(u64.p, 0, sizeof(unsigned long long), st), "memset");
        launch_kick_drift<R>(cur(), bstart.p, g.N, phi.p, chi.p, Bi.p, g.n3, kp, counts.p, bucket.p, rank.p, u64.p, derr.p, st);
        launched("kick/drift");
        if (kp.do_bin) finish_rebin();
        double maxvel = 0.0;
        if (kp.do_kick) {
            unsigned long long bits = 0;
            ck(cudaMemcpyAsync(&bits, u64.p, sizeof(bits), cudaMemcpyDeviceToHost, st), "D2H");
            sync();
            double v2;
            std::memcpy(&v2, &bits, sizeof v2);
            maxvel = std::sqrt(v2);
        }
        return maxvel;
    }

    void power_spectrum(int nb, double kmax, double *kb, double *pw, double *ksc, double *ps, int32_t *occo) override
    {
        need_particles();
        if (nb <= 0) throw ArgError("numbins must be positive");
        const int N = g.N;
        if (kmax <= 0.0) {
            // tools.hpp:144-145 with KTYPE_LINEAR, in the reference's own order of
            // operations: modes with |n|^2 = 3 m^2 lie exactly on bin edges, where
            // one ulp of kmax decides their bin
            double t = 2.0 * M_PI * (double)(N / 2);
            t *= t;
            kmax = std::sqrt(3.0 * t);
        }
        if ((int)occ.n < nb) { bins.alloc(4 * nb, "bins"); occ.alloc(nb, "bins"); }
        ck(cudaMemsetAsync(bins.p, 0, 4 * nb * sizeof(double), st), "memset");
        ck(cudaMemsetAsync(occ.p, 0, nb * sizeof(unsigned long long), st), "memset");
        FzParams fp{};
        fp.err = derr.p;
        fp.op = OP_BIN;
        fp.p0 = nb;
        fp.p1 = kmax;
        fp.bins = bins.p;
        fp.occ = occ.p;
        if constexpr (sizeof(R) == 8) {
            project(GEV_PROJ_CIC, 1.0, 1.0, 0, 0);
            const FftTables<R> tb = tables();
            fx_forward<R>(N, FX_COPY, source.p, g.n3, 1, 0, nullptr, nullptr, 0, 0, 0, 0, W.p, g.nk, nullptr, tb, st);
            launched("fx forward (CIC)");
            fy_pass<R>(N, -1, W.p, g.nk, 1, derr.p, tb, st);
            launched("fy forward (CIC)");
            fz_pass<R>(N, fp, W.p, g.nk, nullptr, nullptr, nullptr, tb, st);
            launched("fz binning");
        } else {
            // Mixed precision measures in FP64: the density contrast of an early,
            // nearly uniform box is ~1e-2 of the density, and FP32 rounding of the
            // density itself would set the small-scale floor of the spectrum.
            // FP64 CIC density of the FP64 positions (atomic adds), FP64
            // transform and binning in the first two FP32 components of W; the
            // FP32 copy of the density is left in the source field as in FP64.
            if (!rho64.p) {
                rho64.alloc(g.n3, "FP64 density");
                make_tables64();
            }
            ck(cudaMemsetAsync(rho64.p, 0, g.n3 * sizeof(double), st), "memset");
            launch_cic_f64<R>(cur(), N, mass * (double)g.n3, rho64.p, st);
            launched("CIC density (FP64)");
            launch_f64_to_f32(rho64.p, g.n3, reinterpret_cast<float *>(source.p), st);
            launched("density to FP32");
            const FftTables<double> tb{tw64_full.p, tw64_half.p, k2.p, ks.p};
            double2 *W64 = reinterpret_cast<double2 *>(W.p);   // W holds 6 FP32 components = 3 FP64 ones
            fx_forward<double>(N, FX_COPY, rho64.p, g.n3, 1, 0, nullptr, nullptr, 0, 0, 0, 0, W64, g.nk, nullptr, tb, st);
            launched("fx forward (CIC, FP64)");
            fy_pass<double>(N, -1, W64, g.nk, 1, derr.p, tb, st);
            launched("fy forward (CIC, FP64)");
            fz_pass<double>(N, fp, W64, g.nk, nullptr, nullptr, nullptr, tb, st);
            launched("fz binning (FP64)");
        }
        std::vector<double> acc(4 * nb);
        std::vector<unsigned long long> oc(nb);
        ck(cudaMemcpyAsync(acc.data(), bins.p, 4 * nb * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(oc.data(), occ.p, nb * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st), "D2H");
        sync();
        // final normalisation, tools.hpp:292-313
        for (int i = 0; i < nb; i++) {
            occo[i] = (int32_t)oc[i];
            if (oc[i] > 0) {
                double o = (double)oc[i];
                kb[i] = acc[i];
                ksc[i] = std::sqrt(acc[nb + i] * o - kb[i] * kb[i]) / o;
                if (!std::isfinite(ksc[i])) ksc[i] = 0.0;
                kb[i] /= o;
                pw[i] = acc[2 * nb + i] / o;
                ps[i] = std::sqrt(acc[3 * nb + i] / o - pw[i] * pw[i]);
                if (!std::isfinite(ps[i])) ps[i] = 0.0;
            } else {
                kb[i] = pw[i] = ksc[i] = ps[i] = 0.0;
            }
        }
    }

    // The shell's kernel arguments and output buffers for this cycle; false when
    // the shell writes nothing this cycle (output.hpp:2093), with the backlog
    // cleared as the reference does (output.hpp:2172).
    bool lightcone_setup(const gev_lightcone_args &lc, double tau, double dtau, double dtau_old, double a,
                         double dadtau, int64_t cap, LcKernelArgs &la, LcOut &lo)
    {
        need_particles();
        if (lc.shell < 0 || lc.shell >= 8) throw ArgError("lightcone shell slot must be 0..7");
        const int s = lc.shell;
        const double dist = lc.d - tau;
        if (!(lc.distance[0] > dist + 0.5 * dtau_old && lc.distance[1] <= dist + 0.5 * dtau_old && dist + 0.5 * dtau_old > 0.)) {
            backlog_valid[s] = false;
            lc_last = 0;
            return false;
        }
        la = LcKernelArgs{};
        const int N = g.N;
        double domain[6];
        for (int i = 0; i < 3; i++) { domain[i] = -0.5 / N; domain[i + 3] = (N + 0.5) / N; }   // output.hpp:1174-1186
        la.inner = dist - 0.5 * dtau;
        la.outer = dist + (0.5 + 0.05) * dtau_old;
        la.dist = dist;
        la.nvtx = find_intersecting(lc.vertex, lc.direction, lc.opening, la.outer, la.inner, domain, la.vtx);
        for (int i = 0; i < 3; i++) { la.lc_vertex[i] = lc.vertex[i]; la.direction[i] = lc.direction[i]; }
        la.opening = lc.opening;
        la.dtau = dtau; la.dtau_old = dtau_old; la.a = a; la.dadtau = dadtau; la.boxsize = cfg.boxsize;
        la.tracer_factor = lc.tracer_factor > 0 ? lc.tracer_factor : 1;
        // ID sets: capacity a power of two >= np/4 (the log holds particles within
        // 0.1 dtau of the inner edge, a small fraction of the box)
        if (idset_cap == 0) {
            int64_t c = 1 << 16;
            while (c < np / 4) c <<= 1;
            idset_cap = c;
        }
        for (int b = 0; b < 2; b++)
            if (!idset[s][b].p) {
                idset[s][b].alloc(idset_cap, "lightcone ID log");
                ck(cudaMemsetAsync(idset[s][b].p, 0xff, idset_cap * sizeof(unsigned long long), st), "memset");
            }
        unsigned long long *older = idset[s][idset_cur[s]].p, *newer = idset[s][1 - idset_cur[s]].p;
        la.backlog = older;
        la.backlog_cap = backlog_valid[s] ? idset_cap : 0;
        ck(cudaMemsetAsync(newer, 0xff, idset_cap * sizeof(unsigned long long), st), "memset");
        const int64_t lcap = std::max<int64_t>(cap, 1);
        la.capacity = lcap;
        if ((int64_t)lc_id.n < lcap) { lc_pos.alloc(3 * lcap, "lightcone"); lc_vel.alloc(3 * lcap, "lightcone"); lc_id.alloc(lcap, "lightcone"); }
        ck(cudaMemsetAsync(u64.p + 1, 0, sizeof(unsigned long long), st), "memset");
        lo = LcOut{lc_pos.p, lc_vel.p, lc_id.p, u64.p + 1, newer, idset_cap};
        return true;
    }

    // after the shell's kernel: the IDs logged near the inner edge become the
    // next cycle's backlog; returns the number selected (synchronises)
    int64_t lightcone_count(int shell)
    {
        idset_cur[shell] = 1 - idset_cur[shell];
        backlog_valid[shell] = true;
        unsigned long long cnt = 0;
        ck(cudaMemcpyAsync(&cnt, u64.p + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st), "D2H");
        sync();
        lc_last = (int64_t)cnt;
        return (int64_t)cnt;
    }

    void lightcone(const gev_lightcone_args &lc, double tau, double dtau, double dtau_old, double a, double dadtau,
                   int64_t cap, float *pos, float *vel, int64_t *ids, int64_t *n_out) override
    {
        *n_out = 0;
        LcKernelArgs la;
        LcOut lo;
        if (!lightcone_setup(lc, tau, dtau, dtau_old, a, dadtau, cap, la, lo)) return;
        launch_lightcone<R>(cur(), bstart.p, g.N, phi.p, la, lo.pos, lo.vel, lo.ids, lo.count, lo.newlog,
                            lo.newlog_cap, derr.p, st);
        launched("lightcone");
        *n_out = lightcone_count(lc.shell);
        if (*n_out > la.capacity) throw CapacityError("lightcone output exceeds the buffer capacity (n_out holds the required size)");
        if (pos || vel || ids) fetch_lightcone(cap, pos, vel, ids, n_out);
    }

    void fetch_lightcone(int64_t cap, float *pos, float *vel, int64_t *ids, int64_t *n_out) override
    {
        *n_out = lc_last;
        if (lc_last > cap) throw CapacityError("host arrays smaller than the lightcone output");
        const int64_t n = lc_last;
        if (n > 0) {
            if (pos) ck(cudaMemcpyAsync(pos, lc_pos.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
            if (vel) ck(cudaMemcpyAsync(vel, lc_vel.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
            if (ids) ck(cudaMemcpyAsync(ids, lc_id.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost, st), "D2H");
        }
        ck(cudaStreamSynchronize(st), "synchronize");
    }
};

}  // namespace gev

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct gev_ctx {
    std::unique_ptr<gev::CtxBase> impl;
    std::string err;
};

namespace {

int fail(gev_ctx *ctx, int code, const char *msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

template <class F> int guarded(gev_ctx *ctx, F &&f)
{
    if (!ctx || !ctx->impl) return GEV_ERR_ARG;
    try {
        f(*ctx->impl);
        return GEV_OK;
    } catch (const gev::ArgError &e) {
        return fail(ctx, GEV_ERR_ARG, e.what());
    } catch (const gev::StateError &e) {
        return fail(ctx, GEV_ERR_STATE, e.what());
    } catch (const gev::DeviceError &e) {
        return fail(ctx, GEV_ERR_DEVICE, e.what());
    } catch (const gev::CapacityError &e) {
        return fail(ctx, GEV_ERR_CAPACITY, e.what());
    } catch (const gev::NoMemError &e) {
        return fail(ctx, GEV_ERR_NOMEM, e.what());
    } catch (const std::exception &e) {
        return fail(ctx, GEV_ERR_CUDA, e.what());
    }
}

bool supported_N(int N)
{
    for (int n : {16, 32, 64, 128, 256, 384, 512, 768})
        if (N == n) return true;
    return false;
}

thread_local std::string g_create_error;

}  // namespace

extern "C" {

const char *gev_version(void) { return "gevolution-b200 1.0 (sm_100a)"; }

int gev_ctx_create(const gev_config *cfg, gev_ctx **out)
{
    if (!cfg || !out) return GEV_ERR_ARG;
    *out = nullptr;
    if (!supported_N(cfg->N) || (cfg->precision != GEV_FP64 && cfg->precision != GEV_MIXED) || cfg->capacity < 0 ||
        (cfg->vector_method != GEV_VECTOR_ELLIPTIC && cfg->vector_method != GEV_VECTOR_PARABOLIC)) {
        g_create_error = "invalid configuration (N must be one of 16,32,64,128,256,384,512,768)";
        return GEV_ERR_ARG;
    }
    auto *c = new gev_ctx;
    try {
        if (cfg->precision == GEV_FP64) c->impl.reset(new gev::Ctx<double>(*cfg));
        else c->impl.reset(new gev::Ctx<float>(*cfg));
    } catch (const gev::NoMemError &e) {
        g_create_error = e.what();
        delete c;
        return GEV_ERR_NOMEM;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        delete c;
        return GEV_ERR_CUDA;
    }
    *out = c;
    return GEV_OK;
}

int gev_ctx_destroy(gev_ctx *ctx)
{
    delete ctx;
    return GEV_OK;
}

const char *gev_last_error(const gev_ctx *ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int gev_particles_set(gev_ctx *ctx, const double *pos, const double *q, const int64_t *id, int64_t n, double mass)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.particles_set(pos, q, id, n, mass); });
}

int gev_particles_get(gev_ctx *ctx, double *pos, double *q, int64_t *id, int64_t capacity, int64_t *n_out)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.particles_get(pos, q, id, capacity, n_out); });
}

int gev_particles_exchange(gev_ctx *ctx, double *pos_out, double *q_out, int64_t *id_out, int64_t capacity,
                           int64_t *n_out, const double *pos_in, const double *q_in, const int64_t *id_in, int64_t n_in,
                           double mass)
{
    return guarded(ctx, [&](gev::CtxBase &c) {
        c.particles_exchange(pos_out, q_out, id_out, capacity, n_out, pos_in, q_in, id_in, n_in, mass);
    });
}

int gev_particles_count(const gev_ctx *ctx, int64_t *n_out)
{
    if (!ctx || !ctx->impl || !n_out) return GEV_ERR_ARG;
    *n_out = ctx->impl->particles_count();
    return GEV_OK;
}

int gev_field_components(int32_t field)
{
    switch (field) {
    case GEV_FIELD_PHI: case GEV_FIELD_CHI: case GEV_FIELD_SOURCE: return 1;
    case GEV_FIELD_SIJ: case GEV_FIELD_HIJ_FT: case GEV_FIELD_HIJP_FT: return 6;
    case GEV_FIELD_BI: case GEV_FIELD_BI_FT: return 3;
    default: return 0;
    }
}

int gev_field_get(gev_ctx *ctx, int32_t field, double *host)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.field_get(field, host); });
}

int gev_field_set(gev_ctx *ctx, int32_t field, const double *host)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.field_set(field, host); });
}

int gev_project(gev_ctx *ctx, uint32_t which, double a, double coeff, int32_t use_phi, int32_t accumulate)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.project(which, a, coeff, use_phi, accumulate); });
}

int gev_solve_phi(gev_ctx *ctx, int32_t prepare, double bgmodel, double coeff, double coeff2, double coeff3,
                  double poisson_coeff, double modif, double *T00sum, double *phi_hom)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.solve_phi(prepare, bgmodel, coeff, coeff2, coeff3, poisson_coeff, modif, T00sum, phi_hom); });
}

int gev_prepare_T00(gev_ctx *ctx, double bgmodel, double coeff, double coeff2, double coeff3, double *T00sum)
{
    return guarded(ctx, [&](gev::CtxBase &c) {
        const double s = c.prepare_t00(bgmodel, coeff, coeff2, coeff3);
        if (T00sum) *T00sum = s;
    });
}

int gev_prepare_Tij(gev_ctx *ctx, double coeff)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.prepare_tij(coeff); });
}

int gev_solve_chi(gev_ctx *ctx, double coeff, int32_t cycle0, double hubble, double dtau, double dtau_old, double a2dtau)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.solve_chi(coeff, cycle0, hubble, dtau, dtau_old, a2dtau); });
}

int gev_solve_B(gev_ctx *ctx, double coeff, double modif)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.solve_B(coeff, modif); });
}

int gev_kick(gev_ctx *ctx, double dtau, double a, double bcoeff, int32_t nfield, double *maxvel)
{
    return guarded(ctx, [&](gev::CtxBase &c) {
        gev::KickDriftParams kp{};
        kp.dtau_k = dtau; kp.a_k = a; kp.b_k = bcoeff; kp.nfield_k = nfield; kp.do_kick = 1;
        double v = c.kick_drift(kp);
        if (maxvel) *maxvel = v;
    });
}

int gev_drift(gev_ctx *ctx, double dtau, double a, double bcoeff, int32_t nfield)
{
    return guarded(ctx, [&](gev::CtxBase &c) {
        gev::KickDriftParams kp{};
        kp.dtau_d = dtau; kp.a_d = a; kp.b_d = bcoeff; kp.nfield_d = nfield; kp.do_drift = 1; kp.do_bin = 1;
        c.kick_drift(kp);
    });
}

int gev_kick_drift(gev_ctx *ctx, double dtau_kick, double a_kick, double bcoeff_kick, int32_t nfield_kick,
                   double dtau_drift, double a_drift, double bcoeff_drift, int32_t nfield_drift, double *maxvel)
{
    return guarded(ctx, [&](gev::CtxBase &c) {
        gev::KickDriftParams kp{};
        kp.dtau_k = dtau_kick; kp.a_k = a_kick; kp.b_k = bcoeff_kick; kp.nfield_k = nfield_kick;
        kp.dtau_d = dtau_drift; kp.a_d = a_drift; kp.b_d = bcoeff_drift; kp.nfield_d = nfield_drift;
        kp.do_kick = 1; kp.do_drift = 1; kp.do_bin = 1;
        double v = c.kick_drift(kp);
        if (maxvel) *maxvel = v;
    });
}

int gev_power_spectrum(gev_ctx *ctx, int32_t numbins, double kmax, double *kbin, double *power, double *kscatter,
                       double *pscatter, int32_t *occupation)
{
    if (!kbin || !power || !kscatter || !pscatter || !occupation) return fail(ctx, GEV_ERR_ARG, "null output array");
    return guarded(ctx, [&](gev::CtxBase &c) { c.power_spectrum(numbins, kmax, kbin, power, kscatter, pscatter, occupation); });
}

int gev_lightcone(gev_ctx *ctx, const gev_lightcone_args *lc, double tau, double dtau, double dtau_old, double a,
                  double dadtau, int64_t capacity, float *pos, float *vel, int64_t *ids, int64_t *n_out)
{
    if (!lc || !n_out || capacity < 0) return fail(ctx, GEV_ERR_ARG, "null argument");
    return guarded(ctx, [&](gev::CtxBase &c) { c.lightcone(*lc, tau, dtau, dtau_old, a, dadtau, capacity, pos, vel, ids, n_out); });
}

int gev_lightcone_fetch(gev_ctx *ctx, int64_t capacity, float *pos, float *vel, int64_t *ids, int64_t *n_out)
{
    if (!n_out) return fail(ctx, GEV_ERR_ARG, "null argument");
    return guarded(ctx, [&](gev::CtxBase &c) { c.fetch_lightcone(capacity, pos, vel, ids, n_out); });
}

double gev_hconf(double a, double fourpiG, const gev_cosmo *cosmo) { return gev::hconf(a, fourpiG, *cosmo); }

void gev_rungekutta4bg(double *a, double fourpiG, const gev_cosmo *cosmo, double dtau) { gev::rk4bg(*a, fourpiG, *cosmo, dtau); }

double gev_particle_horizon(double a, double fourpiG, const gev_cosmo *cosmo) { return gev::particle_horizon(a, fourpiG, *cosmo); }

namespace {

// One cycle of main.cu:608-1317 (GR, CDM, elliptic or parabolic B); with lc,
// the lightcone shell between the solves and the kick.  A lightcone capacity
// overflow lets the cycle finish and is reported at the end.
int step_cycle(gev_ctx *ctx, const gev_cosmo *cosmo, gev_state *s, const gev_lightcone_args *lc, int64_t lc_cap,
               int64_t *lc_n)
{
    if (!cosmo || !s || (lc && (!lc_n || lc_cap < 0))) return fail(ctx, GEV_ERR_ARG, "null argument");
    bool lc_overflow = false;
    const int rc = guarded(ctx, [&](gev::CtxBase &c) {
        const gev_cosmo &cm = *cosmo;
        const int N = c.cfg.N;
        const double dx = 1.0 / N;
        double a = s->a;
        // T00 and Tij with the previous phi (main.cu:623, :756); with elliptic B
        // also the T0i sums that solve_B completes with the new phi
        const bool elliptic = c.cfg.vector_method == GEV_VECTOR_ELLIPTIC;
        c.project(GEV_PROJ_T00 | GEV_PROJ_TIJ | (elliptic ? GEV_PROJ_T0I_SUMS : 0u), a, 1.0, 1, 0);
        // phi (main.cu:719-809)
        if (s->dtau_old > 0.) {
            const double H = gev::hconf(a, cm.fourpiG, cm);
            double sum = 0.0, ph = 0.0;
            c.solve_phi(1, cm.Omega_m, 3. * H * dx * dx / s->dtau_old, cm.fourpiG * dx * dx / a, 3. * H * H * dx * dx,
                        1. / (dx * dx), 3. * H / s->dtau_old, &sum, &ph);
            s->T00hom = sum / ((double)N * N * N);
            s->phi_hom = ph;
        }
        // chi, h_ij (main.cu:820-966)
        const double H = gev::hconf(a, cm.fourpiG, cm);
        c.solve_chi(2. * cm.fourpiG * dx * dx / a, s->cycle == 0, H, s->dtau, s->dtau_old, a * a * s->dtau_old);
        // B elliptic with the new phi (main.cu:836-955): T0i completed in solve_B's x pass
        if (elliptic) c.solve_B(cm.fourpiG * dx * dx, 0.);
        // lightcone shell with this cycle's phi (main.cu:1040-1100)
        if (lc) {
            try {
                c.lightcone(*lc, s->tau, s->dtau, s->dtau_old, a, a * H, lc_cap, nullptr, nullptr, nullptr, lc_n);
            } catch (const gev::CapacityError &) {
                lc_overflow = true;
            }
        }
        // kick, background half step, drift, background half step (main.cu:1225-1283)
        gev::KickDriftParams kp{};
        kp.do_kick = 1; kp.do_drift = 1; kp.do_bin = 1;
        kp.dtau_k = 0.5 * (s->dtau + s->dtau_old);
        kp.a_k = a;
        kp.b_k = a * a * N;
        kp.nfield_k = (1. / a < cm.z_relax + 1.) ? 3 : 2;
        gev::rk4bg(a, cm.fourpiG, cm, 0.5 * s->dtau);
        kp.dtau_d = s->dtau;
        kp.a_d = a;
        kp.b_d = a * a * N;
        kp.nfield_d = (1. / a < cm.z_relax + 1.) ? 3 : 0;
        double mv = c.kick_drift(kp);
        gev::rk4bg(a, cm.fourpiG, cm, 0.5 * s->dtau);
        s->maxvel = mv / std::sqrt(mv * mv + 1.0);
        // step control (main.cu:1286-1310)
        s->tau += s->dtau;
        s->dtau_old = s->dtau;
        const double H2 = gev::hconf(a, cm.fourpiG, cm);
        s->dtau = (cm.Cf * dx < cm.steplimit / H2) ? cm.Cf * dx : cm.steplimit / H2;
        s->a = a;
        s->cycle++;
    });
    if (rc == GEV_OK && lc_overflow)
        return fail(ctx, GEV_ERR_CAPACITY, "lightcone output exceeds the buffer capacity (n_out holds the required size)");
    return rc;
}

}  // namespace

int gev_step(gev_ctx *ctx, const gev_cosmo *cosmo, gev_state *s) { return step_cycle(ctx, cosmo, s, nullptr, 0, nullptr); }

int gev_step_lightcone(gev_ctx *ctx, const gev_cosmo *cosmo, gev_state *s, const gev_lightcone_args *lc,
                       int64_t capacity, int64_t *n_out)
{
    if (!lc) return fail(ctx, GEV_ERR_ARG, "null argument");
    return step_cycle(ctx, cosmo, s, lc, capacity, n_out);
}

int gev_synchronize(gev_ctx *ctx)
{
    return guarded(ctx, [&](gev::CtxBase &c) { c.sync(); });
}

void *gev_stream(gev_ctx *ctx) { return (ctx && ctx->impl) ? (void *)ctx->impl->stream() : nullptr; }

int64_t gev_kernel_launches(const gev_ctx *ctx) { return (ctx && ctx->impl) ? ctx->impl->kernel_launches() : -1; }


int gev_ics_zeldovich(gev_ctx *ctx, const gev_ics_params *p)
{
    if (!p) return fail(ctx, GEV_ERR_ARG, "null argument");
    return guarded(ctx, [&](gev::CtxBase &c) { c.ics_zeldovich(*p); });
}

int gev_ics_basic(gev_ctx *ctx, const gev_ics_basic_params *p)
{
    if (!p) return fail(ctx, GEV_ERR_ARG, "null argument");
    return guarded(ctx, [&](gev::CtxBase &c) { c.ics_basic(*p); });
}

// ---- checkpoint / restart ----
// File: "GEVCKPT1", int32 {version, N, precision, vector_method, tensor, 0},
// int64 np, double {mass, boxsize}, gev_state, particles (pos 3np, q 3np as
// double, id np as int64), then the field planes as doubles: PHI, CHI, BI,
// and HIJ_FT, HIJP_FT (tensor state) and BI_FT (parabolic B state) when the
// context keeps them.  Fields are stored in FP64 whatever the precision mode.
namespace {
const char GEV_CKPT_MAGIC[8] = {'G', 'E', 'V', 'C', 'K', 'P', 'T', '1'};

int64_t field_doubles(const gev_config &c, int f)
{
    const int64_t N = c.N, P = c.N / 2 + 1;
    const bool ft = (f == GEV_FIELD_HIJ_FT || f == GEV_FIELD_HIJP_FT || f == GEV_FIELD_BI_FT);
    return (int64_t)gev_field_components(f) * (ft ? 2 * P * N * N : N * N * N);
}

std::vector<int> ckpt_fields(const gev_config &c)
{
    std::vector<int> f = {GEV_FIELD_PHI, GEV_FIELD_CHI, GEV_FIELD_BI};
    if (c.tensor) { f.push_back(GEV_FIELD_HIJ_FT); f.push_back(GEV_FIELD_HIJP_FT); }
    if (c.vector_method == GEV_VECTOR_PARABOLIC) f.push_back(GEV_FIELD_BI_FT);
    return f;
}

struct FileCloser {
    FILE *f;
    ~FileCloser() { if (f) fclose(f); }
};
}  // namespace

// ---- express particle files (Particles_gevolution.hpp:98-143, saveExpress
// :2641-2767, loadExpress :2769-2902) ----
// One file per rank, "<base>.<rank>" (a numeric suffix of the given name
// replaced): the 120-byte express header (magic "GEXPCDM", version 1, the
// writer's sizeof(Real), sizeof(long) and sizeof(gadget2_header), its rank and
// process grid, lattice sizes and coordinate skip, particle counts and block
// sizes), then positions (3 n Real, box units), momenta (3 n Real), IDs (n
// long) and the Gadget-2 header.  This library is one rank of a 1 x 1 grid.
namespace {
struct ExpressHeader {
    char magic[8];
    uint32_t version, header_size, endian, sizeof_real, sizeof_long, sizeof_gadget2_header;
    int32_t rank, size;
    int32_t grid_size[2];
    int32_t lat_size[3];
    int32_t lat_size_local[3];
    int32_t coord_skip[2];
    uint64_t local_npart, global_npart, position_bytes, momentum_bytes, id_bytes;
};
static_assert(sizeof(ExpressHeader) == 120, "express header layout");
const char EXPRESS_MAGIC_[8] = {'G', 'E', 'X', 'P', 'C', 'D', 'M', '\0'};

// express_rank_filename (Particles_gevolution.hpp:124-143) for rank 0
std::string express_file(const char *name)
{
    std::string f(name);
    const size_t dot = f.find_last_of('.');
    if (dot != std::string::npos && dot + 1 < f.size()) {
        bool digits = true;
        for (size_t i = dot + 1; i < f.size(); i++) digits = digits && f[i] >= '0' && f[i] <= '9';
        if (digits) f.resize(dot);
    }
    return f + ".0";
}
}  // namespace

int gev_express_write(gev_ctx *ctx, const char *filename, const gev_gadget2_header *hdr_in, int32_t real_bytes)
{
    if (!ctx || !ctx->impl || !filename || !hdr_in || (real_bytes != 4 && real_bytes != 8)) return GEV_ERR_ARG;
    return guarded(ctx, [&](gev::CtxBase &c) {
        const int64_t np = c.particles_count();
        std::vector<double> pos(3 * (size_t)np), q(3 * (size_t)np);
        std::vector<int64_t> id((size_t)np);
        int64_t got = 0;
        if (np > 0) c.particles_get(pos.data(), q.data(), id.data(), np, &got);
        gev_gadget2_header hdr = *hdr_in;   // saveExpress:2656-2659
        hdr.num_files = 1;
        hdr.npart[1] = (uint32_t)((uint64_t)np & 0xffffffffull);
        hdr.npartTotal[1] = (uint32_t)((uint64_t)np & 0xffffffffull);
        hdr.npartTotalHW[1] = (uint32_t)((uint64_t)np >> 32);
        ExpressHeader e;
        std::memset(&e, 0, sizeof e);
        std::memcpy(e.magic, EXPRESS_MAGIC_, 8);
        e.version = 1;
        e.header_size = sizeof e;
        e.endian = 0x01020304u;
        e.sizeof_real = (uint32_t)real_bytes;
        e.sizeof_long = 8;
        e.sizeof_gadget2_header = sizeof(gev_gadget2_header);
        e.rank = 0;
        e.size = 1;
        e.grid_size[0] = e.grid_size[1] = 1;
        for (int i = 0; i < 3; i++) e.lat_size[i] = e.lat_size_local[i] = c.cfg.N;
        e.local_npart = e.global_npart = (uint64_t)np;
        e.position_bytes = e.momentum_bytes = 3 * (uint64_t)np * (uint64_t)real_bytes;
        e.id_bytes = (uint64_t)np * 8;
        const std::string path = express_file(filename);
        FileCloser fc{fopen(path.c_str(), "wb")};
        if (!fc.f) throw gev::ArgError("cannot open " + path + " for writing");
        auto put_real = [&](const std::vector<double> &v) {
            if (real_bytes == 8) return fwrite(v.data(), 8, v.size(), fc.f) == v.size();
            std::vector<float> f(v.begin(), v.end());
            return fwrite(f.data(), 4, f.size(), fc.f) == f.size();
        };
        bool ok = fwrite(&e, sizeof e, 1, fc.f) == 1 && put_real(pos) && put_real(q) &&
                  fwrite(id.data(), 8, id.size(), fc.f) == id.size() && fwrite(&hdr, sizeof hdr, 1, fc.f) == 1;
        if (!ok) throw gev::ArgError("write error on " + path);
        if (fclose(fc.f) != 0) { fc.f = nullptr; throw gev::ArgError("write error on " + path); }
        fc.f = nullptr;
    });
}

int gev_express_read(gev_ctx *ctx, const char *filename, double mass, gev_gadget2_header *hdr_out)
{
    if (!ctx || !ctx->impl || !filename) return GEV_ERR_ARG;
    return guarded(ctx, [&](gev::CtxBase &c) {
        const std::string path = express_file(filename);
        FileCloser fc{fopen(path.c_str(), "rb")};
        if (!fc.f) throw gev::ArgError("cannot open " + path);
        ExpressHeader e;
        if (fread(&e, sizeof e, 1, fc.f) != 1) throw gev::ArgError(path + ": no express header");
        // loadExpress's layout checks (:2786-2812) for a one-rank reader; either Real size
        bool ok = std::memcmp(e.magic, EXPRESS_MAGIC_, 8) == 0 && e.version == 1 && e.header_size == sizeof e &&
                  e.endian == 0x01020304u && (e.sizeof_real == 4 || e.sizeof_real == 8) && e.sizeof_long == 8 &&
                  e.sizeof_gadget2_header == sizeof(gev_gadget2_header) && e.rank == 0 && e.size == 1 &&
                  e.grid_size[0] == 1 && e.grid_size[1] == 1 && e.coord_skip[0] == 0 && e.coord_skip[1] == 0;
        for (int i = 0; i < 3; i++) ok = ok && e.lat_size[i] == c.cfg.N && e.lat_size_local[i] == c.cfg.N;
        ok = ok && e.local_npart == e.global_npart && e.position_bytes == 3 * e.local_npart * e.sizeof_real &&
             e.momentum_bytes == 3 * e.local_npart * e.sizeof_real && e.id_bytes == e.local_npart * 8;
        if (!ok) throw gev::ArgError(path + " is not an express file of one rank on this lattice");
        const int64_t np = (int64_t)e.local_npart;
        if (np > c.cfg.capacity) throw gev::CapacityError("the express file holds more particles than the capacity");
        std::vector<double> pos(3 * (size_t)np), q(3 * (size_t)np);
        std::vector<int64_t> id((size_t)np);
        auto get_real = [&](std::vector<double> &v) {
            if (e.sizeof_real == 8) return fread(v.data(), 8, v.size(), fc.f) == v.size();
            std::vector<float> f(v.size());
            if (fread(f.data(), 4, f.size(), fc.f) != f.size()) return false;
            for (size_t i = 0; i < v.size(); i++) v[i] = f[i];
            return true;
        };
        gev_gadget2_header hdr;
        if (!get_real(pos) || !get_real(q) || fread(id.data(), 8, id.size(), fc.f) != id.size() ||
            fread(&hdr, sizeof hdr, 1, fc.f) != 1)
            throw gev::ArgError(path + ": truncated express file");
        const uint64_t total = (uint64_t)hdr.npartTotal[1] + ((uint64_t)hdr.npartTotalHW[1] << 32);
        if (total != e.global_npart || hdr.num_files != 1) throw gev::ArgError(path + ": Gadget-2 metadata does not match");
        c.particles_set(pos.data(), q.data(), id.data(), np, mass);
        if (hdr_out) *hdr_out = hdr;
    });
}

int gev_checkpoint_write(gev_ctx *ctx, const char *path, const gev_state *st)
{
    if (!ctx || !ctx->impl || !path || !st) return GEV_ERR_ARG;
    return guarded(ctx, [&](gev::CtxBase &c) {
        const int64_t np = c.particles_count();
        std::vector<double> pos(3 * (size_t)np), q(3 * (size_t)np);
        std::vector<int64_t> id((size_t)np);
        int64_t got = 0;
        if (np > 0) c.particles_get(pos.data(), q.data(), id.data(), np, &got);
        FileCloser fc{fopen(path, "wb")};
        if (!fc.f) throw gev::ArgError(std::string("cannot open ") + path + " for writing");
        const int32_t hdr[6] = {1, c.cfg.N, c.cfg.precision, c.cfg.vector_method, c.cfg.tensor, 0};
        const double md[2] = {c.particle_mass(), c.cfg.boxsize};
        bool ok = fwrite(GEV_CKPT_MAGIC, 8, 1, fc.f) == 1 && fwrite(hdr, sizeof hdr, 1, fc.f) == 1 &&
                  fwrite(&np, 8, 1, fc.f) == 1 && fwrite(md, sizeof md, 1, fc.f) == 1 &&
                  fwrite(st, sizeof(gev_state), 1, fc.f) == 1;
        if (np > 0)
            ok = ok && fwrite(pos.data(), 8, pos.size(), fc.f) == pos.size() && fwrite(q.data(), 8, q.size(), fc.f) == q.size() &&
                 fwrite(id.data(), 8, id.size(), fc.f) == id.size();
        for (int f : ckpt_fields(c.cfg)) {
            std::vector<double> buf((size_t)field_doubles(c.cfg, f));
            c.field_get(f, buf.data());
            ok = ok && fwrite(buf.data(), 8, buf.size(), fc.f) == buf.size();
        }
        if (!ok) throw gev::ArgError(std::string("write error on ") + path);
        if (fclose(fc.f) != 0) { fc.f = nullptr; throw gev::ArgError(std::string("write error on ") + path); }
        fc.f = nullptr;
    });
}

int gev_checkpoint_read(gev_ctx *ctx, const char *path, gev_state *st)
{
    if (!ctx || !ctx->impl || !path || !st) return GEV_ERR_ARG;
    return guarded(ctx, [&](gev::CtxBase &c) {
        FileCloser fc{fopen(path, "rb")};
        if (!fc.f) throw gev::ArgError(std::string("cannot open ") + path);
        char magic[8];
        int32_t hdr[6];
        int64_t np = 0;
        double md[2];
        gev_state s{};
        if (fread(magic, 8, 1, fc.f) != 1 || memcmp(magic, GEV_CKPT_MAGIC, 8) != 0) throw gev::ArgError("not a checkpoint file");
        if (fread(hdr, sizeof hdr, 1, fc.f) != 1 || fread(&np, 8, 1, fc.f) != 1 || fread(md, sizeof md, 1, fc.f) != 1 ||
            fread(&s, sizeof s, 1, fc.f) != 1)
            throw gev::ArgError("truncated checkpoint header");
        if (hdr[0] != 1) throw gev::ArgError("unsupported checkpoint version");
        if (hdr[1] != c.cfg.N || hdr[3] != c.cfg.vector_method || (hdr[4] != 0) != (c.cfg.tensor != 0))
            throw gev::ArgError("checkpoint grid or metric configuration differs from the context");
        if (np < 0 || np > c.cfg.capacity) throw gev::ArgError("checkpoint holds more particles than the context capacity");
        if (!(md[1] == c.cfg.boxsize)) throw gev::ArgError("checkpoint box size differs from the context");
        // the whole file is read before the context changes: a truncated or
        // mismatched file leaves the context's particles and fields as they were
        std::vector<double> pos(3 * (size_t)np), q(3 * (size_t)np);
        std::vector<int64_t> id((size_t)np);
        if (np > 0 && (fread(pos.data(), 8, pos.size(), fc.f) != pos.size() || fread(q.data(), 8, q.size(), fc.f) != q.size() ||
                       fread(id.data(), 8, id.size(), fc.f) != id.size()))
            throw gev::ArgError("truncated checkpoint particles");
        const std::vector<int> fields = ckpt_fields(c.cfg);
        std::vector<std::vector<double>> bufs;
        for (int f : fields) {
            bufs.emplace_back((size_t)field_doubles(c.cfg, f));
            std::vector<double> &buf = bufs.back();
            if (fread(buf.data(), 8, buf.size(), fc.f) != buf.size()) throw gev::ArgError("truncated checkpoint fields");
        }
        c.particles_set(pos.data(), q.data(), id.data(), np, md[0]);
        for (size_t i = 0; i < fields.size(); i++) c.field_set(fields[i], bufs[i].data());
        *st = s;
    });
}

}  // extern "C"
