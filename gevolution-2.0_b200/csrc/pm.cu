// pm.cu -- differentiable Newtonian particle-mesh run and its hand-written
// adjoint (C ABI gev_pm_*, include/gev.h).
//
// Forward step n (main.cu's gr_flag == 0 branch, CDM only):
//   rho   = scalarProjectionCIC_project          (gevolution.hpp:1902)
//   psi   = solveModifiedPoissonFT(rho, pc_n)     (gevolution.hpp:806, main.cu:765)
//   q    -= kq_n * grad psi (x)                   (update_q_Newton, gevolution.hpp:1051-1118,
//                                                  GRADIENT_ORDER 2; kq_n = dtau_kick * a * N)
//   x    += kx_n * q                              (update_pos_Newton, gevolution.hpp:1270-1273;
//                                                  kx_n = dtau / a_half)
// and after the last step the CIC density contrast delta = CIC(x) N^3/Np - 1.
//
// Particles are kept in ID order with unwrapped FP64 positions (box units), so
// the state is a smooth function of the initial conditions and no
// permutation has to be undone in the reverse pass; deposits use atomics
// (the grids of a differentiable run fit in L2).
//
// Reverse step n, given the cotangents (lx, lq) of (x_{n+1}, q_{n+1}):
//   lq'  = lq + kx lx                                   (drift)
//   lx  += -kq (d grad psi / dx)^T lq'                   (kick, at fixed psi)
//   Lam  = CIC deposit of lq' (3 components)             (transpose of the force gather)
//   lpsi = -kq sum_i (Lam_i(v - e_i) - Lam_i(v + e_i))/2 (transpose of the gradient stencil)
//   lrho = Poisson(lpsi, pc_n)                           (the solve is self-adjoint)
//   lx  += mass N^3 (d CIC / dx)^T lrho                  (transpose of the deposit)
//   lq   = lq'
// States x_n and potentials psi_n are recomputed segment by segment from
// checkpoints (x, q) stored every `checkpoint_every` steps.
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gev.h"
#include "kernels.h"

namespace gev {
namespace {

struct PmError : std::runtime_error {
    int code;
    PmError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void pck(cudaError_t e, const char *what)
{
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        throw PmError(GEV_ERR_NOMEM, std::string(what) + ": " + cudaGetErrorString(e));
    }
    if (e != cudaSuccess) throw PmError(GEV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T> struct PBuf {
    T *p = nullptr;
    size_t n = 0;
    void alloc(size_t count, const char *what)
    {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        pck(cudaMalloc((void **)&p, count * sizeof(T)), what);
        n = count;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~PBuf() { release(); }
};

constexpr int PM_NT = 256;

// cell corner and in-cell offset of an unwrapped box-unit coordinate
__device__ __forceinline__ void pm_cell(double x, int N, int &c, double &d)
{
    const double p = x * (double)N;
    const double f = floor(p);
    d = p - f;
    long long ci = (long long)f % N;
    if (ci < 0) ci += N;
    c = (int)ci;
}

__device__ __forceinline__ int pm_wrap1(int i, int N) { return i >= N ? i - N : (i < 0 ? i + N : i); }

// CIC deposit: out[comp][corner] += w * value (value = cst, or vals[3 i + comp])
template <class R, int NC>
__global__ void k_pm_deposit(const double *__restrict__ x, int64_t np, int N, const double *__restrict__ vals,
                             double cst, R *out)
{
    const int64_t n3 = (int64_t)N * N * N;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        int c[3];
        double d[3];
#pragma unroll
        for (int k = 0; k < 3; k++) pm_cell(x[3 * i + k], N, c[k], d[k]);
        double v[NC];
#pragma unroll
        for (int m = 0; m < NC; m++) v[m] = vals ? vals[3 * i + m] : cst;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
            const double w = (bx ? d[0] : 1.0 - d[0]) * (by ? d[1] : 1.0 - d[1]) * (bz ? d[2] : 1.0 - d[2]);
            const int64_t g = sidx(N, pm_wrap1(c[0] + bx, N), pm_wrap1(c[1] + by, N), pm_wrap1(c[2] + bz, N));
#pragma unroll
            for (int m = 0; m < NC; m++) atomicAdd(out + m * n3 + g, (R)(w * v[m]));
        }
    }
}

template <class R>
__device__ __forceinline__ double pm_ld(const R *f, int N, int x, int y, int z)
{
    return (double)__ldg(f + sidx(N, pm_wrap1(x, N), pm_wrap1(y, N), pm_wrap1(z, N)));
}

// G[i][k] = (psi(c_k + e_i) - psi(c_k - e_i)) / 2 at the 8 corners c_k of the cell
template <class R>
__device__ __forceinline__ void pm_grad_corners(const R *psi, int N, const int c[3], double G[3][8])
{
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int x = c[0] + ((k >> 2) & 1), y = c[1] + ((k >> 1) & 1), z = c[2] + (k & 1);
        G[0][k] = 0.5 * (pm_ld(psi, N, x + 1, y, z) - pm_ld(psi, N, x - 1, y, z));
        G[1][k] = 0.5 * (pm_ld(psi, N, x, y + 1, z) - pm_ld(psi, N, x, y - 1, z));
        G[2][k] = 0.5 * (pm_ld(psi, N, x, y, z + 1) - pm_ld(psi, N, x, y, z - 1));
    }
}

// forward kick (update_q_Newton) and drift (update_pos_Newton)
template <class R>
__global__ void k_pm_kick_drift(double *x, double *q, int64_t np, int N, const R *__restrict__ psi, double kq, double kx)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        int c[3];
        double d[3];
#pragma unroll
        for (int k = 0; k < 3; k++) pm_cell(x[3 * i + k], N, c[k], d[k]);
        double G[3][8];
        pm_grad_corners(psi, N, c, G);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            double g = 0.0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
                const double w = (bx ? d[0] : 1.0 - d[0]) * (by ? d[1] : 1.0 - d[1]) * (bz ? d[2] : 1.0 - d[2]);
                g += w * G[a][k];
            }
            const double qn = q[3 * i + a] - kq * g;
            q[3 * i + a] = qn;
            x[3 * i + a] += kx * qn;
        }
    }
}

// reverse of the drift and of the kick at fixed psi; lq becomes lq' (the
// cotangent of the kicked momentum), which the field part then deposits
template <class R>
__global__ void k_pm_adj_kick(const double *__restrict__ x, int64_t np, int N, const R *__restrict__ psi, double kq,
                              double kx, double *lx, double *lq)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        int c[3];
        double d[3];
#pragma unroll
        for (int k = 0; k < 3; k++) pm_cell(x[3 * i + k], N, c[k], d[k]);
        double lqp[3];
#pragma unroll
        for (int a = 0; a < 3; a++) lqp[a] = lq[3 * i + a] + kx * lx[3 * i + a];
        double G[3][8];
        pm_grad_corners(psi, N, c, G);
        // s_k = sum_a lq'_a G[a][k]; lx_m -= kq N sum_k dw_k/dd_m s_k
        double gm[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
            const double fx = bx ? d[0] : 1.0 - d[0], fy = by ? d[1] : 1.0 - d[1], fz = bz ? d[2] : 1.0 - d[2];
            const double sx = bx ? 1.0 : -1.0, sy = by ? 1.0 : -1.0, sz = bz ? 1.0 : -1.0;
            const double s = lqp[0] * G[0][k] + lqp[1] * G[1][k] + lqp[2] * G[2][k];
            gm[0] += sx * fy * fz * s;
            gm[1] += fx * sy * fz * s;
            gm[2] += fx * fy * sz * s;
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            lx[3 * i + a] -= kq * (double)N * gm[a];
            lq[3 * i + a] = lqp[a];
        }
    }
}

// lpsi(v) = -kq sum_i (Lam_i(v - e_i) - Lam_i(v + e_i)) / 2
template <class R>
__global__ void k_pm_adj_div(const R *__restrict__ lam, int N, double kq, R *lpsi)
{
    const int64_t n3 = (int64_t)N * N * N;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n3; g += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(g % N), y = (int)((g / N) % N), z = (int)(g / ((int64_t)N * N));
        double s = 0.0;
        s += pm_ld(lam, N, x - 1, y, z) - pm_ld(lam, N, x + 1, y, z);
        s += pm_ld(lam + n3, N, x, y - 1, z) - pm_ld(lam + n3, N, x, y + 1, z);
        s += pm_ld(lam + 2 * n3, N, x, y, z - 1) - pm_ld(lam + 2 * n3, N, x, y, z + 1);
        lpsi[g] = (R)(-kq * 0.5 * s);
    }
}

// lx_m += mf N sum_k dw_k/dd_m f(c_k): transpose of a CIC deposit of weight mf
template <class R>
__global__ void k_pm_adj_deposit(const double *__restrict__ x, int64_t np, int N, const R *__restrict__ f, double mf,
                                 double *lx)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        int c[3];
        double d[3];
#pragma unroll
        for (int k = 0; k < 3; k++) pm_cell(x[3 * i + k], N, c[k], d[k]);
        double gm[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int bx = (k >> 2) & 1, by = (k >> 1) & 1, bz = k & 1;
            const double fx = bx ? d[0] : 1.0 - d[0], fy = by ? d[1] : 1.0 - d[1], fz = bz ? d[2] : 1.0 - d[2];
            const double sx = bx ? 1.0 : -1.0, sy = by ? 1.0 : -1.0, sz = bz ? 1.0 : -1.0;
            const double v = pm_ld(f, N, c[0] + bx, c[1] + by, c[2] + bz);
            gm[0] += sx * fy * fz * v;
            gm[1] += fx * sy * fz * v;
            gm[2] += fx * fy * sz * v;
        }
#pragma unroll
        for (int a = 0; a < 3; a++) lx[3 * i + a] += mf * (double)N * gm[a];
    }
}

template <class R>
__global__ void k_pm_contrast(const R *__restrict__ rho, int64_t n3, double *out)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n3; g += (int64_t)gridDim.x * blockDim.x)
        out[g] = (double)rho[g] - 1.0;
}

template <class R>
__global__ void k_pm_to_field(const double *__restrict__ in, int64_t n3, R *out)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n3; g += (int64_t)gridDim.x * blockDim.x)
        out[g] = (R)in[g];
}

struct PmBase {
    virtual ~PmBase() = default;
    virtual void forward(int nsteps, const double *coef, const double *x0, const double *q0, double *delta,
                         double *xo, double *qo) = 0;
    virtual void adjoint(const double *ddelta, double *gx0, double *gq0) = 0;
    virtual cudaStream_t stream() = 0;
};

template <class R> struct Pm final : PmBase {
    using C = typename CT<R>::C;
    int N;
    int64_t np, n3, nk;
    double mass;
    int every;
    cudaStream_t st = nullptr;
    PBuf<R> rho, lam;
    PBuf<C> W, twf, twh;
    PBuf<double> k2;
    PBuf<double2> ks;
    PBuf<double> x, q, lx, lq;
    PBuf<int> derr;                                        // device error word of the Fourier passes
    std::vector<std::unique_ptr<PBuf<double>>> ckx, ckq;   // checkpoints (x, q) before steps 0, k, 2k, ...
    std::vector<std::unique_ptr<PBuf<double>>> segx;       // x_n within the segment being reversed
    std::vector<std::unique_ptr<PBuf<R>>> segpsi;          // psi_n within the segment
    std::vector<double> coefs;                             // 3 per step: kq, kx, pc
    int nsteps = 0;
    bool have_forward = false;

    Pm(const gev_pm_config &cfg) : N(cfg.N), np(cfg.np), mass(cfg.mass), every(cfg.checkpoint_every)
    {
        pck(cudaSetDevice(cfg.device), "cudaSetDevice");
        pck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        n3 = (int64_t)N * N * N;
        nk = (int64_t)(N / 2 + 2) * N * N;   // Fourier rows of pitch N/2+2
        rho.alloc(n3, "fields");
        lam.alloc(3 * n3, "fields");
        W.alloc(nk, "spectrum");
        x.alloc(3 * np, "particles");
        q.alloc(3 * np, "particles");
        lx.alloc(3 * np, "adjoint");
        lq.alloc(3 * np, "adjoint");
        derr.alloc(1, "error word");
        pck(cudaMemset(derr.p, 0, sizeof(int)), "memset");
        std::vector<C> tf(N), th(N / 2);
        for (int k = 0; k < N; k++) {
            const double ang = -2.0 * M_PI * (double)k / N;
            tf[k].x = (R)std::cos(ang);
            tf[k].y = (R)std::sin(ang);
        }
        for (int k = 0; k < N / 2; k++) {
            const double ang = -2.0 * M_PI * (double)k / (N / 2);
            th[k].x = (R)std::cos(ang);
            th[k].y = (R)std::sin(ang);
        }
        std::vector<double> hk2(N);
        std::vector<double2> hks(N);
        for (int i = 0; i < N; i++) {   // gevolution.hpp:269-275
            const double gk = 2.0 * (double)N * std::sin(M_PI * (double)i / (double)N);
            hks[i] = make_double2(gk * std::cos(M_PI * (double)i / (double)N), -gk * std::sin(M_PI * (double)i / (double)N));
            hk2[i] = gk * gk;
        }
        twf.alloc(N, "tables"); twh.alloc(N / 2, "tables"); k2.alloc(N, "tables"); ks.alloc(N, "tables");
        pck(cudaMemcpy(twf.p, tf.data(), N * sizeof(C), cudaMemcpyHostToDevice), "tables");
        pck(cudaMemcpy(twh.p, th.data(), (N / 2) * sizeof(C), cudaMemcpyHostToDevice), "tables");
        pck(cudaMemcpy(k2.p, hk2.data(), N * sizeof(double), cudaMemcpyHostToDevice), "tables");
        pck(cudaMemcpy(ks.p, hks.data(), N * sizeof(double2), cudaMemcpyHostToDevice), "tables");
    }
    ~Pm() override
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
    cudaStream_t stream() override { return st; }

    // after a synchronisation: a bulk tensor copy of a Fourier pass that timed
    // out leaves its pencils untransformed and sets the error word
    void check_device(const char *what)
    {
        int e = 0;
        pck(cudaMemcpy(&e, derr.p, sizeof(int), cudaMemcpyDeviceToHost), "error word");
        if (e) {
            pck(cudaMemset(derr.p, 0, sizeof(int)), "memset");
            throw PmError(GEV_ERR_DEVICE, std::string(what) + ": device error word (bulk tensor copy timed out)");
        }
    }

    unsigned pgrid() const { return (unsigned)std::min<int64_t>((np + PM_NT - 1) / PM_NT, 148 * 16); }
    unsigned fgrid() const { return (unsigned)std::min<int64_t>((n3 + PM_NT - 1) / PM_NT, 148 * 16); }
    FftTables<R> tables() const { return FftTables<R>{twf.p, twh.p, k2.p, ks.p}; }

    // field <- Poisson(field) with coefficient pc (modif 0): the pass sequence of gev_solve_phi
    void poisson(R *f, double pc)
    {
        const FftTables<R> tb = tables();
        fx_forward<R>(N, FX_COPY, f, n3, 1, 0, nullptr, nullptr, 0.0, 0.0, 0.0, 0.0, W.p, nk, nullptr, tb, st);
        fy_pass<R>(N, -1, W.p, nk, 1, derr.p, tb, st);
        FzParams fp{};
        fp.op = OP_POISSON;
        fp.p0 = pc / -((double)N * (double)N * (double)N);
        fp.p1 = 0.0;
        fp.err = derr.p;
        fz_pass<R>(N, fp, W.p, nk, nullptr, nullptr, nullptr, tb, st);
        fy_pass<R>(N, 1, W.p, nk, 1, derr.p, tb, st);
        fx_inverse<R>(N, W.p, nk, f, n3, 1, tb, st);
    }

    // psi_n of state x into `out`
    void potential(const double *xs, double pc, R *out)
    {
        pck(cudaMemsetAsync(out, 0, n3 * sizeof(R), st), "memset");
        k_pm_deposit<R, 1><<<pgrid(), PM_NT, 0, st>>>(xs, np, N, nullptr, mass * (double)n3, out);
        poisson(out, pc);
    }

    void step(int n, double *xs, double *qs, R *psi_out)
    {
        const double kq = coefs[3 * n], kx = coefs[3 * n + 1], pc = coefs[3 * n + 2];
        potential(xs, pc, psi_out);
        k_pm_kick_drift<R><<<pgrid(), PM_NT, 0, st>>>(xs, qs, np, N, psi_out, kq, kx);
    }

    void forward(int ns, const double *coef, const double *x0, const double *q0, double *delta, double *xo,
                 double *qo) override
    {
        nsteps = ns;
        coefs.assign(coef, coef + 3 * (size_t)ns);
        const int nck = (ns + every - 1) / every;
        while ((int)ckx.size() < nck) {
            ckx.emplace_back(new PBuf<double>());
            ckq.emplace_back(new PBuf<double>());
        }
        pck(cudaMemcpyAsync(x.p, x0, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "copy x0");
        pck(cudaMemcpyAsync(q.p, q0, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "copy q0");
        for (int n = 0; n < ns; n++) {
            if (n % every == 0) {
                PBuf<double> &cx = *ckx[n / every], &cq = *ckq[n / every];
                cx.alloc(3 * np, "checkpoint");
                cq.alloc(3 * np, "checkpoint");
                pck(cudaMemcpyAsync(cx.p, x.p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "checkpoint");
                pck(cudaMemcpyAsync(cq.p, q.p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "checkpoint");
            }
            step(n, x.p, q.p, rho.p);
        }
        // final CIC density contrast: mass N^3/Np per particle, minus one
        pck(cudaMemsetAsync(rho.p, 0, n3 * sizeof(R), st), "memset");
        k_pm_deposit<R, 1><<<pgrid(), PM_NT, 0, st>>>(x.p, np, N, nullptr, (double)n3 / (double)np, rho.p);
        k_pm_contrast<R><<<fgrid(), PM_NT, 0, st>>>(rho.p, n3, delta);
        if (xo) pck(cudaMemcpyAsync(xo, x.p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "copy x");
        if (qo) pck(cudaMemcpyAsync(qo, q.p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "copy q");
        pck(cudaGetLastError(), "forward launch");
        pck(cudaStreamSynchronize(st), "forward");
        check_device("forward");
        have_forward = true;
    }

    void adjoint(const double *ddelta, double *gx0, double *gq0) override
    {
        if (!have_forward) throw PmError(GEV_ERR_STATE, "gev_pm_adjoint needs a preceding gev_pm_forward");
        // cotangent of the final positions: transpose of the final deposit
        pck(cudaMemsetAsync(lx.p, 0, 3 * np * sizeof(double), st), "memset");
        pck(cudaMemsetAsync(lq.p, 0, 3 * np * sizeof(double), st), "memset");
        k_pm_to_field<R><<<fgrid(), PM_NT, 0, st>>>(ddelta, n3, rho.p);
        k_pm_adj_deposit<R><<<pgrid(), PM_NT, 0, st>>>(x.p, np, N, rho.p, (double)n3 / (double)np, lx.p);
        const int nseg = (nsteps + every - 1) / every;
        while ((int)segx.size() < every) {
            segx.emplace_back(new PBuf<double>());
            segpsi.emplace_back(new PBuf<R>());
        }
        for (int s = nseg - 1; s >= 0; s--) {
            const int n0 = s * every, n1 = std::min(nsteps, n0 + every);
            // recompute x_n and psi_n of the segment from its checkpoint; q.p (the
            // forward's final momenta were already copied out) is the working q
            pck(cudaMemcpyAsync(q.p, ckq[s]->p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "segment");
            for (int n = n0; n < n1; n++) {
                PBuf<double> &sx = *segx[n - n0];
                PBuf<R> &sp = *segpsi[n - n0];
                sx.alloc(3 * np, "segment");
                sp.alloc(n3, "segment");
                const double *src = (n == n0) ? ckx[s]->p : segx[n - n0 - 1]->p;
                pck(cudaMemcpyAsync(sx.p, src, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "segment");
                if (n > n0) {
                    // x_n = x_{n-1} advanced by step n-1 (q advanced in place in wq)
                    const double kq = coefs[3 * (n - 1)], kx = coefs[3 * (n - 1) + 1];
                    k_pm_kick_drift<R><<<pgrid(), PM_NT, 0, st>>>(sx.p, q.p, np, N, segpsi[n - n0 - 1]->p, kq, kx);
                }
                potential(sx.p, coefs[3 * n + 2], sp.p);
            }
            for (int n = n1 - 1; n >= n0; n--) {
                const double kq = coefs[3 * n], kx = coefs[3 * n + 1], pc = coefs[3 * n + 2];
                const double *xn = segx[n - n0]->p;
                k_pm_adj_kick<R><<<pgrid(), PM_NT, 0, st>>>(xn, np, N, segpsi[n - n0]->p, kq, kx, lx.p, lq.p);
                pck(cudaMemsetAsync(lam.p, 0, 3 * n3 * sizeof(R), st), "memset");
                k_pm_deposit<R, 3><<<pgrid(), PM_NT, 0, st>>>(xn, np, N, lq.p, 0.0, lam.p);
                k_pm_adj_div<R><<<fgrid(), PM_NT, 0, st>>>(lam.p, N, kq, rho.p);
                poisson(rho.p, pc);
                k_pm_adj_deposit<R><<<pgrid(), PM_NT, 0, st>>>(xn, np, N, rho.p, mass * (double)n3, lx.p);
            }
        }
        pck(cudaMemcpyAsync(gx0, lx.p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "copy gx");
        pck(cudaMemcpyAsync(gq0, lq.p, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, st), "copy gq");
        pck(cudaGetLastError(), "adjoint launch");
        pck(cudaStreamSynchronize(st), "adjoint");
        check_device("adjoint");
    }
};

}  // namespace
}  // namespace gev

struct gev_pm {
    std::unique_ptr<gev::PmBase> impl;
    std::string err;
};

namespace {
thread_local std::string g_pm_create_error;

template <class F> int pm_guarded(gev_pm *h, F &&f)
{
    if (!h || !h->impl) return GEV_ERR_ARG;
    try {
        f(*h->impl);
        return GEV_OK;
    } catch (const gev::PmError &e) {
        h->err = e.what();
        return e.code;
    } catch (const std::exception &e) {
        h->err = e.what();
        return GEV_ERR_CUDA;
    }
}
}  // namespace

extern "C" {

int gev_pm_create(const gev_pm_config *cfg, gev_pm **out)
{
    if (!cfg || !out) return GEV_ERR_ARG;
    *out = nullptr;
    const int N = cfg->N;
    const bool okN = N == 16 || N == 32 || N == 64 || N == 128 || N == 256 || N == 384 || N == 512 || N == 768;
    if (!okN || (cfg->precision != GEV_FP64 && cfg->precision != GEV_MIXED) || cfg->np <= 0 ||
        cfg->checkpoint_every <= 0) {
        g_pm_create_error = "invalid configuration (N one of 16..768, np > 0, checkpoint_every > 0)";
        return GEV_ERR_ARG;
    }
    auto *h = new gev_pm;
    try {
        if (cfg->precision == GEV_FP64) h->impl.reset(new gev::Pm<double>(*cfg));
        else h->impl.reset(new gev::Pm<float>(*cfg));
    } catch (const gev::PmError &e) {
        g_pm_create_error = e.what();
        delete h;
        return e.code;
    } catch (const std::exception &e) {
        g_pm_create_error = e.what();
        delete h;
        return GEV_ERR_CUDA;
    }
    *out = h;
    return GEV_OK;
}

int gev_pm_destroy(gev_pm *h)
{
    delete h;
    return GEV_OK;
}

const char *gev_pm_last_error(const gev_pm *h) { return h ? h->err.c_str() : g_pm_create_error.c_str(); }

int gev_pm_forward(gev_pm *h, int32_t nsteps, const double *coef, const double *x0, const double *q0, double *delta,
                   double *x_out, double *q_out)
{
    if (!coef || !x0 || !q0 || !delta || nsteps <= 0) return GEV_ERR_ARG;
    return pm_guarded(h, [&](gev::PmBase &p) { p.forward(nsteps, coef, x0, q0, delta, x_out, q_out); });
}

int gev_pm_adjoint(gev_pm *h, const double *ddelta, double *gx0, double *gq0)
{
    if (!ddelta || !gx0 || !gq0) return GEV_ERR_ARG;
    return pm_guarded(h, [&](gev::PmBase &p) { p.adjoint(ddelta, gx0, gq0); });
}

void *gev_pm_stream(gev_pm *h) { return (h && h->impl) ? (void *)h->impl->stream() : nullptr; }

}  // extern "C"
