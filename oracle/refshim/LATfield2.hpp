// LATfield2.hpp -- minimal single-rank, single-process stand-in for the parts of
// LATfield2 ("v1.1 with GPU support", not vendored with gevolution-2.0) that
// gevolution.hpp, background.hpp and tools.hpp name.
//
// TEST INFRASTRUCTURE ONLY.  It exists so that the reference's own host-side
// arithmetic (the __host__ __device__ particle functors, the prepareFTsource
// functors, the OpenMP Fourier-space solvers, the background integrator and the
// spectrum binning) can be compiled from the reference sources where they lie and
// run on the CPU, as an independent pin for the oracle restatement.  Semantics
// follow the reference's call sites on one rank:
//   * a real-space Site is a lattice point (x,y,z); "site + i" / "site - i" is the
//     periodic neighbour along axis i (the halo of a one-rank lattice is the
//     periodic image, so no fold or halo fill is needed);
//   * an rKSite carries the wavenumber indices (kx in [0,N/2], ky, kz in [0,N));
//   * Field<T> wraps caller-owned memory with one plane per component
//     (index x + N*(y + N*z), or kx + (N/2+1)*(ky + N*kz) for Fourier fields);
//     symmetric 3x3 tensors use the component order 00,01,02,11,12,22.
#ifndef GEV_REFSHIM_LATFIELD2_HPP
#define GEV_REFSHIM_LATFIELD2_HPP

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>
#include <stdexcept>
#include <cuda_runtime.h>

#ifndef LATFIELD2_REAL
#define LATFIELD2_REAL double
#endif

typedef LATFIELD2_REAL Real;

#define COLORTEXT_WHITE ""
#define COLORTEXT_CYAN ""
#define COLORTEXT_GREEN ""
#define COLORTEXT_RED ""
#define COLORTEXT_YELLOW ""
#define COLORTEXT_RESET ""
#define COUT std::cout


// ---- single-process MPI stand-ins used by tools.hpp's spectrum reduction ----
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_IN_PLACE ((void *)1)
#define MPI_FLOAT 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_SUM 0
#define MPI_MAX 1
inline int MPI_Reduce(const void *, void *, int, MPI_Datatype, MPI_Op, int, MPI_Comm) { return 0; }

// ---- MPI file and point-to-point names that Particles_gevolution.hpp's output
// routines use: declared so that the header compiles for its lightcone
// selection kernels; the single-process stand-in writes no files, so calling
// any of them aborts ----
typedef int MPI_Request;
typedef int MPI_File;
typedef int MPI_Info;
typedef long long MPI_Offset;
struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };
#define MPI_BYTE 4
#define MPI_UNSIGNED 5
#define MPI_UNSIGNED_LONG_LONG 6
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_RDONLY 2
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
inline int MPI_File_open(MPI_Comm, const char *, int, MPI_Info, MPI_File *) { std::abort(); }
inline int MPI_File_close(MPI_File *) { std::abort(); }
inline int MPI_File_set_size(MPI_File, MPI_Offset) { std::abort(); }
inline int MPI_File_write_at(MPI_File, MPI_Offset, const void *, int, MPI_Datatype, MPI_Status *) { std::abort(); }
inline int MPI_File_write_at_all(MPI_File, MPI_Offset, const void *, int, MPI_Datatype, MPI_Status *) { std::abort(); }
inline int MPI_File_read_at(MPI_File, MPI_Offset, void *, int, MPI_Datatype, MPI_Status *) { std::abort(); }
inline int MPI_File_read_at_all(MPI_File, MPI_Offset, void *, int, MPI_Datatype, MPI_Status *) { std::abort(); }
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { std::abort(); }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { std::abort(); }
inline int MPI_Wait(MPI_Request *, MPI_Status *) { std::abort(); }
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { std::abort(); }
inline int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) { std::abort(); }
#define MPI_SUCCESS 0
#define MPI_SEEK_SET 0
#define MPI_LONG_LONG 7
#define MPI_FILE_NULL (-1)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
inline int MPI_File_seek(MPI_File, MPI_Offset, int) { std::abort(); }
inline int MPI_File_read_all(MPI_File, void *, int, MPI_Datatype, MPI_Status *) { std::abort(); }
inline int MPI_Barrier(MPI_Comm) { std::abort(); }
inline int MPI_Alltoall(const void *, int, MPI_Datatype, void *, int, MPI_Datatype, MPI_Comm) { std::abort(); }

namespace LATfield2
{

enum matrixSymmetry { unsymmetric = 0, symmetric = 1 };

// reduction selectors passed to lattice_for_each / moveParticles
enum reductionOp { SUM = 0, MAX = 1, MIN = 2 };

class Imag
{
public:
	__host__ __device__ Imag() : re_(0), im_(0) {}
	__host__ __device__ Imag(Real re, Real im) : re_(re), im_(im) {}
	__host__ __device__ Real real() const { return re_; }
	__host__ __device__ Real imag() const { return im_; }
	__host__ __device__ Real & real() { return re_; }
	__host__ __device__ Real & imag() { return im_; }
	__host__ __device__ Imag conj() const { return Imag(re_, -im_); }
	__host__ __device__ Imag operator-() const { return Imag(-re_, -im_); }
	__host__ __device__ Imag operator+(const Imag & o) const { return Imag(re_ + o.re_, im_ + o.im_); }
	__host__ __device__ Imag operator-(const Imag & o) const { return Imag(re_ - o.re_, im_ - o.im_); }
	__host__ __device__ Imag operator*(const Imag & o) const { return Imag(re_ * o.re_ - im_ * o.im_, re_ * o.im_ + im_ * o.re_); }
	__host__ __device__ Imag operator*(Real s) const { return Imag(re_ * s, im_ * s); }
	__host__ __device__ Imag operator/(Real s) const { return Imag(re_ / s, im_ / s); }
	__host__ __device__ Imag operator/(const Imag & o) const
	{
		const Real den = o.re_ * o.re_ + o.im_ * o.im_;
		return Imag((re_ * o.re_ + im_ * o.im_) / den, (im_ * o.re_ - re_ * o.im_) / den);
	}
	__host__ __device__ Imag & operator+=(const Imag & o) { re_ += o.re_; im_ += o.im_; return *this; }
	__host__ __device__ Imag & operator-=(const Imag & o) { re_ -= o.re_; im_ -= o.im_; return *this; }
	__host__ __device__ Imag & operator*=(Real s) { re_ *= s; im_ *= s; return *this; }
	__host__ __device__ Imag & operator/=(Real s) { re_ /= s; im_ /= s; return *this; }
private:
	Real re_, im_;
};

__host__ __device__ inline Imag operator*(Real s, const Imag & z) { return z * s; }

class Lattice
{
public:
	__host__ __device__ Lattice() : N_(0), fourier_(false) {}
	__host__ __device__ Lattice(int N, bool fourier) : N_(N), fourier_(fourier) {}
	__host__ __device__ int size(int i) const { return (fourier_ && i == 0) ? N_ / 2 + 1 : N_; }
	__host__ __device__ int sizeLocal(int i) const { return size(i); }
	__host__ __device__ int halo() const { return 0; }
	__host__ __device__ const int * coordSkip() const { return skip_; }
	__host__ __device__ long sitesLocal() const { return (long) size(0) * size(1) * size(2); }
	__host__ __device__ long sitesLocalGross() const { return sitesLocal(); }
	__host__ __device__ int N() const { return N_; }
	__host__ __device__ bool fourier() const { return fourier_; }
	// linear site indexes without halo: the first site is 0, a step along
	// dimension i jumps by the product of the sizes below it
	__host__ __device__ long siteFirst() const { return 0; }
	__host__ __device__ long siteLast() const { return sitesLocal() - 1; }
	__host__ __device__ long jump(int i) const { return i == 0 ? 1 : (i == 1 ? (long) size(0) : (long) size(0) * size(1)); }
private:
	int N_;
	bool fourier_;
	int skip_[2] = {0, 0};
};

class Site
{
public:
	__host__ __device__ Site() : lat_(nullptr) { c_[0] = c_[1] = c_[2] = 0; }
	__host__ __device__ explicit Site(const Lattice & lat) : lat_(&lat) { c_[0] = c_[1] = c_[2] = 0; }
	__host__ __device__ Site(const Lattice & lat, int x, int y, int z) : lat_(&lat) { c_[0] = x; c_[1] = y; c_[2] = z; }
	// the site of linear index idx (Lattice::jump)
	__host__ __device__ Site(const Lattice & lat, long idx) : lat_(&lat)
	{
		const long n = lat.N();
		c_[0] = (int) (idx % n);
		c_[1] = (int) ((idx / n) % n);
		c_[2] = (int) (idx / (n * n));
	}
	__host__ __device__ void initialize(const Lattice & lat) { lat_ = &lat; first(); }
	__host__ __device__ bool setCoord(int x, int y, int z)
	{
		const int n = lat_->N();
		if (x < 0 || x >= n || y < 0 || y >= n || z < 0 || z >= n) return false;
		c_[0] = x; c_[1] = y; c_[2] = z;
		return true;
	}
	__host__ __device__ void first() { c_[0] = c_[1] = c_[2] = 0; }
	__host__ __device__ bool test() const { return c_[2] < lat_->N(); }
	__host__ __device__ void next()
	{
		if (++c_[0] == lat_->N()) { c_[0] = 0; if (++c_[1] == lat_->N()) { c_[1] = 0; ++c_[2]; } }
	}
	__host__ __device__ int coord(int i) const { return c_[i]; }
	__host__ __device__ long index() const { return (long) c_[0] + (long) lat_->N() * ((long) c_[1] + (long) lat_->N() * c_[2]); }
	__host__ __device__ Site operator+(int dir) const
	{
		Site s(*this);
		s.c_[dir] = (s.c_[dir] + 1) % lat_->N();
		return s;
	}
	__host__ __device__ Site operator-(int dir) const
	{
		Site s(*this);
		s.c_[dir] = (s.c_[dir] + lat_->N() - 1) % lat_->N();
		return s;
	}
	__host__ __device__ const Lattice & lattice() const { return *lat_; }
private:
	const Lattice * lat_;
	int c_[3];
};

class rKSite
{
public:
	__host__ __device__ explicit rKSite(const Lattice & lat) : lat_(&lat) { c_[0] = c_[1] = c_[2] = 0; }
	// the site of linear index idx (x fastest)
	__host__ __device__ void initialize(const Lattice & lat, long idx)
	{
		lat_ = &lat;
		c_[0] = (int) (idx % lat.size(0));
		c_[1] = (int) ((idx / lat.size(0)) % lat.size(1));
		c_[2] = (int) (idx / ((long) lat.size(0) * lat.size(1)));
	}
	__host__ __device__ bool setCoord(int x, int y, int z)
	{
		if (x < 0 || x >= lat_->size(0) || y < 0 || y >= lat_->size(1) || z < 0 || z >= lat_->size(2)) return false;
		c_[0] = x; c_[1] = y; c_[2] = z;
		return true;
	}
	__host__ __device__ void first() { c_[0] = c_[1] = c_[2] = 0; }
	__host__ __device__ bool test() const { return c_[2] < lat_->size(2); }
	__host__ __device__ void next()
	{
		if (++c_[0] == lat_->size(0)) { c_[0] = 0; if (++c_[1] == lat_->size(1)) { c_[1] = 0; ++c_[2]; } }
	}
	__host__ __device__ int coord(int i) const { return c_[i]; }
	__host__ __device__ long index() const { return (long) c_[0] + (long) lat_->size(0) * ((long) c_[1] + (long) lat_->size(1) * c_[2]); }
private:
	const Lattice * lat_;
	int c_[3];
};

template <class T>
class Field
{
public:
	__host__ __device__ Field() : lat_(nullptr), data_(nullptr), comp_(1), sym_(unsymmetric) {}
	__host__ __device__ Field(const Lattice & lat, T * data, int components, matrixSymmetry sym = unsymmetric)
		: lat_(&lat), data_(data), comp_(components), sym_(sym) {}
	__host__ __device__ const Lattice & lattice() const { return *lat_; }
	__host__ __device__ int components() const { return comp_; }
	__host__ __device__ matrixSymmetry symmetry() const { return sym_; }
	__host__ __device__ T * data() { return data_; }
	__host__ __device__ T & operator()(const Site & s) { return data_[s.index()]; }
	__host__ __device__ T & operator()(const Site & s, int c) { return data_[c * lat_->sitesLocal() + s.index()]; }
	__host__ __device__ T & operator()(const Site & s, int i, int j) { return data_[sym_index(i, j) * lat_->sitesLocal() + s.index()]; }
	__host__ __device__ T & operator()(const rKSite & k) { return data_[k.index()]; }
	__host__ __device__ T & operator()(const rKSite & k, int c) { return data_[c * lat_->sitesLocal() + k.index()]; }
	__host__ __device__ T & operator()(const rKSite & k, int i, int j) { return data_[sym_index(i, j) * lat_->sitesLocal() + k.index()]; }
	__host__ __device__ T & operator()(long idx) { return data_[idx]; }
	__host__ __device__ T & operator()(long idx, int c) { return data_[c * lat_->sitesLocal() + idx]; }
	__host__ __device__ T & operator()(long idx, int i, int j) { return data_[sym_index(i, j) * lat_->sitesLocal() + idx]; }
	void updateHalo() {}
private:
	__host__ __device__ static int sym_index(int i, int j)
	{
		if (i > j) { int t = i; i = j; j = t; }
		return (i == 0) ? j : (i == 1 ? 2 + j : 5);
	}
	const Lattice * lat_;
	T * data_;
	int comp_;
	matrixSymmetry sym_;
};

class Parallel
{
public:
	int rank() const { return 0; }
	int size() const { return 1; }
	bool isRoot() const { return true; }
	MPI_Comm lat_world_comm() const { return 0; }
	template <class T> void sum(T &) {}
	template <class T> void sum(T *, int) {}
	template <class T> void max(T &) {}
	template <class T> void max(T *, int) {}
	template <class T> void min(T &) {}
	template <class T> void broadcast(T &, int) {}
	template <class T> void broadcast(T *, int, int) {}
	// one rank: the neighbour in every direction is this rank itself
	template <class T> void sendUp_dim0(T * send, T * recv, long n) { std::memcpy(recv, send, sizeof(T) * n); }
	template <class T> void sendUp_dim1(T * send, T * recv, long n) { std::memcpy(recv, send, sizeof(T) * n); }
	template <class T> void sendUpDown_dim0(T * s1, T * r1, long n1, T * s2, T * r2, long n2) { std::memcpy(r1, s1, sizeof(T) * n1); std::memcpy(r2, s2, sizeof(T) * n2); }
	template <class T> void sendUpDown_dim1(T * s1, T * r1, long n1, T * s2, T * r2, long n2) { std::memcpy(r1, s1, sizeof(T) * n1); std::memcpy(r2, s2, sizeof(T) * n2); }
	void abortForce() { std::abort(); }
	// the process grid of one rank (1 x 1), and point-to-point transfers a
	// single process never makes
	const int * grid_rank() const { static const int r[2] = {0, 0}; return r; }
	const int * grid_size() const { static const int s[2] = {1, 1}; return s; }
	const MPI_Comm * dim0_comm() const { static const MPI_Comm c[1] = {0}; return c; }
	const MPI_Comm * dim1_comm() const { static const MPI_Comm c[1] = {0}; return c; }
	template <class T> void send(T &, int) { std::abort(); }
	template <class T> void receive(T &, int) { std::abort(); }
	template <class T> void send_dim0(T &, int) { std::abort(); }
	template <class T> void receive_dim0(T &, int) { std::abort(); }
	template <class T> void send_dim1(T &, int) { std::abort(); }
	template <class T> void receive_dim1(T &, int) { std::abort(); }
	template <class T> void broadcast_dim0(T &, int) {}
	template <class T> void broadcast_dim0(T *, int, int) {}
	template <class T> void broadcast_dim1(T &, int) {}
};

inline Parallel parallel;

// ---- PlanFFT: R2C / C2R over every component of a field pair.  The
// transforms themselves (the oracle's FFT by default) are supplied by the
// caller through gev_shim_r2c / gev_shim_c2r, with the conventions of the
// oracle's: unnormalised, half spectrum kx + (N/2+1)(ky + N kz) ----
#define FFT_FORWARD 0
#define FFT_BACKWARD 1
typedef void (*gev_shim_fft_fn)(int N, const double * in, double * out);
inline gev_shim_fft_fn gev_shim_r2c = nullptr;
inline gev_shim_fft_fn gev_shim_c2r = nullptr;

template <class C>
class PlanFFT
{
public:
	PlanFFT() {}
	PlanFFT(Field<Real> * r, Field<C> * k, int components = 1) : r_(r), k_(k), comp_(components) {}
	void initialize(Field<Real> * r, Field<C> * k, int components = 1) { r_ = r; k_ = k; comp_ = components; }
	void preallocate(size_t) {}
	void execute(int dir)
	{
		if (!r_ || !k_ || !gev_shim_r2c || !gev_shim_c2r) std::abort();
		const int N = r_->lattice().N();
		const long n3 = (long) N * N * N, nk = (long) (N / 2 + 1) * N * N;
		for (int c = 0; c < comp_; c++)
		{
			double * re = r_->data() + c * n3;
			double * ft = reinterpret_cast<double *>(k_->data() + c * nk);
			if (dir == FFT_FORWARD) gev_shim_r2c(N, re, ft);
			else gev_shim_c2r(N, ft, re);
		}
	}
private:
	Field<Real> * r_ = nullptr;
	Field<C> * k_ = nullptr;
	int comp_ = 1;
};

// scalarProjectionCIC_comm, projection_T0i_comm, projection_Tij_comm: the
// stand-in's projections wrap periodically, there is no halo to fold
inline void scalarProjectionCIC_comm(Field<Real> *) {}

struct TempMemory
{
	void reserveDeviceWorkspaceBytes(size_t, const char *) {}
	void * deviceWorkspace() { return nullptr; }
	size_t deviceWorkspaceBytes() { return 0; }
};

inline TempMemory tempMemory;

} // namespace LATfield2

using LATfield2::parallel;

#include "particles/LATfield2_perfParticles.hpp"

#endif
