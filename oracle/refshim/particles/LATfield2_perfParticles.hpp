// LATfield2_perfParticles.hpp -- single-rank CPU stand-in for LATfield2's
// perfParticles container (TEST INFRASTRUCTURE ONLY, see ../LATfield2.hpp).
//
// A particle sits in the cell floor(pos/dx) and the functors receive
// ref_dist = pos/dx - cell, as the reference's CPU projections compute it
// (gevolution.hpp:1339, :1358).  updateVel returns the square root of the largest
// functor return value (ic_basic.hpp:2433 divides it by a to obtain a velocity
// from a functor that returns q^2); moveParticles wraps positions into [0,1).
//
// Threads (OpenMP): updateVel and moveParticles touch one particle per functor
// call and run over particles in parallel.  A projection functor adds into the
// cells of its particle's stencil, which never reaches beyond one cell on
// either side along z (gevolution.hpp:1729-1854, :2031-2201, :2582-2965), so
// projections run by z-planes of cells in four rounds (cz mod 4): planes of one
// round are at least 4 apart and their particles write disjoint field planes.
// Within a plane particles keep their order.
#ifndef GEV_REFSHIM_PERFPARTICLES_HPP
#define GEV_REFSHIM_PERFPARTICLES_HPP

#include <cmath>
#include <cstdint>
#include <vector>
#include <omp.h>

struct part_simple
{
	Real pos[3];
	Real vel[3];
	long ID;
};

struct part_simple_info
{
	double mass;
	int relativistic;
	char type_name[64];
};

struct part_simple_dataType {};

namespace LATfield2
{

// LATfield2's general particle handler: the reference's non-CDM species use
// it; the runs here have none, so it only has to compile
template <typename part, typename part_info, typename part_dataType>
class Particles
{
public:
	struct CellList { std::vector<part> parts; };
	struct CellField { CellList cell; CellList & operator()(const Site &) { return cell; } };
	const Lattice & lattice() const { return *lat_; }
	CellField & field() { return field_; }
	template <class... A> void initialize(A &&...) { std::abort(); }
	template <class... A> void addParticle_global(A &&...) { std::abort(); }
	template <class... A> void moveParticles(A &&...) { std::abort(); }
	template <class... A> Real updateVel(A &&...) { std::abort(); }
private:
	const Lattice * lat_ = nullptr;
	CellField field_;
};

template <typename part, typename part_info, typename part_dataType>
void scalarProjectionCIC_project(Particles<part, part_info, part_dataType> *, Field<Real> *) { std::abort(); }

template <typename part, typename part_info>
class perfParticles
{
public:
	perfParticles() : lat_(nullptr) {}
	void attach(const Lattice * lat, part * parts, long count, const part_info & info)
	{
		lat_ = lat; parts_ = parts; count_ = count; info_ = info;
	}
	long num_particles() const { return count_; }
	const Lattice & lattice() const { return *lat_; }

	// particle handler of its own (the initial-condition generator's use):
	// initialize, then addParticle_global for each particle
	void initialize(const part_info & info, const Lattice * lat, const Real * boxSize, long capacity, long extra)
	{
		(void) boxSize; (void) extra;
		lat_ = lat;
		info_ = info;
		owned_.clear();
		owned_.reserve(capacity > 0 ? (size_t) capacity : 0);
		parts_ = owned_.data();
		count_ = 0;
	}
	void addParticle_global(const part & p)
	{
		owned_.push_back(p);
		parts_ = owned_.data();
		count_ = (long) owned_.size();
	}
	void updateRowBuffers() {}
	const part * particles() const { return parts_; }

	template <class F>
	void projectParticles(F f, Field<Real> ** fields, int nfield, double * params)
	{
		for_each_particle(f, 0., fields, nfield, params);
	}
	template <class F>
	void projectParticles_Async(F f, Field<Real> ** fields, int nfield, double * params)
	{
		for_each_particle(f, 0., fields, nfield, params);
	}
	template <class F>
	Real updateVel(F f, double dtau, Field<Real> ** fields, int nfield, double * params = nullptr)
	{
		Real vmax = 0;
#pragma omp parallel for reduction(max : vmax) schedule(static)
		for (long p = 0; p < count_; p++)
		{
			double ref_dist[3];
			Site sites[4];
			locate(p, fields, nfield, ref_dist, sites);
			Real v = f(dtau, 1.0 / lat_->N(), parts_ + p, ref_dist, info_, fields, sites, nfield, params, nullptr, 0);
			if (v > vmax) vmax = v;
		}
		return std::sqrt(vmax);
	}
	template <class F>
	void moveParticles(F f, double dtau, Field<Real> ** fields, int nfield, double * params)
	{
#pragma omp parallel for schedule(static)
		for (long p = 0; p < count_; p++)
		{
			double ref_dist[3];
			Site sites[4];
			locate(p, fields, nfield, ref_dist, sites);
			f(dtau, 1.0 / lat_->N(), parts_ + p, ref_dist, info_, fields, sites, nfield, params, nullptr, 0);
			for (int i = 0; i < 3; i++) parts_[p].pos[i] -= std::floor(parts_[p].pos[i]);
		}
	}
	// moveParticles with the functor's outputs reduced over the particles
	// (MAX or SUM per output, as LATfield2's reductionOp)
	template <class F>
	void moveParticles(F f, double dtau, Field<Real> ** fields, int nfield, double * params, double * outputs, int * ops, int noutputs)
	{
		std::vector<double> red(noutputs > 0 ? noutputs : 1, 0.0);
		for (long p = 0; p < count_; p++)
		{
			double ref_dist[3];
			double out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
			Site sites[4];
			locate(p, fields, nfield, ref_dist, sites);
			f(dtau, 1.0 / lat_->N(), parts_ + p, ref_dist, info_, fields, sites, nfield, params, out, noutputs);
			for (int i = 0; i < 3; i++) parts_[p].pos[i] -= std::floor(parts_[p].pos[i]);
			for (int o = 0; o < noutputs && o < 8; o++)
				red[o] = (ops && ops[o] == MAX) ? (out[o] > red[o] ? out[o] : red[o]) : red[o] + out[o];
		}
		for (int o = 0; o < noutputs; o++) outputs[o] = red[o];
	}
	void meshprojection_project(Field<Real> * field)
	{
		const double dx = 1.0 / lat_->N();
		const double mass = info_.mass / (dx * dx * dx);
		by_z_planes([&](long p)
		{
			double d[3];
			Site sites[4];
			locate(p, &field, 1, d, sites);
			for (int k = 0; k < 8; k++)
			{
				Site s = sites[0];
				if (k & 4) s = s + 0;
				if (k & 2) s = s + 1;
				if (k & 1) s = s + 2;
				(*field)(s) += mass * ((k & 4) ? d[0] : 1. - d[0]) * ((k & 2) ? d[1] : 1. - d[1]) * ((k & 1) ? d[2] : 1. - d[2]);
			}
		});
	}

private:
	void locate(long p, Field<Real> ** fields, int nfield, double * ref_dist, Site * sites)
	{
		const int N = lat_->N();
		int c[3];
		for (int i = 0; i < 3; i++)
		{
			double s = (double) parts_[p].pos[i] * N;
			double fl = std::floor(s);
			ref_dist[i] = s - fl;
			c[i] = ((int) fl % N + N) % N;
		}
		for (int i = 0; i < nfield && i < 4; i++)
			sites[i] = Site(fields[i] ? fields[i]->lattice() : *lat_, c[0], c[1], c[2]);
	}
	// body(p) for every particle, by z-planes of cells in four rounds (see the top)
	template <class B>
	void by_z_planes(B && body)
	{
		const int N = lat_->N();
		std::vector<long> start(N + 1, 0), order(count_);
		std::vector<int> cz(count_);
		for (long p = 0; p < count_; p++)
		{
			cz[p] = ((int) std::floor((double) parts_[p].pos[2] * N) % N + N) % N;
			start[cz[p] + 1]++;
		}
		for (int z = 0; z < N; z++) start[z + 1] += start[z];
		std::vector<long> fill(start.begin(), start.end() - 1);
		for (long p = 0; p < count_; p++) order[fill[cz[p]]++] = p;
		if (N % 4 != 0)   // the rounds need N a multiple of 4 (planes N-4+r and r are 4 apart)
		{
			for (long i = 0; i < count_; i++) body(order[i]);
			return;
		}
		for (int round = 0; round < 4; round++)
		{
#pragma omp parallel for schedule(dynamic, 1)
			for (int z = round; z < N; z += 4)
				for (long i = start[z]; i < start[z + 1]; i++) body(order[i]);
		}
	}
	template <class F>
	void for_each_particle(F f, double dtau, Field<Real> ** fields, int nfield, double * params)
	{
		by_z_planes([&](long p)
		{
			double ref_dist[3];
			Site sites[4];
			locate(p, fields, nfield, ref_dist, sites);
			f(dtau, 1.0 / lat_->N(), parts_ + p, ref_dist, info_, fields, sites, nfield, params, nullptr, 0);
		});
	}
	const Lattice * lat_;
	std::vector<part> owned_;
	part * parts_ = nullptr;
	long count_ = 0;
	part_info info_{};

public:
	// The GPU particle layout that Particles_gevolution.hpp's output kernels
	// read (count_tracer_particles, buffer_tracer_particles,
	// bufferTracerParticle): per row buffer the positions p (box units,
	// xyz-interleaved), momenta q and IDs (`other`); with the lattice size,
	// the rank's coordinate skip (zero on one rank) and the box size (1: box
	// units).  Filled by the caller, in memory the device can read.
	struct RowBuffer
	{
		int count;
		Real * p;
		Real * q;
		long * other;
	};
	// the particle arrays saveExpress / loadExpress copy from and to (device
	// memory in LATfield2: managed memory here), their count and capacity
	Real * p = nullptr;
	Real * q = nullptr;
	long * other = nullptr;
	long num_particles_ = 0;
	uint64_t extra_capacity_ = 0;
	void resizeGlobalBuffers(uint64_t) { std::abort(); }
	RowBuffer * row_buffers_ = nullptr;
	int num_row_buffers_ = 0;
	int lat_size_[3] = {0, 0, 0};
	int lat_size_local_[3] = {0, 0, 0};
	int coordSkip_[2] = {0, 0};
	Real boxSize_[3] = {1, 1, 1};
	uint64_t total_capacity_ = 0;
};

} // namespace LATfield2

#endif
