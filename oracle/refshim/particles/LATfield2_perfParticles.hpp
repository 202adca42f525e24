// LATfield2_perfParticles.hpp -- single-rank CPU stand-in for LATfield2's
// perfParticles container (TEST INFRASTRUCTURE ONLY, see ../LATfield2.hpp).
//
// A particle sits in the cell floor(pos/dx) and the functors receive
// ref_dist = pos/dx - cell, as the reference's CPU projections compute it
// (gevolution.hpp:1339, :1358).  updateVel returns the square root of the largest
// functor return value (ic_basic.hpp:2433 divides it by a to obtain a velocity
// from a functor that returns q^2); moveParticles wraps positions into [0,1).
#ifndef GEV_REFSHIM_PERFPARTICLES_HPP
#define GEV_REFSHIM_PERFPARTICLES_HPP

#include <cmath>
#include <vector>

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

template <typename part, typename part_info, typename part_dataType>
class Particles;

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
	Real updateVel(F f, double dtau, Field<Real> ** fields, int nfield, double * params)
	{
		Real vmax = 0;
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
		for_each_particle(f, dtau, fields, nfield, params);
		for (long p = 0; p < count_; p++)
			for (int i = 0; i < 3; i++) parts_[p].pos[i] -= std::floor(parts_[p].pos[i]);
	}
	void meshprojection_project(Field<Real> * field)
	{
		const double dx = 1.0 / lat_->N();
		const double mass = info_.mass / (dx * dx * dx);
		for (long p = 0; p < count_; p++)
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
		}
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
	template <class F>
	void for_each_particle(F f, double dtau, Field<Real> ** fields, int nfield, double * params)
	{
		for (long p = 0; p < count_; p++)
		{
			double ref_dist[3];
			Site sites[4];
			locate(p, fields, nfield, ref_dist, sites);
			f(dtau, 1.0 / lat_->N(), parts_ + p, ref_dist, info_, fields, sites, nfield, params, nullptr, 0);
		}
	}
	const Lattice * lat_;
	part * parts_ = nullptr;
	long count_ = 0;
	part_info info_{};
};

} // namespace LATfield2

#endif
