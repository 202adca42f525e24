// lattice_loop.hpp -- stand-in for LATfield2's lattice_for_each kernel
// (TEST INFRASTRUCTURE ONLY).  The reference launches it as
// lattice_for_each<<<dim3(N, N), 128>>>(functor, N, fields, nfield, params,
// outputs, reduce); this stand-in keeps that signature so the reference sources
// compile.  The CPU pin in ref_entry.cu calls the functors site by site instead.
#ifndef GEV_REFSHIM_LATTICE_LOOP_HPP
#define GEV_REFSHIM_LATTICE_LOOP_HPP

template <class F, int NRED = 0>
__global__ void lattice_for_each(F f, int numpts, LATfield2::Field<Real> ** fields, int nfields, double * params, double * outputs, int * reduce)
{
	LATfield2::Site sites[4];
	for (int x = threadIdx.x; x < numpts; x += blockDim.x)
	{
		for (int i = 0; i < nfields && i < 4; i++)
			sites[i] = LATfield2::Site(fields[i]->lattice(), x, blockIdx.x, blockIdx.y);
		double out[NRED > 0 ? NRED : 1];
		f(fields, sites, nfields, params, out);
	}
}

#endif
