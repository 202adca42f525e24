// lightcone.cu -- particle lightcone crossing for one shell and one cycle.
//
// One CTA per tile of particles: the tile first culls the periodic images of
// the vertex whose shell cannot reach it, then every particle takes the shell
// and cone test of count_tracer_particles / buffer_tracer_particles
// (Particles_gevolution.hpp:1271-1345, :1381-1466) against the kept images,
// the ID-backlog de-duplication of the check zone
// (count_lightcone_duplicate_ids / mark_lightcone_kept_particles, :1468-1510),
// the interpolation to the crossing time (bufferTracerParticle with
// EXACT_OUTPUT_REDSHIFTS, :500-560) and the logging of IDs near the inner edge
// for the next cycle.
//
// The ID logs are open-addressing hash sets in device memory (keys are particle
// IDs, EMPTY marks a free slot): membership is a set property, so the result
// does not depend on insertion order, and no host sort of the log is needed
// (the reference sorts its backlog, lightcone_id_backlog.hpp:58-70, for binary
// search).  Output slots come from one atomic counter; the output order is not
// significant (the reference's is not either).
#include "lightcone.cuh"

namespace gev {

constexpr int LC_NT = 256;

// One CTA per tile of 8^3 cells (particles are in bucket order).  The CTA
// first keeps the vertex images whose shell [inner, outer) can reach the
// tile's bounding box and exits when none does; each particle then takes the
// FP32 pre-test and, near the shell, the reference's exact FP64 test.
template <class R>
__global__ void __launch_bounds__(LC_NT, 4) k_lightcone(PView<R> p, const uint32_t *__restrict__ bstart, int N, int nt,
                                                     const R *__restrict__ phi, const __grid_constant__ LcKernelArgs la,
                                                     float *opos,
                                                     float *ovel, int64_t *oid, unsigned long long *count,
                                                     unsigned long long *newlog, int64_t newlog_cap, int *err,
                                                     FastDiv fN)
{
    __shared__ int vlist[64];
    __shared__ unsigned int vmask[2];
    const int tile = blockIdx.x;
    const int tx = tile % nt, ty = (tile / nt) % nt, tz = tile / (nt * nt);
    lc_cull_images(la, N, tx, ty, tz, vmask);
    __syncthreads();
    const int nkeep = lc_compact_images(vmask, vlist);
    if (nkeep == 0) return;
    __syncthreads();

    const LcShell sh(la, N);
    const uint32_t plo = bstart[8 * tile], phi_ = bstart[8 * tile + 8];
    for (uint32_t ii = plo + threadIdx.x; ii < phi_; ii += LC_NT) {
        const int64_t i = ii;
        const uint32_t cell = p.cell[i];
        if ((int64_t)cell >= (int64_t)N * N * N) { atomicOr(err, ERR_BAD_CELL); continue; }
        int c[3];
        decode_cell(cell, fN, c[0], c[1], c[2]);
        const double fr[3] = {p.off[i], p.off[p.cap + i], p.off[2 * p.cap + i]};
        lc_visit(p, i, N, c, fr, phi, la, sh, vlist, nkeep, opos, ovel, oid, count, newlog, newlog_cap, err);
    }
}


template <class R>
void launch_lightcone(const PView<R> &p, const uint32_t *bstart, int N, const R *phi, const LcKernelArgs &la, float *pos, float *vel,
                      int64_t *ids, unsigned long long *count, unsigned long long *newlog, int64_t newlog_cap, int *err,
                      cudaStream_t st)
{
    if (p.n > 0)
        k_lightcone<R><<<(unsigned)((N / 8) * (N / 8) * (N / 8)), LC_NT, 0, st>>>(
            p, bstart, N, N / 8, phi, la, pos, vel, ids, count, newlog, newlog_cap, err, FastDiv((uint32_t)N));
}

template void launch_lightcone<float>(const PView<float> &, const uint32_t *, int, const float *, const LcKernelArgs &, float *, float *,
                                      int64_t *, unsigned long long *, unsigned long long *, int64_t, int *, cudaStream_t);
template void launch_lightcone<double>(const PView<double> &, const uint32_t *, int, const double *, const LcKernelArgs &, float *,
                                       float *, int64_t *, unsigned long long *, unsigned long long *, int64_t, int *,
                                       cudaStream_t);

}  // namespace gev
