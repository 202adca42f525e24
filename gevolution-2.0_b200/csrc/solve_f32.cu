// solve_f32.cu -- FP32 (mixed-precision) instantiation of the pencil passes.
#include "solve_impl.cuh"

namespace gev {
GEV_SOLVE_INST(float)
int fx_rows_per_block(int N, bool fp64) { (void)N; return fp64 ? PassCfg<double>::TX : PassCfg<float>::TX; }
}  // namespace gev
