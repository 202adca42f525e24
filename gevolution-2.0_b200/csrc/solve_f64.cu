// solve_f64.cu -- FP64 instantiation of the pencil passes.
#include "solve_impl.cuh"

namespace gev {
GEV_SOLVE_INST(double)
}  // namespace gev
