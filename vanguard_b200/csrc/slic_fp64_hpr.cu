// Exact-FP64 kernels of the single-material HPR gas, with the RK4 forcing and the stiff relaxation that the mixed form
// also calls.  Compiled with -fmad=false.
#include "slic_fp64.cuh"

namespace vg {

Ops fp64_ops_hpr17() { return fp64::make_ops<HPRF64>(); }

cudaError_t hpr_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st) {
    return fp64::forcing_impl<HPRF64>(a, subcycles, st);
}
cudaError_t hpr_relax_fp64(const SweepArgs& a, cudaStream_t st) { return fp64::relax_impl<HPRF64>(a, st); }

}  // namespace vg
