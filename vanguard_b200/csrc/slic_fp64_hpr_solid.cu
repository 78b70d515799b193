// Exact-FP64 kernels of the single-material HPR model with every equation-of-state branch and the plastic relaxation
// (the solids), with the forcing and relaxation the mixed form also calls.  Compiled with -fmad=false.
#include "slic_fp64.cuh"

namespace vg {

Ops fp64_ops_hpr17s() { return fp64::make_ops<HPRSolidF64>(); }

cudaError_t hpr_solid_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st) {
    return fp64::forcing_impl<HPRSolidF64>(a, subcycles, st);
}
cudaError_t hpr_solid_relax_fp64(const SweepArgs& a, cudaStream_t st) { return fp64::relax_impl<HPRSolidF64>(a, st); }

}  // namespace vg
