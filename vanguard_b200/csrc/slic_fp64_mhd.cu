// Exact-FP64 kernels of the MHD models: single-material (reduced and full variants, with the GLM forcing that the
// mixed form also calls) and the reduced, intermediate and multiphysics two-material models.  Compiled with
// -fmad=false.
#include "slic_fp64.cuh"

namespace vg {

Ops fp64_ops_mhd7() { return fp64::make_ops<MHDF64<false>>(); }
Ops fp64_ops_mhd9() { return fp64::make_ops<MHDF64<true>>(); }
Ops fp64_ops_mred11() { return fp64::make_ops<MHDReducedF64>(); }
Ops fp64_ops_mint12() { return fp64::make_ops<MHDIntermediateF64>(); }
Ops fp64_ops_mmph16() { return fp64::make_ops<MHDMultiphysicsF64>(); }

cudaError_t mhd_reduced_reinit_fp64(const SweepArgs& a, cudaStream_t st) {
    return reduced_reinit<ReinitMHDReduced>(a, st);
}
cudaError_t mhd_intermediate_reinit_fp64(const SweepArgs& a, cudaStream_t st) {
    return reduced_reinit<ReinitMHDIntermediate>(a, st);
}
cudaError_t mhd7_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st) {
    return fp64::forcing_impl<MHDF64<false>>(a, subcycles, st);
}
cudaError_t mhd9_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st) {
    return fp64::forcing_impl<MHDF64<true>>(a, subcycles, st);
}

}  // namespace vg
