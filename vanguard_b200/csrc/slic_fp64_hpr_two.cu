// Exact-FP64 kernels of the HPR reduced, intermediate and multiphysics two-material models with their volume-fraction
// reinitialisation.  Compiled with -fmad=false.
#include "slic_fp64.cuh"

namespace vg {

Ops fp64_ops_hred19() { return fp64::make_ops<HPRReducedF64>(); }
Ops fp64_ops_hint20() { return fp64::make_ops<HPRIntermediateF64>(); }
Ops fp64_ops_hmph32() { return fp64::make_ops<HPRMultiphysicsF64>(); }

cudaError_t hpr_reduced_reinit_fp64(const SweepArgs& a, cudaStream_t st) {
    return reduced_reinit<ReinitHPRReduced>(a, st);
}
cudaError_t hpr_intermediate_reinit_fp64(const SweepArgs& a, cudaStream_t st) {
    return reduced_reinit<ReinitHPRIntermediate>(a, st);
}
cudaError_t hpr_multiphysics_reinit_fp64(const SweepArgs& a, cudaStream_t st) {
    return reduced_reinit<ReinitHPRMultiphysics>(a, st);
}

}  // namespace vg
