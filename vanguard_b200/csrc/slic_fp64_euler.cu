// Exact-FP64 kernels of the Euler models: single-material 1D and 2D, and the reduced and multiphysics two-material
// models with their volume-fraction reinitialisation.  Compiled with -fmad=false.
#include "slic_fp64.cuh"

namespace vg {

Ops fp64_ops_euler1() { return fp64::make_ops<EulerF64<1>>(); }
Ops fp64_ops_euler2() { return fp64::make_ops<EulerF64<2>>(); }
Ops fp64_ops_red6() { return fp64::make_ops<EulerReducedF64>(); }
Ops fp64_ops_mph7() { return fp64::make_ops<EulerMultiphysicsF64>(); }

cudaError_t reduced_reinit_fp64(const SweepArgs& a, cudaStream_t st) {
    return reduced_reinit<ReinitEulerReduced>(a, st);
}
cudaError_t multiphysics_reinit_fp64(const SweepArgs& a, cudaStream_t st) {
    return reduced_reinit<ReinitEulerMultiphysics>(a, st);
}

}  // namespace vg
