// Exact-FP64 kernels of the Euler models: single-material 1D and 2D, and the reduced and multiphysics two-material
// models with their volume-fraction reinitialisation.  Compiled with -fmad=false.
#include "slic_fp64.cuh"
#include "solve1d_kernels.cuh"

namespace vg {

namespace {
template <class M>
cudaError_t solve1d_impl(const SweepArgs& a, cudaStream_t st) {
    const size_t bytes = (size_t)solve1d_smem_doubles<M>(solve1d_seg(a.nx)) * sizeof(double);
    if (a.nx < solve1d_min_cells() || a.nx > solve1d_max_cells() || a.in != a.out || bytes > 48 * 1024)
        return cudaErrorInvalidValue;
    solve1d_kernel<M><<<S1D_CL, S1D_NT, bytes, st>>>(a);
    return cudaGetLastError();
}
}  // namespace

Ops fp64_ops_euler1() {
    Ops o = fp64::make_ops<EulerF64<1>>();
    o.solve1d = &solve1d_impl<EulerF64<1>>;
    o.solve1d_min = solve1d_min_cells();
    o.solve1d_max = solve1d_max_cells();
    return o;
}
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
