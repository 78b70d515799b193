// Mixed FP32/FP64 SLIC kernels (VG_MIXED).  Compiled with FMA contraction on.
#include "physics_mixed.cuh"
#include "slic_kernels.cuh"
#include "slic_mixed.cuh"
#include "vg_ops.h"

namespace vg {
namespace {

constexpr int XP = 128;
constexpr int XL = 1;
constexpr int YTX = 64;
constexpr int YTY = 64;
constexpr int MW_NT = 256;

template <class M>
cudaError_t sweep_impl(int axis, const SweepArgs& a, cudaStream_t st) {
    if (axis == 0) {
        dim3 grid((a.nx + XP - 3) / (XP - 2), (a.ny + XL - 1) / XL);
        sweep_x_mixed_kernel<M, XP, XL><<<grid, XP * XL, 0, st>>>(a);
    } else {
        dim3 grid((a.nx + YTX - 1) / YTX, (a.ny + YTY - 1) / YTY);
        sweep_y_mixed_kernel<M, YTX, YTY><<<grid, YTX, 0, st>>>(a);
    }
    return cudaGetLastError();
}

template <>
cudaError_t sweep_impl<EulerMixed<1>>(int axis, const SweepArgs& a, cudaStream_t st) {
    if (axis != 0) return cudaErrorInvalidValue;
    dim3 grid((a.nx + XP - 3) / (XP - 2), (a.ny + XL - 1) / XL);
    sweep_x_mixed_kernel<EulerMixed<1>, XP, XL><<<grid, XP * XL, 0, st>>>(a);
    return cudaGetLastError();
}

template <class M>
cudaError_t max_wave_impl(const SweepArgs& a, cudaStream_t st) {
    long n = (long)a.nx * a.ny;
    int blocks = (int)((n + MW_NT - 1) / MW_NT);
    if (blocks > 148 * 8) blocks = 148 * 8;
    max_wave_kernel<M, MW_NT><<<blocks, MW_NT, 0, st>>>(a.in, a.plane, a.pitch, a.nx, a.ny, a.ctrl, a);
    return cudaGetLastError();
}

template <class M>
cudaError_t step_begin_impl(const SweepArgs& a, cudaStream_t st) {
    step_begin_kernel<M><<<1, 32, 0, st>>>(a.ctrl, a);
    return cudaGetLastError();
}

template <class M>
cudaError_t finish_impl(const SweepArgs& a, double* out, cudaStream_t st) {
    max_wave_finish_kernel<M><<<1, 32, 0, st>>>(a.ctrl, a, out);
    return cudaGetLastError();
}

template <class M>
constexpr Ops make_ops() {
    return Ops{M::NW, &sweep_impl<M>, &max_wave_impl<M>, &step_begin_impl<M>, &finish_impl<M>};
}

const Ops kOps[V_COUNT] = {
    make_ops<EulerMixed<1>>(),
    make_ops<EulerMixed<2>>(),
    make_ops<MHDMixed<false>>(),
    make_ops<MHDMixed<true>>(),
};

}  // namespace

const Ops* ops_mixed(int variant) { return (variant >= 0 && variant < V_COUNT) ? &kOps[variant] : nullptr; }

}  // namespace vg
