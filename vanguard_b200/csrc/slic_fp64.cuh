// The exact-FP64 kernel launchers and the Ops table entry of one model, shared by the slic_fp64_*.cu units.  Each
// unit instantiates a few models, so ptxas runs on the units in parallel.  Every unit including this header MUST be
// compiled with -fmad=false: the reference's x86-64 build forms no fused multiply-adds, and bitwise parity depends on
// every product being rounded before it is added.
#pragma once

#include "first_order_kernels.cuh"
#include "forcing_kernels.cuh"
#include "relax_kernels.cuh"
#include "physics_fp64.cuh"
#include "physics_hpr.cuh"
#include "slic_kernels.cuh"
#include "reduced_kernels.cuh"
#include "sweep_table.cuh"
#include "vg_ops.h"

#include <type_traits>

namespace vg {
namespace fp64 {

constexpr int MW_NT = 256;

struct Fp64Kernels {
    template <class M, int P, int LPB, int MINB>
    static void x(dim3 grid, int nt, cudaStream_t st, const SweepArgs& a) {
        sweep_x_kernel<M, P, LPB, MINB><<<grid, nt, 0, st>>>(a);
    }
    template <class M, int TX, int TY, int MINB>
    static int y_resident() {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, sweep_y_kernel<M, TX, TY, MINB>, TX, 0);
        return b;
    }
    template <class M, int TX, int TY, int MINB>
    static void y(dim3 grid, int nt, cudaStream_t st, const SweepArgs& a) {
        sweep_y_kernel<M, TX, TY, MINB><<<grid, nt, 0, st>>>(a);
    }
};

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
cudaError_t forcing_impl(const SweepArgs& a, int subcycles, cudaStream_t st) {
    static_assert(M::NU <= aux_planes(M::NW), "the forcing scratch holds aux_planes(NW) conserved planes");
    if (!a.aux) return cudaErrorInvalidValue;
    long n = (long)a.nx * a.ny;
    roundtrip_kernel<M><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a);
    forcing_kernel<M><<<(unsigned)((n + FT - 1) / FT), FT, sizeof(double) * 3 * M::NU * FT, st>>>(a, subcycles);
    return cudaGetLastError();
}

template <class M>
cudaError_t force1_x(const SweepArgs& a, cudaStream_t st) {
    constexpr int P = M::NU > 21 ? 64 : 128;  // the two shared tiles within the 48 KB static limit
    force1_x_kernel<M, P><<<dim3((a.nx + P - 1) / P, a.ny), P, 0, st>>>(a);
    return cudaGetLastError();
}

template <class M>
cudaError_t force1_y(const SweepArgs& a, cudaStream_t st) {
    if constexpr (!M::HAS_Y) {
        return cudaErrorInvalidValue;
    } else {
        constexpr int TX = 64, TY = 64;
        force1_y_kernel<M, TX, TY><<<dim3((a.nx + TX - 1) / TX, (a.ny + TY - 1) / TY), TX, 0, st>>>(a);
        return cudaGetLastError();
    }
}

using ForcingFn = cudaError_t (*)(const SweepArgs&, int, cudaStream_t);

template <class M>
constexpr ForcingFn forcing_of() {
    if constexpr (M::HAS_SOURCE) return &forcing_impl<M>;
    else return nullptr;
}

template <class M>
cudaError_t relax_impl(const SweepArgs& a, cudaStream_t st) {
    long n = (long)a.nx * a.ny;
    relax_kernel<M><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

template <class M>
constexpr SweepFn relax_of() {
    if constexpr (M::NW == 17) return &relax_impl<M>;
    else return nullptr;
}

template <class M>
constexpr Ops make_ops() {
    return Ops{M::NW,
               SweepTable<Fp64Kernels, M>::x,
               SweepTable<Fp64Kernels, M>::y,
               &max_wave_impl<M>,
               &step_begin_impl<M>,
               &finish_impl<M>,
               forcing_of<M>(),
               tile_kind<M>(),
               &force1_x<M>,
               &force1_y<M>,
               relax_of<M>(),
               0,
               std::is_same<M, EulerReducedF64>::value        ? &reduced_reinit_fp64
               : std::is_same<M, EulerMultiphysicsF64>::value ? &multiphysics_reinit_fp64
               : std::is_same<M, MHDReducedF64>::value        ? &mhd_reduced_reinit_fp64
               : std::is_same<M, MHDIntermediateF64>::value   ? &mhd_intermediate_reinit_fp64
               : std::is_same<M, HPRReducedF64>::value        ? &hpr_reduced_reinit_fp64
               : std::is_same<M, HPRIntermediateF64>::value   ? &hpr_intermediate_reinit_fp64
               : std::is_same<M, HPRMultiphysicsF64>::value   ? &hpr_multiphysics_reinit_fp64
                                                              : nullptr};
}

}  // namespace fp64
}  // namespace vg
