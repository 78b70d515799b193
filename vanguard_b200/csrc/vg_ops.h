// Host-side dispatch table between the C ABI (vg_api.cu) and the kernel instantiations.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "sweep_table.cuh"
#include "vg_common.cuh"

namespace vg {

// Model variants: which primitive planes are carried on the device.
enum Variant : int {
    V_EULER1 = 0,  // Euler, 1 velocity (1D with v == 0):  rho, u, p
    V_EULER2 = 1,  // Euler, 2 velocities:                 rho, u, v, p
    V_MHD7 = 2,    // MHD with w == Bz == 0:               rho, u, v, p, Bx, By, psi
    V_MHD9 = 3,    // MHD, all components:                 rho, u, v, w, p, Bx, By, Bz, psi
    V_HPR17 = 4,   // HPR, all 17 components:              rho, p, A(9), u, v, w, Jx, Jy, Jz
    V_HPR17S = 5,  // HPR solid (ShockMieGruneisen / GodunovRomenski) or plastic material, same planes
    V_RED6 = 6,    // Euler reduced two-material, w == 0:    alpha1, u, v, rho1, rho2, p
    V_MPH7 = 7,    // Euler multiphysics two-material, w == 0: alpha1, u, v, rho1, p1, rho2, p2
    V_MRED11 = 8,  // MHD reduced two-material: alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi
    V_MINT12 = 9,  // MHD intermediate two-material: alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz, psi
    V_HRED19 = 10,  // HPR reduced two-material: alpha1, p, A(9), u, v, w, Jx, Jy, Jz, rho1, rho2
    V_HINT20 = 11,  // HPR intermediate two-material: alpha1, A(9), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2
    V_HMPH32 = 12,  // HPR multiphysics two-material (1D): alpha1, u, v, w, rho1, p1, A1(9), J1(3), rho2, p2, A2(9), J2(3)
    V_MMPH16 = 13,  // MHD multiphysics two-material (1D): alpha1, u, v, w, rho1, p1, B1(3), psi1, rho2, p2, B2(3), psi2
    V_COUNT = 14
};

struct Ops {
    int nw;  // carried primitive planes
    // One sweep per launch configuration (see sweep_table.cuh).  a.in / a.out must not alias.
    const SweepFn* x;
    const SweepFn* y;
    // Maximum wave speed of a.in folded into ctrl->smax_next (caller zeroes it first).
    cudaError_t (*max_wave)(const SweepArgs& a, cudaStream_t st);
    // dt for the next step from ctrl->smax_next (and corner ghosts in 2D); zeroes smax_next.
    cudaError_t (*step_begin)(const SweepArgs& a, cudaStream_t st);
    // *out = maximum wave speed including corner ghosts (reads ctrl->smax_next).
    cudaError_t (*max_wave_finish)(const SweepArgs& a, double* out, cudaStream_t st);
    // One relaxation-source sub-cycle of length 0.5 dt / subcycles, a.in -> a.out, with a.aux as scratch
    // (kForcingLaunches kernels; null: model has no source).
    cudaError_t (*forcing)(const SweepArgs& a, int subcycles, cudaStream_t st);
    int tile_kind;  // SweepTable kind: 0 default, 1 big models, 2 PAIR_X models (names of the launch configurations)
    // First-order FORCE sweeps (FirstOrderSolver), null where the form has none.
    SweepFn x1 = nullptr;
    SweepFn y1 = nullptr;
    // Stiff relaxation of the source over dt * a.dt_scale, in place on a.out (HPR), null where the model has none.
    SweepFn relax = nullptr;
    // Planes of the box of the TMA-staged X sweep (its tensor maps: box {130, 2, tma_planes}); 0: no TMA sweep.
    int tma_planes = 0;
    // Volume-fraction reinitialisation of one step, in place on a.out (Euler reduced model), null for the others.
    SweepFn reinit = nullptr;
    // The whole second-order 1D run in one thread block, in place on a.in == a.out (solve1d_kernels.cuh), for rows of
    // solve1d_min .. solve1d_max cells; null where the model has none (models with a source or a per-step c_h).
    SweepFn solve1d = nullptr;
    long solve1d_min = 0, solve1d_max = 0;
};

constexpr int kForcingLaunches = 2;  // kernels per forcing sub-cycle

// Exact-FP64 kernels (compiled with -fmad=false; bitwise parity with the reference).
const Ops* ops_fp64(int variant);
// Mixed FP32/FP64 kernels.
const Ops* ops_mixed(int variant);
// The exact source sub-cycles (slic_fp64.cu), which the mixed form uses unchanged: HPR relaxation, MHD GLM damping.
cudaError_t hpr_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st);
cudaError_t mhd7_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st);
cudaError_t mhd9_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st);
// The stiff HPR relaxation (slic_fp64.cu), FP64 in both forms.
cudaError_t hpr_relax_fp64(const SweepArgs& a, cudaStream_t st);
cudaError_t hpr_solid_forcing_fp64(const SweepArgs& a, int subcycles, cudaStream_t st);
cudaError_t hpr_solid_relax_fp64(const SweepArgs& a, cudaStream_t st);
// The reduced model's volume-fraction reinitialisation (slic_fp64.cu), shared by both forms.
cudaError_t reduced_reinit_fp64(const SweepArgs& a, cudaStream_t st);
cudaError_t multiphysics_reinit_fp64(const SweepArgs& a, cudaStream_t st);
cudaError_t mhd_reduced_reinit_fp64(const SweepArgs& a, cudaStream_t st);
cudaError_t mhd_intermediate_reinit_fp64(const SweepArgs& a, cudaStream_t st);
cudaError_t hpr_reduced_reinit_fp64(const SweepArgs& a, cudaStream_t st);
cudaError_t hpr_intermediate_reinit_fp64(const SweepArgs& a, cudaStream_t st);
cudaError_t hpr_multiphysics_reinit_fp64(const SweepArgs& a, cudaStream_t st);

// Planes of the source sub-cycles' scratch (SweepArgs::aux), which holds conserved vectors: a model carries at most
// one conserved component more than primitive planes (the two-material models' rho alpha1), which forcing_impl
// checks at compile time.
constexpr int aux_planes(int max_nw) { return max_nw + 1; }

// Record the text returned by vg_last_error_string() on this thread.
void set_last_error(const std::string& msg);

}  // namespace vg
