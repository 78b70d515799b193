// Volume-fraction reinitialisation of the Euler reduced two-material model:
// MultiphysicsSolvers::reinitialiseVolumeFraction (Solvers/multiphysicssolvers.cpp:164-191 in 1D, :193-... in 2D),
// which solve{,2D} call after every reinitialisationFrequency-th step.  In place on a.out (the step's result);
// the device step counter decides (ctrl->it, already advanced by the step), so the whole time loop stays in one
// CUDA graph.  The layout L names the planes of the two densities (L::R1, L::R2) and, for the multiphysics model
// whose cells also relax both pressures to their volume-fraction mean (relaxTotalPressure), of the two pressures
// (L::PRESSURE, L::P1, L::P2); alpha1 is plane 0 in every model.  The MHD reduced model's reinitialisation
// (Solvers/multiphysicssolvers.cpp:656-... in 1D and 2D) is the Euler reduced model's on its own planes, the MHD
// intermediate model's (:499-...) the multiphysics model's, the HPR reduced model's (:997-1024 in 1D, :1026-...
// in 2D) the Euler reduced model's on its density planes, and the HPR intermediate model's (:841-869 in 1D,
// :871-995 in 2D) the multiphysics model's on its density and pressure planes.
//
// A crossing is a cell j >= 1 with alpha_j < 0.5 <= alpha_{j-1} (descending) or, in 2D, alpha_j > 0.5 >= alpha_{j-1}
// (ascending).  The four cells j-2 .. j+1 take the mixture density in both materials (relaxTotalDensity) and the
// pure volume fraction of their side.  1D: the last descending crossing only, or cell 0 when there is none (the
// reference's loop, run on one thread); 2D: every crossing of every row, then of every column, at most 100 of each
// kind per line as the reference's arrays hold.  Window cells outside the grid, which the reference writes out of
// bounds, are skipped; cell 0 is never a crossing (the reference would compare it with cell -1).
#pragma once

#include "vg_common.cuh"

namespace vg {

struct ReinitEulerReduced {  // alpha1, u, v, rho1, rho2, p
    static constexpr int R1 = 3, R2 = 4, P1 = 0, P2 = 0;
    static constexpr bool PRESSURE = false;
};
struct ReinitEulerMultiphysics {  // alpha1, u, v, rho1, p1, rho2, p2
    static constexpr int R1 = 3, R2 = 5, P1 = 4, P2 = 6;
    static constexpr bool PRESSURE = true;
};
struct ReinitMHDReduced {  // alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi
    static constexpr int R1 = 4, R2 = 5, P1 = 0, P2 = 0;
    static constexpr bool PRESSURE = false;
};
struct ReinitMHDIntermediate {  // alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz, psi
    static constexpr int R1 = 4, R2 = 6, P1 = 5, P2 = 7;
    static constexpr bool PRESSURE = true;
};
struct ReinitHPRReduced {  // alpha1, p, A (9), u, v, w, Jx, Jy, Jz, rho1, rho2
    static constexpr int R1 = 17, R2 = 18, P1 = 0, P2 = 0;
    static constexpr bool PRESSURE = false;
};
struct ReinitHPRIntermediate {  // alpha1, A (9), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2
    static constexpr int R1 = 16, R2 = 18, P1 = 17, P2 = 19;
    static constexpr bool PRESSURE = true;
};
// The HPR multiphysics model (1D; Solvers/multiphysicssolvers.cpp:807-839): relaxTotalDensity, relaxTotalPressure,
// relaxTotalDistortionTensor (pow(alpha_k, 1/3)-weighted) and relaxTotal{X,Y,Z}ThermalImpulse
// (HPR/Multiphysics/hprmultiphysicsstatevector.cpp:614-704), each with the cell's own alpha, then the volume fraction.
// Planes: alpha1, u, v, w, rho1, p1, A1 (9), J1 (3), rho2, p2, A2 (9), J2 (3).
struct ReinitHPRMultiphysics {
    __device__ static void reset(const SweepArgs& a, long idx, double alpha) {
        double* o = a.out;
        const long n = a.plane;
        const double a1 = o[idx], a2 = 1.0 - a1;
        const double rho = (a1 * o[4 * n + idx]) + (a2 * o[18 * n + idx]);
        o[4 * n + idx] = rho;
        o[18 * n + idx] = rho;
        const double p = (a1 * o[5 * n + idx]) + (a2 * o[19 * n + idx]);
        o[5 * n + idx] = p;
        o[19 * n + idx] = p;
        for (int e = 0; e < 9; e++) {
            const double A = (pow(a1, (1.0 / 3.0)) * o[(6 + e) * n + idx]) + (pow(a2, (1.0 / 3.0)) * o[(20 + e) * n + idx]);
            o[(6 + e) * n + idx] = A;
            o[(20 + e) * n + idx] = A;
        }
        for (int e = 0; e < 3; e++) {
            const double J = (a1 * o[(15 + e) * n + idx]) + (a2 * o[(29 + e) * n + idx]);
            o[(15 + e) * n + idx] = J;
            o[(29 + e) * n + idx] = J;
        }
        o[idx] = alpha;
    }
};
template <class L, class = void>
struct custom_reset {
    static constexpr bool value = false;
};
template <class L>
struct custom_reset<L, decltype((void)&L::reset)> {
    static constexpr bool value = true;
};

// relaxTotalDensity (Euler/Multiphysics/eulerreducedstatevector.cpp:281-287, eulermultiphysicsstatevector.cpp:308-314,
// MHD/Multiphysics/mhdreducedstatevector.cpp's relaxTotalDensity), for the multiphysics model relaxTotalPressure
// (:316-329), then the cell's volume fraction
template <class L>
__device__ inline void reduced_reset_cell(const SweepArgs& a, long idx, double alpha) {
    if constexpr (custom_reset<L>::value) {
        L::reset(a, idx, alpha);
    } else {
        const double a1 = a.out[idx];
        const double rho = (a1 * a.out[L::R1 * a.plane + idx]) + ((1.0 - a1) * a.out[L::R2 * a.plane + idx]);
        a.out[L::R1 * a.plane + idx] = rho;
        a.out[L::R2 * a.plane + idx] = rho;
        if constexpr (L::PRESSURE) {
            const double p = (a1 * a.out[L::P1 * a.plane + idx]) + ((1.0 - a1) * a.out[L::P2 * a.plane + idx]);
            a.out[L::P1 * a.plane + idx] = p;
            a.out[L::P2 * a.plane + idx] = p;
        }
        a.out[idx] = alpha;
    }
}

__device__ inline bool reduced_reinit_due(const SweepArgs& a) {
    return !a.ctrl || (a.ctrl->active && a.reinit_freq > 0 && (a.ctrl->it % a.reinit_freq) == 0);
}

template <class L, int NT>
__global__ void __launch_bounds__(NT) reduced_reinit1d_kernel(SweepArgs a) {
    if (!reduced_reinit_due(a)) return;
    __shared__ int part[NT / 32];
    int loc = 0;
    for (int i = 1 + (int)threadIdx.x; i < a.nx; i += NT)
        if (a.out[i] < 0.5 && a.out[i - 1] >= 0.5 && i > loc) loc = i;
    for (int o = 16; o > 0; o >>= 1) loc = max(loc, __shfl_xor_sync(0xffffffffu, loc, o));
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = loc;
    __syncthreads();
    if (threadIdx.x < 4) {
        loc = 0;
        for (int w = 0; w < NT / 32; w++) loc = max(loc, part[w]);
        const int i = loc - 2 + (int)threadIdx.x;
        if (i >= 0 && i < a.nx) reduced_reset_cell<L>(a, i, i < loc ? 0.999 : 0.001);
    }
}

// one line (row: stride 1, or column: stride pitch) of the 2D reinitialisation, by one thread
template <class L>
__device__ inline void reduced_reinit_line(const SweepArgs& a, long start, long stride, int len) {
    int loc1[100], loc2[100], n1 = 0, n2 = 0;
    for (int j = 1; j < len; j++) {
        const double x = a.out[start + j * stride], y = a.out[start + (j - 1) * stride];
        if (x < 0.5 && y >= 0.5 && n1 < 100) loc1[n1++] = j;
        if (x > 0.5 && y <= 0.5 && n2 < 100) loc2[n2++] = j;
    }
    for (int k = 0; k < n1; k++)
        for (int j = loc1[k] - 2; j < loc1[k] + 2; j++)
            if (j >= 0 && j < len) reduced_reset_cell<L>(a, start + j * stride, j < loc1[k] ? 0.999 : 0.001);
    for (int k = 0; k < n2; k++)
        for (int j = loc2[k] - 2; j < loc2[k] + 2; j++)
            if (j >= 0 && j < len) reduced_reset_cell<L>(a, start + j * stride, j < loc2[k] ? 0.001 : 0.999);
}

template <class L>
__global__ void reduced_reinit_rows_kernel(SweepArgs a) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= a.ny || !reduced_reinit_due(a)) return;
    reduced_reinit_line<L>(a, (long)row * a.pitch, 1, a.nx);
}

template <class L>
__global__ void reduced_reinit_cols_kernel(SweepArgs a) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.nx || !reduced_reinit_due(a)) return;
    reduced_reinit_line<L>(a, col, a.pitch, a.ny);
}

// The reinitialisation of one step (kernels: 1 in 1D, 2 in 2D), in place on a.out.
template <class L>
inline cudaError_t reduced_reinit(const SweepArgs& a, cudaStream_t st) {
    if (a.ny == 1) {
        reduced_reinit1d_kernel<L, 256><<<1, 256, 0, st>>>(a);
    } else {
        constexpr int T = 64;
        reduced_reinit_rows_kernel<L><<<(a.ny + T - 1) / T, T, 0, st>>>(a);
        reduced_reinit_cols_kernel<L><<<(a.nx + T - 1) / T, T, 0, st>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace vg
