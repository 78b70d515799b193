// Volume-fraction reinitialisation of the Euler reduced two-material model:
// MultiphysicsSolvers::reinitialiseVolumeFraction (Solvers/multiphysicssolvers.cpp:164-191 in 1D, :193-... in 2D),
// which solve{,2D} call after every reinitialisationFrequency-th step.  In place on a.out (the step's result);
// the device step counter decides (ctrl->it, already advanced by the step), so the whole time loop stays in one
// CUDA graph.  MPH selects the multiphysics model: planes alpha1 0, rho1 3, p1 4, rho2 5, p2 6, and its cells also
// relax both pressures to their volume-fraction mean (relaxTotalPressure); the reduced model's planes are alpha1 0,
// rho1 3, rho2 4.
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

// relaxTotalDensity (Euler/Multiphysics/eulerreducedstatevector.cpp:281-287, eulermultiphysicsstatevector.cpp:308-314),
// for the multiphysics model relaxTotalPressure (:316-329), then the cell's volume fraction
template <bool MPH>
__device__ inline void reduced_reset_cell(const SweepArgs& a, long idx, double alpha) {
    constexpr int I1 = 3, I2 = MPH ? 5 : 4;
    const double a1 = a.out[idx];
    const double rho = (a1 * a.out[I1 * a.plane + idx]) + ((1.0 - a1) * a.out[I2 * a.plane + idx]);
    a.out[I1 * a.plane + idx] = rho;
    a.out[I2 * a.plane + idx] = rho;
    if constexpr (MPH) {
        const double p = (a1 * a.out[4 * a.plane + idx]) + ((1.0 - a1) * a.out[6 * a.plane + idx]);
        a.out[4 * a.plane + idx] = p;
        a.out[6 * a.plane + idx] = p;
    }
    a.out[idx] = alpha;
}

__device__ inline bool reduced_reinit_due(const SweepArgs& a) {
    return !a.ctrl || (a.ctrl->active && a.reinit_freq > 0 && (a.ctrl->it % a.reinit_freq) == 0);
}

template <bool MPH, int NT>
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
        if (i >= 0 && i < a.nx) reduced_reset_cell<MPH>(a, i, i < loc ? 0.999 : 0.001);
    }
}

// one line (row: stride 1, or column: stride pitch) of the 2D reinitialisation, by one thread
template <bool MPH>
__device__ inline void reduced_reinit_line(const SweepArgs& a, long start, long stride, int len) {
    int loc1[100], loc2[100], n1 = 0, n2 = 0;
    for (int j = 1; j < len; j++) {
        const double x = a.out[start + j * stride], y = a.out[start + (j - 1) * stride];
        if (x < 0.5 && y >= 0.5 && n1 < 100) loc1[n1++] = j;
        if (x > 0.5 && y <= 0.5 && n2 < 100) loc2[n2++] = j;
    }
    for (int k = 0; k < n1; k++)
        for (int j = loc1[k] - 2; j < loc1[k] + 2; j++)
            if (j >= 0 && j < len) reduced_reset_cell<MPH>(a, start + j * stride, j < loc1[k] ? 0.999 : 0.001);
    for (int k = 0; k < n2; k++)
        for (int j = loc2[k] - 2; j < loc2[k] + 2; j++)
            if (j >= 0 && j < len) reduced_reset_cell<MPH>(a, start + j * stride, j < loc2[k] ? 0.001 : 0.999);
}

template <bool MPH>
__global__ void reduced_reinit_rows_kernel(SweepArgs a) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= a.ny || !reduced_reinit_due(a)) return;
    reduced_reinit_line<MPH>(a, (long)row * a.pitch, 1, a.nx);
}

template <bool MPH>
__global__ void reduced_reinit_cols_kernel(SweepArgs a) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.nx || !reduced_reinit_due(a)) return;
    reduced_reinit_line<MPH>(a, col, a.pitch, a.ny);
}

// The reinitialisation of one step (kernels: 1 in 1D, 2 in 2D), in place on a.out.
template <bool MPH>
inline cudaError_t reduced_reinit(const SweepArgs& a, cudaStream_t st) {
    if (a.ny == 1) {
        reduced_reinit1d_kernel<MPH, 256><<<1, 256, 0, st>>>(a);
    } else {
        constexpr int T = 64;
        reduced_reinit_rows_kernel<MPH><<<(a.ny + T - 1) / T, T, 0, st>>>(a);
        reduced_reinit_cols_kernel<MPH><<<(a.nx + T - 1) / T, T, 0, st>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace vg
