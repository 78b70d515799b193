// The homogeneous HPR source step shared by the source batch's forward (source_batch.cu, compiled without FMA
// contraction so that it equals the reference's forcing step) and its reverse pass (source_adjoint.cu, compiled
// with contraction: it only needs the stage states as evaluation points of the derivatives, and its own
// recomputations are consistent among themselves, so every checkpoint schedule gives the same bits).
//
// One step of length h is one sub-cycle of HPRForcingSolver's RK4 (Solvers/hprforcingsolver.cpp:332-357) on a
// uniform 1D field with zero limiter bias: there the neighbours of a cell equal each other, so every slope of the
// fractional flux predictor is exactly zero and the predictor reduces to the primitive round trip it performs
// (setConservedVariableVector on a default-constructed state, then computeConservedVariableVector).
#pragma once

#include <cuda_runtime.h>

#include "physics_hpr.cuh"

namespace vg {
namespace srcb {

using H = HPRModel<false>;
constexpr int NV = 17;
constexpr int BT = 128;  // threads per block

__device__ __forceinline__ H::P cell_params(const double* prm, const double* tau, long n, long c) {
    H::P q = H::params(prm, 0.0);
    q.tau1 = tau[c];
    q.tau2 = tau[n + c];
    return q;
}

// The primitive round trip of the forcing's fractional predictor: setcons into a default-constructed state.
__device__ __forceinline__ void set_default(const double* U, const H::P& q, double* W) {
    H::default_state(W);
    H::setcons(U, q, W);
}

// One source step from conserved U; keeps the stage states (conserved, after their round trips) for the reverse
// pass when `stages` is given; returns U'.
__device__ __forceinline__ void step_u(const double* U, const H::P& q, double h, double* Unew, double (*stages)[NV]) {
    double k[4][NV], S[NV], wm[NV], ut[NV];
    H::source(U, q, S);
    for (int v = 0; v < NV; v++) k[0][v] = h * S[v];
    if (stages)
        for (int v = 0; v < NV; v++) stages[0][v] = U[v];
#pragma unroll 1
    for (int s = 0; s < 3; s++) {
        for (int v = 0; v < NV; v++) ut[v] = U[v] + (s < 2 ? (0.5 * k[s][v]) : k[s][v]);
        set_default(ut, q, wm);
        // the 1D predictor X(f): cons of the stage state, plus the zero flux difference (F(U) - F(U) = +0, which
        // turns a -0 component into +0), set into a default-constructed state
        H::cons(wm, q, ut);
        for (int v = 0; v < NV; v++) ut[v] = ut[v] + 0.0;
        set_default(ut, q, wm);
        H::cons(wm, q, ut);
        if (stages)
            for (int v = 0; v < NV; v++) stages[s + 1][v] = ut[v];
        H::source(ut, q, S);
        for (int v = 0; v < NV; v++) k[s + 1][v] = h * S[v];
    }
    for (int v = 0; v < NV; v++) Unew[v] = U[v] + ((1.0 / 6.0) * (k[0][v] + ((2.0 * k[1][v]) + ((2.0 * k[2][v]) + k[3][v]))));
}

// W <- W after `steps` steps (the cell keeps the fields setConservedVariableVector leaves alone: J when not thermal)
__device__ __forceinline__ void advance(double* W, const H::P& q, double h, int steps) {
    double U[NV], Un[NV];
#pragma unroll 1
    for (int i = 0; i < steps; i++) {
        H::cons(W, q, U);
        step_u(U, q, h, Un, nullptr);
        H::setcons(Un, q, W);
    }
}

// One operation of the reversal: advance slot `src` by `count` steps into slot `dst`, or reverse step `step` from
// the state held in slot `src`.
struct Op {
    int kind;  // 0 advance, 1 reverse
    int src, dst, count, step;
};

struct GradArgs {
    const double* W0;      // 17 x n initial state (slot 0)
    double* slots;         // nslot x 17 x n checkpoint slots (slot k at k * 17 * n; slot 0 unused: W0)
    const double* tau;     // 2 x n
    const double* lamT;    // 17 x n  dL/dW(T)
    double* gW;            // 17 x n  dL/dW(0)
    double* gtau;          // 2 x n   dL/dtau
    const Op* ops;
    int nops;
    long n;
    double h;
    int steps;
    double params[kParams];
};

cudaError_t launch_gradient(const GradArgs& a, unsigned blocks, cudaStream_t st);

}  // namespace srcb
}  // namespace vg
