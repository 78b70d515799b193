// Relaxation-source sub-cycle: HPRForcingSolver's RK4 with fractional flux predictors, one thread per cell; the
// MHD GLM damping of MHDForcingSolver (Solvers/mhdforcingsolver.cpp) is the same scheme with the MHD model.
//
// HPRForcingSolver::computeRungeKuttaTimeStep{,2D} (Solvers/hprforcingsolver.cpp:341-357, :394-418) evaluates,
// for every cell, four source terms S(U) at stage states that are advanced by slope-limited fractional flux steps
// (dims == 1: X with fractions 1/2, 1/2, 1; dims == 2: X(f/2) Y(f) X(f/2) with f = 1/2, 1/2, 1), and combines them
// as U + (k1 + 2 k2 + 2 k3 + k4) / 6 (:332-339).  Neighbours come from the 1-ghost boundary
// (insertBoundaryCells{,2D}(cells, 1): copies of the edge cells, or wrap-around).  Out of place.
//
// Two launches per sub-cycle.  roundtrip_kernel stores, for every cell, the conserved vector that each fractional
// flux step evaluates for it as a neighbour (its conserved vector set into a default-constructed state, converted
// back); forcing_kernel then reads neighbours from there instead of recomputing them in every stage.  The RK4
// increments k1..k3 of each thread live in shared memory, and the stages and the X(f/2) Y(f) X(f/2) predictor
// sequence are loops rather than unrolled copies, so the 17-component model code is instantiated once per axis.
#pragma once

#include "slic_kernels.cuh"
#include "vg_common.cuh"

namespace vg {

__device__ __forceinline__ int ghost1_index(int k, int n, int periodic) {
    if (k >= 0 && k < n) return k;
    if (periodic) return k < 0 ? k + n : k - n;
    return k < 0 ? 0 : n - 1;
}

// HPRSolvers::evolveStateByFractional{X,Y}TimeStep (Solvers/hprsolvers.cpp:606-620, :673-687) with
// evolveStateByFractionalTimeStep (:791-797) on the conserved vectors of the three cells; the result is set into a
// default-constructed state (primitive out).
template <class M, int AXIS>
__device__ __forceinline__ void frac_evolve_u(double frac, const double* uL, const double* uM, const double* uR,
                                              double dt, double dx, const SweepConst& k, const typename M::P& q,
                                              double* out) {
    constexpr int NU = M::NU;
    double xl[NU], xr[NU], fl[NU], fr[NU];
#pragma unroll
    for (int i = 0; i < NU; i++) {
        double s = slope_f64(uL[i], uM[i], uR[i], k);
        xl[i] = uM[i] - (0.5 * s);
        xr[i] = uM[i] + (0.5 * s);
    }
    M::template flux<AXIS>(xl, q, fl);
    M::template flux<AXIS>(xr, q, fr);
    double c = frac * (dt / dx);
#pragma unroll
    for (int i = 0; i < NU; i++) xl[i] = uM[i] + (c * (fl[i] - fr[i]));
    M::default_state(out);
    M::setcons(xl, q, out);
}

// Neighbour round trip of every cell into a.aux (conserved planes): cons -> setConservedVariableVector on a
// default-constructed state -> cons (Solvers/hprforcingsolver.cpp:138-147 then :606-620).
template <class M>
__global__ void __launch_bounds__(256) roundtrip_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW;
    const long n = (long)a.nx * a.ny;
    const long idx = blockIdx.x * 256L + threadIdx.x;
    if (idx >= n || (a.ctrl && !a.ctrl->active)) return;
    const int i = (int)(idx / a.nx), j = (int)(idx - (long)i * a.nx);
    const long self = (long)i * a.pitch + j;
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);
    double W[NW], U[NU];
    for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + self];
    M::cons(W, q, U);
    M::default_state(W);
    M::setcons(U, q, W);
    M::cons(W, q, U);
    for (int v = 0; v < NU; v++) a.aux[v * a.plane + self] = U[v];
}

constexpr int FT = 64;  // threads per forcing block

// Minimum resident blocks asked of the register allocator: 6 (168 registers) measured fastest for HPR; a model may
// ask for more with FORCING_MIN_BLOCKS.  The kernel is FP64-latency bound, so more resident warps can pay for a few
// spills; the choice never changes a result.
template <class M, class = void>
struct forcing_blocks {
    static constexpr int value = 6;
};
template <class M>
struct forcing_blocks<M, decltype((void)M::FORCING_MIN_BLOCKS)> {
    static constexpr int value = M::FORCING_MIN_BLOCKS;
};

template <class M>
__global__ void __launch_bounds__(FT, forcing_blocks<M>::value) forcing_kernel(SweepArgs a, int subcycles) {
    constexpr int NU = M::NU, NW = M::NW;
    extern __shared__ double ksh[];  // k1, k2, k3 of this block's threads: [stage][component][thread]
    const long n = (long)a.nx * a.ny;
    const long idx = blockIdx.x * (long)FT + threadIdx.x;
    if (idx >= n) return;
    const int i = (int)(idx / a.nx), j = (int)(idx - (long)i * a.nx);
    const long self = (long)i * a.pitch + j;
    if (a.ctrl && !a.ctrl->active) {
        for (int v = 0; v < NW; v++) a.out[v * a.plane + self] = a.in[v * a.plane + self];
        return;
    }
    // Solvers/hprsecondordersolver.cpp:516-519: time step 0.5 * (dt / subcyclingIterations)
    const double dt = 0.5 * ((a.ctrl ? a.ctrl->dt : a.dt_host) / subcycles);
    SweepConst k;
    k.cm = 0.5 * (1.0 + a.bias);
    k.cp = 0.5 * (1.0 - a.bias);
    k.bias = a.bias;
    k.floor5 = a.floor5;
    k.limiter = a.limiter;
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);
    const int dims = a.ny > 1 ? 2 : 1;
    auto kk = [&](int s, int v) -> double& { return ksh[(s * NU + v) * FT + threadIdx.x]; };
    // neighbours through the 1-ghost boundary: left, right, top, bottom
    const long nb[4] = {(long)i * a.pitch + ghost1_index(j - 1, a.nx, a.periodic),
                        (long)i * a.pitch + ghost1_index(j + 1, a.nx, a.periodic),
                        dims == 2 ? (long)ghost1_index(i - 1, a.ny, a.periodic) * a.pitch + j : self,
                        dims == 2 ? (long)ghost1_index(i + 1, a.ny, a.periodic) * a.pitch + j : self};

    double uM[NU], S[NU], W[NW];
    for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + self];
    M::cons(W, q, uM);
    M::source(uM, q, S);
    for (int v = 0; v < NU; v++) kk(0, v) = dt * S[v];
    const double stage_frac[3] = {0.5, 0.5, 1.0};
#pragma unroll 1
    for (int s = 0; s < 3; s++) {
        double ut[NU], wm[NW];
        for (int v = 0; v < NU; v++) ut[v] = uM[v] + (s < 2 ? (0.5 * kk(s, v)) : kk(s, v));
        M::default_state(wm);
        M::setcons(ut, q, wm);
        const double f = stage_frac[s];
        // dims == 1: X(f); dims == 2: X(f/2), Y(f), X(f/2)
        const int nsub = dims == 1 ? 1 : 3;
#pragma unroll 1
        for (int p = 0; p < nsub; p++) {
            const int axis = (dims == 2 && p == 1) ? 1 : 0;
            const double fr = dims == 1 ? f : (p == 1 ? f : 0.5 * f);
            double uA[NU], uB[NU], um[NU];
            for (int v = 0; v < NU; v++) {
                uA[v] = a.aux[v * a.plane + nb[2 * axis]];
                uB[v] = a.aux[v * a.plane + nb[2 * axis + 1]];
            }
            M::cons(wm, q, um);
            if (axis == 0)
                frac_evolve_u<M, 0>(fr, uA, um, uB, dt, a.dx, k, q, wm);
            else
                frac_evolve_u<M, 1>(fr, uA, um, uB, dt, a.dx, k, q, wm);
        }
        M::cons(wm, q, ut);
        M::source(ut, q, S);
        if (s < 2)
            for (int v = 0; v < NU; v++) kk(s + 1, v) = dt * S[v];
    }
    // S holds the last stage's source; k4 = dt * S
    for (int v = 0; v < NU; v++) {
        const double k4 = dt * S[v];
        uM[v] = uM[v] + ((1.0 / 6.0) * (kk(0, v) + ((2.0 * kk(1, v)) + ((2.0 * kk(2, v)) + k4))));
    }
    M::setcons(uM, q, W);  // the cell keeps its own primitives for fields setConservedVariableVector leaves alone
    for (int v = 0; v < NW; v++) a.out[v * a.plane + self] = W[v];
    if (bad_state<M>(W, q)) atomicOr(a.err, ERR_STATE);
}

}  // namespace vg
