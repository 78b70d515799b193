// HPR relaxation-source sub-cycle: HPRForcingSolver's RK4 with fractional flux predictors, one thread per cell.
//
// HPRForcingSolver::computeRungeKuttaTimeStep{,2D} (Solvers/hprforcingsolver.cpp:341-357, :394-418) evaluates,
// for every cell, four source terms S(U) at stage states that are advanced by slope-limited fractional flux steps
// (dims == 1: X with fractions 1/2, 1/2, 1; dims == 2: X(f/2) Y(f) X(f/2) with f = 1/2, 1/2, 1), and combines them
// as U + (k1 + 2 k2 + 2 k3 + k4) / 6 (:332-339).  Neighbours come from the 1-ghost boundary
// (insertBoundaryCells{,2D}(cells, 1): copies of the edge cells, or wrap-around).  Out of place.
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
// evolveStateByFractionalTimeStep (:791-797); primitive in, primitive out (default-constructed target).
template <class M, int AXIS>
__device__ void frac_evolve(double frac, const double* wl, const double* wm, const double* wr, double dt, double dx,
                            const SweepConst& k, const typename M::P& q, double* out) {
    constexpr int NU = M::NU;
    double uL[NU], uM[NU], uR[NU], xl[NU], xr[NU], fl[NU], fr[NU];
    M::cons(wl, q, uL);
    M::cons(wm, q, uM);
    M::cons(wr, q, uR);
    for (int i = 0; i < NU; i++) {
        double s = slope_f64(uL[i], uM[i], uR[i], k);
        xl[i] = uM[i] - (0.5 * s);
        xr[i] = uM[i] + (0.5 * s);
    }
    M::template flux<AXIS>(xl, q, fl);
    M::template flux<AXIS>(xr, q, fr);
    double c = frac * (dt / dx);
    for (int i = 0; i < NU; i++) xl[i] = uM[i] + (c * (fl[i] - fr[i]));
    M::default_state(out);
    M::setcons(xl, q, out);
}

template <class M>
__global__ void __launch_bounds__(128) forcing_kernel(SweepArgs a, int subcycles) {
    constexpr int NU = M::NU, NW = M::NW;
    const long n = (long)a.nx * a.ny;
    const long idx = blockIdx.x * 128L + threadIdx.x;
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
    const typename M::P q = M::params(a.params, 0.0);
    const int dims = a.ny > 1 ? 2 : 1;

    auto load = [&](long at, double* W) {
        for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + at];
    };
    double W[NW], U[NU], wl[NW], wr[NW], wt[NW], wb[NW];
    // neighbours as the reference builds them: conserved vector of the ghosted cell, then setConservedVariableVector
    // on a default-constructed state (Solvers/hprforcingsolver.cpp:138-147)
    auto neighbour = [&](long at, double* out) {
        load(at, W);
        M::cons(W, q, U);
        M::default_state(out);
        M::setcons(U, q, out);
    };
    neighbour((long)i * a.pitch + ghost1_index(j - 1, a.nx, a.periodic), wl);
    neighbour((long)i * a.pitch + ghost1_index(j + 1, a.nx, a.periodic), wr);
    if (dims == 2) {
        neighbour((long)ghost1_index(i - 1, a.ny, a.periodic) * a.pitch + j, wt);
        neighbour((long)ghost1_index(i + 1, a.ny, a.periodic) * a.pitch + j, wb);
    }
    double uM[NU], S[NU], kk[4][NU], ut[NU], wm[NW], e1[NW], e2[NW], e[NW], ue[NU];
    load(self, W);
    M::cons(W, q, uM);
    M::source(uM, q, S);
    for (int v = 0; v < NU; v++) kk[0][v] = dt * S[v];
    M::default_state(wm);
    const double stage_frac[3] = {0.5, 0.5, 1.0};
    for (int s = 0; s < 3; s++) {
        for (int v = 0; v < NU; v++) ut[v] = uM[v] + (s < 2 ? (0.5 * kk[s][v]) : kk[s][v]);
        M::setcons(ut, q, wm);
        double f = stage_frac[s];
        if (dims == 1) {
            frac_evolve<M, 0>(f, wl, wm, wr, dt, a.dx, k, q, e);
        } else {
            frac_evolve<M, 0>(0.5 * f, wl, wm, wr, dt, a.dx, k, q, e1);
            frac_evolve<M, 1>(f, wt, e1, wb, dt, a.dx, k, q, e2);
            frac_evolve<M, 0>(0.5 * f, wl, e2, wr, dt, a.dx, k, q, e);
        }
        M::cons(e, q, ue);
        M::source(ue, q, S);
        for (int v = 0; v < NU; v++) kk[s + 1][v] = dt * S[v];
    }
    for (int v = 0; v < NU; v++)
        ut[v] = uM[v] + ((1.0 / 6.0) * (kk[0][v] + ((2.0 * kk[1][v]) + ((2.0 * kk[2][v]) + kk[3][v]))));
    M::setcons(ut, q, W);  // the cell keeps its own primitives for fields setConservedVariableVector leaves alone
    for (int v = 0; v < NW; v++) a.out[v * a.plane + self] = W[v];
    if (bad_state<M>(W)) atomicOr(a.err, ERR_STATE);
}

}  // namespace vg
