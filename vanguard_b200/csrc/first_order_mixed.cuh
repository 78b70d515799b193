// First-order FORCE sweeps in the mixed FP32/FP64 form: the FirstOrderSolver loop of first_order_kernels.cuh
// (Solvers/firstordersolver.cpp:232-247, :286-308, :357-379) with the arithmetic split of the mixed SLIC sweeps.
// The interface flux is force_flux_mixed of the two cells' conserved vectors in the model's reconstruction type
// (M::R: FP32 for Euler, FP64 for MHD and HPR) with FP32 flux values; the update accumulates the FP64 difference of
// the two FP32 interface fluxes into the FP64 cell state, so mass, momentum and energy telescope to round-off.
#pragma once

#include "slic_mixed.cuh"

namespace vg {

template <class M, int P>
__global__ void __launch_bounds__(P) force1_x_mixed_kernel(SweepArgs a) {
    using R = typename M::R;
    constexpr int NU = M::NU, NW = M::NW;
    __shared__ double Us[NU][P + 2];
    __shared__ double Fs[NU][P + 1];
    const int p = threadIdx.x;
    const int row = blockIdx.y;
    const int s0 = blockIdx.x * P;
    const int cell = s0 + p;
    const bool out_ok = cell < a.nx;
    const long rowbase = (long)row * a.pitch;
    if (a.ctrl && !a.ctrl->active) {
        if (out_ok)
            for (int v = 0; v < NW; v++) a.out[v * a.plane + rowbase + cell] = a.in[v * a.plane + rowbase + cell];
        return;
    }
    double ts;
    const MixedConst k = mixed_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);
    auto conserve = [&](int slot) {  // slot s holds cell s0 - 1 + s
        const int c = ghost_index(s0 - 1 + slot, a.nx, a.periodic);
        double W[NW], U[NU];
#pragma unroll
        for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + rowbase + c];
        M::cons(W, q, U);
#pragma unroll
        for (int v = 0; v < NU; v++) Us[v][slot] = U[v];
    };
    conserve(p + 1);
    if (p == 0) conserve(0);
    if (p == P - 1) conserve(P + 1);
    __syncthreads();
    auto interface = [&](int f) {  // between slots f and f + 1 (left of cell s0 + f)
        R ua[NU], ub[NU];
        float F[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) {
            ua[v] = (R)Us[v][f];
            ub[v] = (R)Us[v][f + 1];
        }
        force_flux_mixed<M, 0>(ua, ub, k, q, F);
#pragma unroll
        for (int v = 0; v < NU; v++) Fs[v][f] = (double)F[v];
    };
    interface(p);
    if (p == P - 1) interface(P);
    __syncthreads();
    double wave = 0.0;
    if (out_ok) {
        double Un[NU], W[NW];
#pragma unroll
        for (int v = 0; v < NU; v++) Un[v] = fma(k.r, Fs[v][p] - Fs[v][p + 1], Us[v][p + 1]);
        keep_fields<M>(a, rowbase + cell, q, W);
        M::setcons(Un, q, W);
#pragma unroll
        for (int v = 0; v < NW; v++) a.out[v * a.plane + rowbase + cell] = W[v];
        if (bad_state_mixed<M>(W, q)) atomicOr(a.err, ERR_STATE);
        if (a.accumulate_wave) {
            const double s = M::wave(W, q, a.dims);
            if (s > wave) wave = s;
        }
    }
    if (a.accumulate_wave) block_max_to<P>(wave, a.wave_acc);
    if (a.advance_time && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        a.ctrl->t += a.ctrl->dt;
        a.ctrl->it += 1;
    }
}

template <class M, int TX, int TY>
__global__ void __launch_bounds__(TX) force1_y_mixed_kernel(SweepArgs a) {
    using R = typename M::R;
    constexpr int NU = M::NU, NW = M::NW;
    const int col = blockIdx.x * TX + threadIdx.x;
    const bool col_ok = col < a.nx;
    const int c = col_ok ? col : 0;
    const int r0 = blockIdx.y * TY;
    const int r1 = min(r0 + TY, a.ny);
    if (a.ctrl && !a.ctrl->active) {
        if (col_ok)
            for (int r = r0; r < r1; r++)
                for (int v = 0; v < NW; v++)
                    a.out[v * a.plane + (long)r * a.pitch + c] = a.in[v * a.plane + (long)r * a.pitch + c];
        return;
    }
    double ts;
    const MixedConst k = mixed_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);
    auto conserve = [&](int r, double* U) {
        const int rr = ghost_index(r, a.ny, a.periodic);
        double W[NW];
#pragma unroll
        for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + (long)rr * a.pitch + c];
        M::cons(W, q, U);
    };
    auto flux = [&](const double* lo, const double* hi, double* F) {
        R ua[NU], ub[NU];
        float f[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) {
            ua[v] = (R)lo[v];
            ub[v] = (R)hi[v];
        }
        force_flux_mixed<M, 1>(ua, ub, k, q, f);
#pragma unroll
        for (int v = 0; v < NU; v++) F[v] = (double)f[v];
    };
    double u0[NU], u1[NU], F0[NU], F1[NU];
    conserve(r0 - 1, u0);
    conserve(r0, u1);
    flux(u0, u1, F0);  // interface r0 - 1/2
    double wave = 0.0;
    for (int r = r0; r < r1; r++) {
        conserve(r + 1, u0);  // u0 <- cell r + 1
        flux(u1, u0, F1);     // interface r + 1/2
        if (col_ok) {
            const long idx = (long)r * a.pitch + c;
            double Un[NU], W[NW];
#pragma unroll
            for (int v = 0; v < NU; v++) Un[v] = fma(k.r, F0[v] - F1[v], u1[v]);
            keep_fields<M>(a, idx, q, W);
            M::setcons(Un, q, W);
#pragma unroll
            for (int v = 0; v < NW; v++) a.out[v * a.plane + idx] = W[v];
            if (bad_state_mixed<M>(W, q)) atomicOr(a.err, ERR_STATE);
            if (a.accumulate_wave) {
                const double s = M::wave(W, q, 2);
                if (s > wave) wave = s;
            }
        }
#pragma unroll
        for (int v = 0; v < NU; v++) {
            F0[v] = F1[v];
            u1[v] = u0[v];
        }
    }
    if (a.accumulate_wave) block_max_to<TX>(wave, a.wave_acc);
    if (a.advance_time && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        a.ctrl->t += a.ctrl->dt;
        a.ctrl->it += 1;
    }
}

}  // namespace vg
