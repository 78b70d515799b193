// Mixed FP32/FP64 SLIC sweep kernels (VG_MIXED), generic over a model policy from physics_mixed.cuh.
// Same tiling as slic_kernels.cuh (staged shared-memory X sweep, register-marching Y sweep); states stay
// FP64, slopes / fluxes / evolution increments are FP32, the update accumulates in FP64.
#pragma once

#include "vg_common.cuh"

namespace vg {

__device__ __forceinline__ float limiter_f32(float r, float w, int id) {
    if (r < 0.0f) return 0.0f;
    float xi_r = __fdividef(2.0f, (1.0f - w) + (1.0f + w) * r);
    if (id == 0) {
        if (r < 0.5f) return 2.0f * r;
        if (r < 1.0f) return 1.0f;
        return fminf(fminf(r, xi_r), 2.0f);
    } else if (id == 1) {
        return fminf(__fdividef(2.0f * r, 1.0f + r), xi_r);
    }
    if (r < 1.0f) return r;
    return fminf(1.0f, xi_r);
}

struct MixedConst {
    float half_r, r_f, rinv_f, cm, cp, bias, floor5;
    double r;
    int limiter;
};

__device__ __forceinline__ MixedConst mixed_const(const SweepArgs& a, double& ts) {
    ts = (a.ctrl ? a.ctrl->dt : a.dt_host) * a.dt_scale;
    MixedConst k;
    k.r = ts / a.dx;
    k.r_f = (float)k.r;
    k.rinv_f = (float)(a.dx / ts);
    k.half_r = (float)(0.5 * k.r);
    k.cm = (float)(0.5 * (1.0 + a.bias));
    k.cp = (float)(0.5 * (1.0 - a.bias));
    k.bias = (float)a.bias;
    k.floor5 = 1e-5f;
    k.limiter = a.limiter;
    return k;
}

// Both evolved edge states of one cell (FP64), from the FP64 conserved vectors of the cell and its
// neighbours.  ua_left_side: x_L + dt/2 evolution; ua_right_side: x_R + dt/2 evolution.
template <class M, int AXIS>
__device__ __forceinline__ void evolve_edges_mixed(const double* uL, const double* u, const double* uR,
                                                   const MixedConst& k, const typename M::P& q,
                                                   double* ua_left_side, double* ua_right_side) {
    constexpr int NU = M::NU;
    double xl[NU], xr[NU];
#pragma unroll
    for (int i = 0; i < NU; i++) {
        float dm = (float)(u[i] - uL[i]);
        float dp = (float)(uR[i] - u[i]);
        float s = fmaf(k.cm, dm, k.cp * dp);
        float num = fabsf(dm) < k.floor5 ? k.floor5 : dm;
        float den = fabsf(dp) < k.floor5 ? k.floor5 : dp;
        s *= limiter_f32(__fdividef(num, den), k.bias, k.limiter);
        double hs = (double)(0.5f * s);
        xl[i] = u[i] - hs;
        xr[i] = u[i] + hs;
    }
    float fl[NU], fr[NU];
    M::template flux<AXIS>(xl, q, fl);
    M::template flux<AXIS>(xr, q, fr);
#pragma unroll
    for (int i = 0; i < NU; i++) {
        double ev = (double)(k.half_r * (fl[i] - fr[i]));
        ua_left_side[i] = xl[i] + ev;
        ua_right_side[i] = xr[i] + ev;
    }
}

// FORCE flux of FP64 states ua (left) and ub (right), FP32 result.
template <class M, int AXIS>
__device__ __forceinline__ void force_flux_mixed(const double* ua, const double* ub, const MixedConst& k,
                                                 const typename M::P& q, float* F) {
    constexpr int NU = M::NU;
    float fa[NU], fb[NU], fri[NU];
    double uri[NU];
    M::template flux<AXIS>(ua, q, fa);
    M::template flux<AXIS>(ub, q, fb);
#pragma unroll
    for (int i = 0; i < NU; i++) uri[i] = 0.5 * (ua[i] + ub[i]) + (double)(0.5f * k.r_f * (fa[i] - fb[i]));
    M::template flux<AXIS>(uri, q, fri);
#pragma unroll
    for (int i = 0; i < NU; i++) {
        float lf = 0.5f * (fa[i] + fb[i]) + 0.5f * k.rinv_f * (float)(ua[i] - ub[i]);
        F[i] = 0.5f * (lf + fri[i]);
    }
}

template <class M>
__device__ __forceinline__ bool bad_state_mixed(const double* W) {
    double rho = M::density(W), p = M::pressure(W);
    return !(rho > 0.0) || !(p > 0.0) || !isfinite(rho) || !isfinite(p);
}

// ----------------------------------------------------------------------------------------- X sweep
template <class M, int P, int LPB>
__global__ void __launch_bounds__(P* LPB) sweep_x_mixed_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW;
    constexpr int NT = P * LPB;
    __shared__ double Us[NU][LPB][P + 2];
    __shared__ double Es[NU][LPB][P];
    __shared__ float Fs[NU][LPB][P];

    const int p = threadIdx.x % P, l = threadIdx.x / P;
    const int row = blockIdx.y * LPB + l;
    const int len = a.nx;
    const int s0 = blockIdx.x * (P - 2);
    const int cell = s0 - 1 + p;
    const bool row_ok = row < a.ny;
    const bool out_ok = row_ok && p >= 1 && p <= P - 2 && cell < len;
    const long rowbase = (long)(row_ok ? row : 0) * a.pitch;

    if (a.ctrl && !a.ctrl->active) {
        if (out_ok)
            for (int v = 0; v < NW; v++) a.out[v * a.plane + rowbase + cell] = a.in[v * a.plane + rowbase + cell];
        return;
    }
    double ts;
    const MixedConst k = mixed_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);

    auto conserve = [&](int slot) {
        int c = ghost_index(s0 - 2 + slot, len, a.periodic);
        double W[NW], U[NU];
#pragma unroll
        for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + rowbase + c];
        M::cons(W, q, U);
#pragma unroll
        for (int v = 0; v < NU; v++) Us[v][l][slot] = U[v];
    };
    conserve(p + 1);
    if (p == 0) conserve(0);
    if (p == P - 1) conserve(P + 1);
    __syncthreads();

    double ub[NU];
    {
        double uL[NU], u[NU], uR[NU], ua[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) {
            uL[v] = Us[v][l][p];
            u[v] = Us[v][l][p + 1];
            uR[v] = Us[v][l][p + 2];
        }
        evolve_edges_mixed<M, 0>(uL, u, uR, k, q, ub, ua);
#pragma unroll
        for (int v = 0; v < NU; v++) Es[v][l][p] = ua[v];
    }
    __syncthreads();

    if (p >= 1) {
        double ua[NU];
        float F[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) ua[v] = Es[v][l][p - 1];
        force_flux_mixed<M, 0>(ua, ub, k, q, F);
#pragma unroll
        for (int v = 0; v < NU; v++) Fs[v][l][p] = F[v];
    }
    __syncthreads();

    double wave = 0.0;
    if (out_ok) {
        double Un[NU], W[NW];
#pragma unroll
        for (int v = 0; v < NU; v++)
            Un[v] = fma(k.r, (double)Fs[v][l][p] - (double)Fs[v][l][p + 1], Us[v][l][p + 1]);
        M::setcons(Un, q, W);
#pragma unroll
        for (int v = 0; v < NW; v++) a.out[v * a.plane + rowbase + cell] = W[v];
        if (bad_state_mixed<M>(W)) atomicOr(a.err, ERR_STATE);
        if (a.accumulate_wave) {
            double s = M::wave(W, q, a.dims);
            if (s > wave) wave = s;
        }
    }
    if (a.accumulate_wave) block_max_to<NT>(wave, a.wave_acc);
    if (a.advance_time && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        a.ctrl->t += a.ctrl->dt;
        a.ctrl->it += 1;
    }
}

// ----------------------------------------------------------------------------------------- Y sweep
template <class M, int TX, int TY>
__global__ void __launch_bounds__(TX) sweep_y_mixed_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW;
    const int col = blockIdx.x * TX + threadIdx.x;
    const bool col_ok = col < a.nx;
    const int len = a.ny;
    const int r0 = blockIdx.y * TY;
    const int r1 = min(r0 + TY, len);
    const int c = col_ok ? col : 0;

    if (a.ctrl && !a.ctrl->active) {
        if (col_ok)
            for (int r = r0; r < r1; r++)
                for (int v = 0; v < NW; v++) a.out[v * a.plane + (long)r * a.pitch + c] = a.in[v * a.plane + (long)r * a.pitch + c];
        return;
    }
    double ts;
    const MixedConst k = mixed_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);

    auto conserve = [&](int r, double* U) {
        int rr = ghost_index(r, len, a.periodic);
        double W[NW];
#pragma unroll
        for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + (long)rr * a.pitch + c];
        M::cons(W, q, U);
    };

    double um1[NU], u0[NU], up1[NU], ua_prev[NU], dummy[NU];
    float f_prev[NU];
    double wave = 0.0;
    conserve(r0 - 2, up1);
    conserve(r0 - 1, um1);
    conserve(r0, u0);
    evolve_edges_mixed<M, 1>(up1, um1, u0, k, q, dummy, ua_prev);
    for (int r = r0; r <= r1; r++) {
        conserve(r + 1, up1);
        double ub[NU], ua_next[NU];
        evolve_edges_mixed<M, 1>(um1, u0, up1, k, q, ub, ua_next);
        float F[NU];
        force_flux_mixed<M, 1>(ua_prev, ub, k, q, F);
        if (r > r0 && col_ok) {
            double Un[NU], W[NW];
#pragma unroll
            for (int v = 0; v < NU; v++) Un[v] = fma(k.r, (double)f_prev[v] - (double)F[v], um1[v]);
            M::setcons(Un, q, W);
#pragma unroll
            for (int v = 0; v < NW; v++) a.out[v * a.plane + (long)(r - 1) * a.pitch + c] = W[v];
            if (bad_state_mixed<M>(W)) atomicOr(a.err, ERR_STATE);
            if (a.accumulate_wave) {
                double s = M::wave(W, q, 2);
                if (s > wave) wave = s;
            }
        }
#pragma unroll
        for (int v = 0; v < NU; v++) {
            f_prev[v] = F[v];
            ua_prev[v] = ua_next[v];
            um1[v] = u0[v];
            u0[v] = up1[v];
        }
    }
    if (a.accumulate_wave) block_max_to<TX>(wave, a.wave_acc);
    if (a.advance_time && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        a.ctrl->t += a.ctrl->dt;
        a.ctrl->it += 1;
    }
}

}  // namespace vg
