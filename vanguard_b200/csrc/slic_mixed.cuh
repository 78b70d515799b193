// Mixed FP32/FP64 SLIC sweep kernels (VG_MIXED), generic over a model policy from physics_mixed.cuh.
// Same tiling as slic_kernels.cuh (staged shared-memory X sweep, register-marching Y sweep); states stay
// FP64, flux values and their combinations are FP32, the update accumulates in FP64.
#pragma once

#include "physics_mixed.cuh"
#include "slic_kernels.cuh"
#include "vg_common.cuh"

namespace vg {

// Limiter of Solvers/slopelimiters.cpp:7-74 on the FP64 slope ratio; the ratio and xi_R use the hardware
// reciprocal approximation (relative error ~2^-22), which only moves the limiter's kinks by that amount.
__device__ __forceinline__ double limiter_approx(double r, double w, int id) {
    if (r < 0.0) return 0.0;
    double xi_r = 2.0 * rcp_approx((1.0 - w) + (1.0 + w) * r);
    if (id == 0) {
        if (r < 0.5) return 2.0 * r;
        if (r < 1.0) return 1.0;
        return fmin(fmin(r, xi_r), 2.0);
    } else if (id == 1) {
        return fmin(2.0 * r * rcp_approx(1.0 + r), xi_r);
    }
    if (r < 1.0) return r;
    return fmin(1.0, xi_r);
}

// FP32 twin of limiter_approx for models whose reconstruction is FP32.
__device__ __forceinline__ float limiter_approx(float r, float w, int id) {
    if (r < 0.0f) return 0.0f;
    float xi_r = 2.0f * rcp_approx_f((1.0f - w) + (1.0f + w) * r);
    if (id == 0) {
        if (r < 0.5f) return 2.0f * r;
        if (r < 1.0f) return 1.0f;
        return fminf(fminf(r, xi_r), 2.0f);
    } else if (id == 1) {
        return fminf(2.0f * r * rcp_approx_f(1.0f + r), xi_r);
    }
    if (r < 1.0f) return r;
    return fminf(1.0f, xi_r);
}

struct MixedConst {
    float half_r, r_f, rinv_f;
    double r, cm, cp, bias, floor5;
    float cm_f, cp_f, bias_f, floor5_f;
    int limiter;
    bool one_rcp;  // superbee or minbee with |bias| <= 1: half_slope_mixed needs one reciprocal
};

// Half the limited slope, (Delta / 2) xi(r), of SlopeLimiters::computeSlopeVector (Solvers/slopelimiters.cpp:217-246)
// and computeSlopeLimiter (:7-74) in the mixed form.  For |w| <= 1 and r >= 1, xi_R = 2 / ((1 - w) + (1 + w) r) is
// at most 1, hence at most r and 2, so superbee's min(r, xi_R, 2) and minbee's min(1, xi_R) are xi_R, and
// xi_R / 2 = den / ((1 - w) den + (1 + w) num).  The branch tests r < 0, 1/2, 1 are sign tests of (num - t den) den,
// so one reciprocal (of den, or of that denominator) serves every branch.  Van Leer and |w| > 1 use limiter_approx.
__device__ __forceinline__ double half_slope_mixed(double dm, double dp, const MixedConst& k) {
    const double num = fabs(dm) < k.floor5 ? k.floor5 : dm;
    const double den = fabs(dp) < k.floor5 ? k.floor5 : dp;
    const double base = fma(k.cm, dm, k.cp * dp);
    if (!k.one_rcp) return 0.5 * base * limiter_approx(num * rcp_approx(den), k.bias, k.limiter);
    const bool ge1 = (num - den) * den >= 0.0;
    const double f = (ge1 ? den : num) * rcp_approx(ge1 ? fma(1.0 + k.bias, num, (1.0 - k.bias) * den) : den);
    double half_xi;
    if (k.limiter == 0)
        half_xi = (ge1 || (num - 0.5 * den) * den < 0.0) ? f : 0.5;
    else
        half_xi = ge1 ? f : 0.5 * f;
    return num * den < 0.0 ? 0.0 : base * half_xi;
}

// FP32 twin of half_slope_mixed (same branches, FP32 operands) for FP32 reconstruction.
__device__ __forceinline__ float half_slope_mixed(float dm, float dp, const MixedConst& k) {
    const float num = fabsf(dm) < k.floor5_f ? k.floor5_f : dm;
    const float den = fabsf(dp) < k.floor5_f ? k.floor5_f : dp;
    const float base = fmaf(k.cm_f, dm, k.cp_f * dp);
    if (!k.one_rcp) return 0.5f * base * limiter_approx(num * rcp_approx_f(den), k.bias_f, k.limiter);
    const bool ge1 = (num - den) * den >= 0.0f;
    const float f = (ge1 ? den : num) * rcp_approx_f(ge1 ? fmaf(1.0f + k.bias_f, num, (1.0f - k.bias_f) * den) : den);
    float half_xi;
    if (k.limiter == 0)
        half_xi = (ge1 || (num - 0.5f * den) * den < 0.0f) ? f : 0.5f;
    else
        half_xi = ge1 ? f : 0.5f * f;
    return num * den < 0.0f ? 0.0f : base * half_xi;
}

__device__ __forceinline__ MixedConst mixed_const(const SweepArgs& a, double& ts) {
    MixedConst k;
    if (a.ctrl) {
        ts = a.ctrl->dt * a.dt_scale;
        k.r = a.ctrl->kr[a.kslot];
        k.r_f = a.ctrl->kr_f[a.kslot];
        k.rinv_f = a.ctrl->krinv_f[a.kslot];
        k.half_r = a.ctrl->khalf_r_f[a.kslot];
    } else {
        ts = a.dt_host * a.dt_scale;
        k.r = a.r_host;
        k.r_f = a.r_host_f;
        k.rinv_f = a.rinv_host_f;
        k.half_r = a.half_r_host_f;
    }
    k.cm = 0.5 * (1.0 + a.bias);
    k.cp = 0.5 * (1.0 - a.bias);
    k.bias = a.bias;
    k.floor5 = a.floor5;
    k.cm_f = (float)k.cm;
    k.cp_f = (float)k.cp;
    k.bias_f = (float)a.bias;
    k.floor5_f = (float)a.floor5;
    k.limiter = a.limiter;
    k.one_rcp = a.limiter != 1 && fabs(a.bias) <= 1.0;
    return k;
}

// Models whose evolved states must pass through the stored primitive form, as the reference's do, declare
// ROUNDTRIP_EVOLVED (for the others that trip only rounds, and the mixed form skips it).
template <class M, class = void>
struct roundtrip_evolved {
    static constexpr bool value = false;
};
template <class M>
struct roundtrip_evolved<M, decltype((void)M::ROUNDTRIP_EVOLVED)> {
    static constexpr bool value = M::ROUNDTRIP_EVOLVED;
};

// Both evolved edge states of one cell (type M::R), from the cell's FP64 conserved vector u and its slope
// differences dm = u - uL and dp = uR - u, formed in FP64 and rounded to R.  ua_left_side: x_L + dt/2 evolution;
// ua_right_side: x_R + dt/2 evolution.
template <class M, int AXIS>
__device__ __forceinline__ void evolve_edges_mixed_d(const typename M::R* dm, const typename M::R* dp, const double* u,
                                                     const MixedConst& k, const typename M::P& q,
                                                     typename M::R* ua_left_side, typename M::R* ua_right_side) {
    using R = typename M::R;
    constexpr int NU = M::NU;
    R xl[NU], xr[NU];
#pragma unroll
    for (int i = 0; i < NU; i++) {
        R hs = half_slope_mixed(dm[i], dp[i], k);
        R uc = (R)u[i];
        xl[i] = uc - hs;
        xr[i] = uc + hs;
    }
    float fl[NU], fr[NU];
    M::template flux<AXIS>(xl, q, fl);
    M::template flux<AXIS>(xr, q, fr);
#pragma unroll
    for (int i = 0; i < NU; i++) {
        R ev = (R)(k.half_r * (fl[i] - fr[i]));
        ua_left_side[i] = xl[i] + ev;
        ua_right_side[i] = xr[i] + ev;
    }
    if constexpr (roundtrip_evolved<M>::value) {
        // the reference stores each evolved state in a state vector (Solvers/solvers.cpp:584-599): for models where
        // that is a projection (the reduced model's clamped volume fraction and mixture density), do the same
        double w[M::NW];
        M::setcons(ua_left_side, q, w);
        M::cons(w, q, ua_left_side);
        M::setcons(ua_right_side, q, w);
        M::cons(w, q, ua_right_side);
    }
}

// evolve_edges_mixed_d from the FP64 conserved vectors of the cell and its neighbours.
template <class M, int AXIS>
__device__ __forceinline__ void evolve_edges_mixed(const double* uL, const double* u, const double* uR,
                                                   const MixedConst& k, const typename M::P& q,
                                                   typename M::R* ua_left_side, typename M::R* ua_right_side) {
    using R = typename M::R;
    R dm[M::NU], dp[M::NU];
#pragma unroll
    for (int i = 0; i < M::NU; i++) {
        dm[i] = (R)(u[i] - uL[i]);
        dp[i] = (R)(uR[i] - u[i]);
    }
    evolve_edges_mixed_d<M, AXIS>(dm, dp, u, k, q, ua_left_side, ua_right_side);
}

// FORCE flux of the evolved states ua (left) and ub (right), FP32 result.
template <class M, int AXIS>
__device__ __forceinline__ void force_flux_mixed(const typename M::R* ua, const typename M::R* ub,
                                                 const MixedConst& k, const typename M::P& q, float* F) {
    using R = typename M::R;
    constexpr int NU = M::NU;
    float fa[NU], fb[NU], fri[NU];
    R uri[NU];
    M::template flux<AXIS>(ua, q, fa);
    M::template flux<AXIS>(ub, q, fb);
#pragma unroll
    for (int i = 0; i < NU; i++) uri[i] = (R)0.5 * (ua[i] + ub[i]) + (R)(0.5f * k.r_f * (fa[i] - fb[i]));
    M::template flux<AXIS>(uri, q, fri);
#pragma unroll
    for (int i = 0; i < NU; i++) {
        float lf = 0.5f * (fa[i] + fb[i]) + 0.5f * k.rinv_f * (float)(ua[i] - ub[i]);
        F[i] = 0.5f * (lf + fri[i]);
    }
}

template <class M>
__device__ __forceinline__ bool bad_state_mixed(const double* W, const typename M::P& q) {
    double rho = M::density(W), p = M::pressure(W);
    if (!pressure_rule<M>::positive(q)) return !(rho > 0.0) || !isfinite(rho) || !isfinite(p);
    return !(rho > 0.0) || !(p > pressure_floor<typename M::P>::of(q)) || !isfinite(rho) || !isfinite(p);
}

// ----------------------------------------------------------------------------------------- X sweep
template <class M, int P, int LPB, int MINB>
__global__ void __launch_bounds__(P* LPB, MINB) sweep_x_mixed_kernel(SweepArgs a) {
    using R = typename M::R;
    constexpr int NU = M::NU, NW = M::NW;
    constexpr int NT = P * LPB;
    __shared__ double Us[NU][LPB][P + 2];
    __shared__ R Es[NU][LPB][P];
    __shared__ double Fs[NU][LPB][P];  // interface fluxes, widened once to FP64 for the update

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

    R ub[NU];
    {
        double uL[NU], u[NU], uR[NU];
        R ua[NU];
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
        R ua[NU];
        float F[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) ua[v] = Es[v][l][p - 1];
        force_flux_mixed<M, 0>(ua, ub, k, q, F);
#pragma unroll
        for (int v = 0; v < NU; v++) Fs[v][l][p] = (double)F[v];
    }
    __syncthreads();

    double wave = 0.0;
    if (out_ok) {
        double Un[NU], W[NW];
#pragma unroll
        for (int v = 0; v < NU; v++)
            Un[v] = fma(k.r, Fs[v][l][p] - Fs[v][l][p + 1], Us[v][l][p + 1]);
        keep_fields<M>(a, rowbase + cell, q, W);
        M::setcons(Un, q, W);
#pragma unroll
        for (int v = 0; v < NW; v++) a.out[v * a.plane + rowbase + cell] = W[v];
        if (bad_state_mixed<M>(W, q)) atomicOr(a.err, ERR_STATE);
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
template <class M, int TX, int TY, int MINB>
__global__ void __launch_bounds__(TX, MINB) sweep_y_mixed_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW;
    const int col = blockIdx.x * TX + threadIdx.x;
    const bool col_ok = col < a.nx;
    const int len = a.ny;
    const int ty = a.ty_rows > 0 ? a.ty_rows : TY;
    const int r0 = blockIdx.y * ty;
    const int r1 = min(r0 + ty, len);
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

    auto load = [&](int r, double* W) {
        int rr = ghost_index(r, len, a.periodic);
#pragma unroll
        for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + (long)rr * a.pitch + c];
    };

    using R = typename M::R;
    double um1[NU], u0[NU], up1[NU], wnext[NW];
    float f_prev[NU];  // FP32 interface flux, widened exactly at its use
    R ua_prev[NU], dummy[NU];
    double wave = 0.0;
    load(r0 - 2, wnext);
    M::cons(wnext, q, up1);
    load(r0 - 1, wnext);
    M::cons(wnext, q, um1);
    load(r0, wnext);
    M::cons(wnext, q, u0);
    load(r0 + 1, wnext);  // prefetched one row ahead of its use
    // slope differences: the lower one of a row is the upper one of the row before, carried down the march
    R dlo[NU], dhi[NU];
#pragma unroll
    for (int v = 0; v < NU; v++) {
        dlo[v] = (R)(um1[v] - up1[v]);  // up1 holds row r0 - 2 here
        dhi[v] = (R)(u0[v] - um1[v]);
    }
    evolve_edges_mixed_d<M, 1>(dlo, dhi, um1, k, q, dummy, ua_prev);
#pragma unroll
    for (int v = 0; v < NU; v++) dlo[v] = dhi[v];
    for (int r = r0; r <= r1; r++) {
        M::cons(wnext, q, up1);
        if (r < r1) load(r + 2, wnext);
#pragma unroll
        for (int v = 0; v < NU; v++) dhi[v] = (R)(up1[v] - u0[v]);
        R ub[NU], ua_next[NU];
        evolve_edges_mixed_d<M, 1>(dlo, dhi, u0, k, q, ub, ua_next);
        float F[NU];
        force_flux_mixed<M, 1>(ua_prev, ub, k, q, F);
        if (r > r0 && col_ok) {
            double Un[NU], W[NW];
#pragma unroll
            for (int v = 0; v < NU; v++) Un[v] = fma(k.r, (double)f_prev[v] - (double)F[v], um1[v]);
            keep_fields<M>(a, (long)(r - 1) * a.pitch + c, q, W);
            M::setcons(Un, q, W);
#pragma unroll
            for (int v = 0; v < NW; v++) a.out[v * a.plane + (long)(r - 1) * a.pitch + c] = W[v];
            if (bad_state_mixed<M>(W, q)) atomicOr(a.err, ERR_STATE);
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
            dlo[v] = dhi[v];
        }
    }
    if (a.accumulate_wave) block_max_to<TX>(wave, a.wave_acc);
    if (a.advance_time && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        a.ctrl->t += a.ctrl->dt;
        a.ctrl->it += 1;
    }
}

// ------------------------------------------------------------------------------ X sweep, two rows per thread
// Models with PAIR_X (FP32 reconstruction) run the X sweep with each thread carrying the same column of two
// adjacent rows.  Every stencil neighbour of the sweep lies along x, so the two rows never exchange data and all
// FP32 arithmetic runs as packed two-lane instructions (lane x = the even row); the FP64 parts (conserved
// variables, slope differences, update, primitive recovery) stay scalar per row.  The per-cell operations are
// those of evolve_edges_mixed / force_flux_mixed with R = float.

__device__ __forceinline__ f2 half_slope2(f2 dm, f2 dp, const MixedConst& k) {
    const f2 fl = splat2(k.floor5_f);
    const f2 num = sel2(fabsf(dm.v.x) < k.floor5_f, fabsf(dm.v.y) < k.floor5_f, fl, dm);
    const f2 den = sel2(fabsf(dp.v.x) < k.floor5_f, fabsf(dp.v.y) < k.floor5_f, fl, dp);
    const f2 base = fma2(splat2(k.cm_f), dm, splat2(k.cp_f) * dp);
    if (!k.one_rcp) {
        const f2 r = num * rcp2(den);
        return splat2(0.5f) * base *
               mk2(limiter_approx(r.v.x, k.bias_f, k.limiter), limiter_approx(r.v.y, k.bias_f, k.limiter));
    }
    const f2 t = (num - den) * den;
    const bool gx = t.v.x >= 0.0f, gy = t.v.y >= 0.0f;
    const f2 q = fma2(splat2(1.0f + k.bias_f), num, splat2(1.0f - k.bias_f) * den);
    const f2 f = sel2(gx, gy, den, num) * rcp2(sel2(gx, gy, q, den));
    f2 half_xi;
    if (k.limiter == 0) {
        const f2 t2 = fma2(splat2(-0.5f), den, num) * den;
        half_xi = sel2(gx || t2.v.x < 0.0f, gy || t2.v.y < 0.0f, f, splat2(0.5f));
    } else {
        half_xi = sel2(gx, gy, f, splat2(0.5f) * f);
    }
    const f2 nd = num * den;
    return sel2(nd.v.x < 0.0f, nd.v.y < 0.0f, splat2(0.0f), base * half_xi);
}

// evolve_edges_mixed for two lanes: get(i, o) returns component i of the FP64 conserved vector of the left
// neighbour (o = 0), the cell (1) and the right neighbour (2), one lane each in the double2's x and y.  Same
// operations as the inline stages of sweep_x_pair_kernel (used by the TMA-staged sweep, whose shared tiles keep the
// two rows apart).
template <class M, int AXIS, class Get>
__device__ __forceinline__ void evolve_edges_pair(Get get, const MixedConst& k, const typename M::P& q,
                                                  f2* ua_left_side, f2* ua_right_side) {
    constexpr int NU = M::NU;
    f2 xl[NU], xr[NU], fl[NU], fr[NU];
#pragma unroll
    for (int i = 0; i < NU; i++) {
        const double2 L = get(i, 0), C = get(i, 1), R = get(i, 2);
        const f2 hs = half_slope2(mk2((float)(C.x - L.x), (float)(C.y - L.y)),
                                  mk2((float)(R.x - C.x), (float)(R.y - C.y)), k);
        const f2 uc = mk2((float)C.x, (float)C.y);
        xl[i] = uc - hs;
        xr[i] = uc + hs;
    }
    M::template flux2<AXIS>(xl, q, fl);
    M::template flux2<AXIS>(xr, q, fr);
#pragma unroll
    for (int i = 0; i < NU; i++) {
        const f2 ev = splat2(k.half_r) * (fl[i] - fr[i]);
        ua_left_side[i] = xl[i] + ev;
        ua_right_side[i] = xr[i] + ev;
    }
}

// force_flux_mixed for two lanes
template <class M, int AXIS>
__device__ __forceinline__ void force_flux_pair(const f2* ua, const f2* ub, const MixedConst& k,
                                                const typename M::P& q, f2* F) {
    constexpr int NU = M::NU;
    f2 fa[NU], fb[NU], uri[NU], fri[NU];
    M::template flux2<AXIS>(ua, q, fa);
    M::template flux2<AXIS>(ub, q, fb);
#pragma unroll
    for (int i = 0; i < NU; i++) uri[i] = fma2(splat2(0.5f), ua[i] + ub[i], splat2(0.5f * k.r_f) * (fa[i] - fb[i]));
    M::template flux2<AXIS>(uri, q, fri);
#pragma unroll
    for (int i = 0; i < NU; i++) {
        const f2 lf = fma2(splat2(0.5f), fa[i] + fb[i], splat2(0.5f * k.rinv_f) * (ua[i] - ub[i]));
        F[i] = splat2(0.5f) * (lf + fri[i]);
    }
}

template <class M, int P, int LPB, int MINB>
__global__ void __launch_bounds__(P* LPB, MINB) sweep_x_pair_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW;
    constexpr int NT = P * LPB;
    __shared__ double2 Us[NU][LPB][P + 2];
    __shared__ float2 Es[NU][LPB][P];
    __shared__ double2 Fs[NU][LPB][P];  // interface fluxes, widened once to FP64 for the update

    const int p = threadIdx.x % P, l = threadIdx.x / P;
    const int row0 = (blockIdx.y * LPB + l) * 2;
    const int len = a.nx;
    const int s0 = blockIdx.x * (P - 2);
    const int cell = s0 - 1 + p;
    const bool ok0 = row0 < a.ny, ok1 = row0 + 1 < a.ny;
    const bool col_ok = p >= 1 && p <= P - 2 && cell < len;
    // a missing second row (odd ny) repeats the first; it is computed but never stored
    const long base[2] = {(long)(ok0 ? row0 : 0) * a.pitch, (long)(ok1 ? row0 + 1 : (ok0 ? row0 : 0)) * a.pitch};

    if (a.ctrl && !a.ctrl->active) {
        if (col_ok)
            for (int h = 0; h < (ok1 ? 2 : ok0 ? 1 : 0); h++)
                for (int v = 0; v < NW; v++) a.out[v * a.plane + base[h] + cell] = a.in[v * a.plane + base[h] + cell];
        return;
    }
    double ts;
    const MixedConst k = mixed_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);

    auto conserve = [&](int slot) {
        int c = ghost_index(s0 - 2 + slot, len, a.periodic);
        double W0[NW], W1[NW], U0[NU], U1[NU];
#pragma unroll
        for (int v = 0; v < NW; v++) {
            W0[v] = a.in[v * a.plane + base[0] + c];
            W1[v] = a.in[v * a.plane + base[1] + c];
        }
        M::cons(W0, q, U0);
        M::cons(W1, q, U1);
#pragma unroll
        for (int v = 0; v < NU; v++) Us[v][l][slot] = make_double2(U0[v], U1[v]);
    };
    conserve(p + 1);
    if (p == 0) conserve(0);
    if (p == P - 1) conserve(P + 1);
    __syncthreads();

    f2 ub[NU];
    {
        f2 xl[NU], xr[NU], fl[NU], fr[NU];
#pragma unroll
        for (int i = 0; i < NU; i++) {
            const double2 L = Us[i][l][p], C = Us[i][l][p + 1], R = Us[i][l][p + 2];
            const f2 hs = half_slope2(mk2((float)(C.x - L.x), (float)(C.y - L.y)),
                                      mk2((float)(R.x - C.x), (float)(R.y - C.y)), k);
            const f2 uc = mk2((float)C.x, (float)C.y);
            xl[i] = uc - hs;
            xr[i] = uc + hs;
        }
        M::template flux2<0>(xl, q, fl);
        M::template flux2<0>(xr, q, fr);
#pragma unroll
        for (int i = 0; i < NU; i++) {
            const f2 ev = splat2(k.half_r) * (fl[i] - fr[i]);
            ub[i] = xl[i] + ev;
            Es[i][l][p] = (xr[i] + ev).v;
        }
    }
    __syncthreads();

    if (p >= 1) {
        f2 ua[NU], fa[NU], fb[NU], uri[NU], fri[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) ua[v].v = Es[v][l][p - 1];
        M::template flux2<0>(ua, q, fa);
        M::template flux2<0>(ub, q, fb);
#pragma unroll
        for (int i = 0; i < NU; i++)
            uri[i] = fma2(splat2(0.5f), ua[i] + ub[i], splat2(0.5f * k.r_f) * (fa[i] - fb[i]));
        M::template flux2<0>(uri, q, fri);
#pragma unroll
        for (int i = 0; i < NU; i++) {
            const f2 lf = fma2(splat2(0.5f), fa[i] + fb[i], splat2(0.5f * k.rinv_f) * (ua[i] - ub[i]));
            const f2 F = splat2(0.5f) * (lf + fri[i]);
            Fs[i][l][p] = make_double2((double)F.v.x, (double)F.v.y);
        }
    }
    __syncthreads();

    double wave = 0.0;
    if (col_ok) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (!(h == 0 ? ok0 : ok1)) continue;
            double Un[NU], W[NW];
#pragma unroll
            for (int v = 0; v < NU; v++) {
                const double2 fl = Fs[v][l][p], fr = Fs[v][l][p + 1], c = Us[v][l][p + 1];
                Un[v] = h == 0 ? fma(k.r, fl.x - fr.x, c.x) : fma(k.r, fl.y - fr.y, c.y);
            }
            keep_fields<M>(a, base[h] + cell, q, W);
            M::setcons(Un, q, W);
#pragma unroll
            for (int v = 0; v < NW; v++) a.out[v * a.plane + base[h] + cell] = W[v];
            if (bad_state_mixed<M>(W, q)) atomicOr(a.err, ERR_STATE);
            if (a.accumulate_wave) {
                double s = M::wave(W, q, a.dims);
                if (s > wave) wave = s;
            }
        }
    }
    if (a.accumulate_wave) block_max_to<NT>(wave, a.wave_acc);
    if (a.advance_time && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        a.ctrl->t += a.ctrl->dt;
        a.ctrl->it += 1;
    }
}

}  // namespace vg
