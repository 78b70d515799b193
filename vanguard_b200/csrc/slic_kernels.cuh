// SLIC sweep kernels, generic over a model policy M (see physics_fp64.cuh).
//
// One sweep updates every cell once: U_i <- U_i + (dt/dx)(F_{i-1/2} - F_{i+1/2}) with the SLIC interface
// flux F = FORCE(evolve(L-side of right cell), evolve(R-side of left cell)).  The reference evaluates each
// interface flux twice (once per neighbour, Solvers/secondordersolver.cpp:146-161) and the half-step
// evolved edge states four times; here every cell's conserved vector, every evolved edge state and every
// interface flux is computed exactly once per sweep (plus a 1-3 % halo) -- the values are pure functions
// of the same inputs, so the result is unchanged.
//
// X sweep (along the contiguous column index): a block owns LPB row segments of P cells; the stages
// (conserve -> evolve edges -> FORCE -> update) exchange neighbours through shared memory.
// Y sweep (along rows): each thread owns one column and marches down a segment of TY rows keeping a
// sliding window of the stencil in registers; a warp reads 32 consecutive doubles per plane-row.
#pragma once

#include <utility>

#include "vg_common.cuh"

namespace vg {

// SlopeLimiters::computeSlopeLimiter (Solvers/slopelimiters.cpp:7-74)
__device__ __forceinline__ double limiter_f64(double r, double w, int id) {
    if (id == 0) {
        if (r < 0.0) return 0.0;
        if (r < 0.5) return 2.0 * r;
        if (r < 1.0) return 1.0;
        return std_min(std_min(r, 2.0 / ((1.0 - w) + ((1.0 + w) * r))), 2.0);
    } else if (id == 1) {
        if (r < 0.0) return 0.0;
        return std_min((2.0 * r) / (1.0 + r), 2.0 / ((1.0 - w) + ((1.0 + w) * r)));
    }
    if (r < 0.0) return 0.0;
    if (r < 1.0) return r;
    return std_min(1.0, 2.0 / ((1.0 - w) + ((1.0 + w) * r)));
}

// One component of SlopeLimiters::computeSlopeVector (Solvers/slopelimiters.cpp:217-246).
__device__ __forceinline__ double slope_f64(double uL, double u, double uR, const SweepConst& k) {
    double dm = u - uL;
    double dp = uR - u;
    double s = (k.cm * dm) + (k.cp * dp);
    double num = dm, den = dp;
    if (fabs(num) < k.floor5) num = k.floor5;
    if (fabs(den) < k.floor5) den = k.floor5;
    return s * limiter_f64(num / den, k.bias, k.limiter);
}

// Solvers::evolveStateByHalf{X,Y}TimeStep for both sides of one cell (Solvers/solvers.cpp:454-466,
// :502-514, :550-565): returns the conserved vectors of the two evolved edge states after the reference's
// primitive round trip (setConservedVariableVector then computeConservedVariableVector).
template <class M, int AXIS>
__device__ __forceinline__ void evolve_edges(const double* uL, const double* u, const double* uR, const SweepConst& k,
                                             const typename M::P& q, double* ua_left_side, double* ua_right_side,
                                             bool want_left, bool want_right) {
    constexpr int NU = M::NU;
    double xl[NU], xr[NU], fl[NU], fr[NU];
#pragma unroll
    for (int i = 0; i < NU; i++) {
        double s = slope_f64(uL[i], u[i], uR[i], k);
        xl[i] = u[i] - (0.5 * s);
        xr[i] = u[i] + (0.5 * s);
    }
    M::template flux<AXIS>(xl, q, fl);
    M::template flux<AXIS>(xr, q, fr);
    double a[NU], b[NU];
#pragma unroll
    for (int i = 0; i < NU; i++) {
        double ev = k.half_r * (fl[i] - fr[i]);
        a[i] = xl[i] + ev;
        b[i] = xr[i] + ev;
    }
    double w[M::NW];
    if (want_left) {
        M::setcons(a, q, w);
        M::cons(w, q, ua_left_side);
    }
    if (want_right) {
        M::setcons(b, q, w);
        M::cons(w, q, ua_right_side);
    }
}

// FirstOrderSolver::compute{X,Y}FORCEFlux (Solvers/firstordersolver.cpp:173-230) on the conserved vectors
// of the left state ua and right state ub.
template <class M, int AXIS>
__device__ __forceinline__ void force_flux(const double* ua, const double* ub, const SweepConst& k,
                                           const typename M::P& q, double* F) {
    constexpr int NU = M::NU;
    double fa[NU], fb[NU], uri[NU], fri[NU];
    M::template flux<AXIS>(ua, q, fa);
    M::template flux<AXIS>(ub, q, fb);
#pragma unroll
    for (int i = 0; i < NU; i++) uri[i] = 0.5 * ((ua[i] + ub[i]) + (k.r * (fa[i] - fb[i])));
    M::template flux<AXIS>(uri, q, fri);
#pragma unroll
    for (int i = 0; i < NU; i++) {
        double lf = 0.5 * ((fa[i] + fb[i]) + (k.rinv * (ua[i] - ub[i])));
        F[i] = 0.5 * (lf + fri[i]);
    }
}

__device__ __forceinline__ SweepConst sweep_const(const SweepArgs& a, double& ts) {
    SweepConst k;
    if (a.ctrl) {
        ts = a.ctrl->dt * a.dt_scale;
        k.r = a.ctrl->kr[a.kslot];
        k.rinv = a.ctrl->krinv[a.kslot];
        k.half_r = a.ctrl->khalf_r[a.kslot];
    } else {
        ts = a.dt_host * a.dt_scale;
        k.r = a.r_host;
        k.rinv = a.rinv_host;
        k.half_r = a.half_r_host;
    }
    k.cm = 0.5 * (1.0 + a.bias);
    k.cp = 0.5 * (1.0 - a.bias);
    k.bias = a.bias;
    k.floor5 = a.floor5;
    k.limiter = a.limiter;
    return k;
}

template <class M>
__device__ __forceinline__ void load_w(const SweepArgs& a, long idx, double* W) {
#pragma unroll
    for (int v = 0; v < M::NW; v++) W[v] = a.in[v * a.plane + idx];
}

template <class M>
__device__ __forceinline__ void store_w(const SweepArgs& a, long idx, const double* W) {
#pragma unroll
    for (int v = 0; v < M::NW; v++) a.out[v * a.plane + idx] = W[v];
}

// Fields setConservedVariableVector leaves alone keep the cell's own values, as when the reference updates the
// cell object in place (Solvers/firstordersolver.cpp:428-433): HPR's J (planes 14-16) when the material is not
// thermal (HPR/hprstatevector.cpp:78-103), and the HPR two-material models' J when neither material is (planes 14-16
// of the reduced model, HPR/Multiphysics/hprreducedstatevector.cpp:111-152; 13-15 of the intermediate model,
// hprintermediatestatevector.cpp:112-159).  Models with heat flux name its first plane in J_PLANE; a model whose
// materials keep their heat fluxes separately (the HPR multiphysics model) has its own keep_cold.
template <class M, class = void>
struct heat_flux_plane {
    static constexpr int value = -1;
};
template <class M>
struct heat_flux_plane<M, decltype((void)M::J_PLANE)> {
    static constexpr int value = M::J_PLANE;
};
template <class M, class = void>
struct cold_fields {
    __device__ static void keep(const SweepArgs& a, long idx, const typename M::P& q, double* W) {
        constexpr int j0 = heat_flux_plane<M>::value;
        if constexpr (j0 >= 0) {
            if (!q.thermal)
                for (int v = j0; v < j0 + 3; v++) W[v] = a.in[v * a.plane + idx];
        }
    }
};
template <class M>
struct cold_fields<M, decltype((void)&M::keep_cold)> {
    __device__ static void keep(const SweepArgs& a, long idx, const typename M::P& q, double* W) {
        M::keep_cold(a, idx, q, W);
    }
};
template <class M>
__device__ __forceinline__ void keep_fields(const SweepArgs& a, long idx, const typename M::P& q, double* W) {
    cold_fields<M>::keep(a, idx, q, W);
}

// Whether a state of model M must have a positive pressure: models with a positive_pressure(q) member decide
// (HPR: only its gas equation of state); every other model requires it.
template <class M, class = void>
struct pressure_rule {
    __device__ static bool positive(const typename M::P&) { return true; }
};
template <class M>
struct pressure_rule<M, decltype((void)&M::positive_pressure)> {
    __device__ static bool positive(const typename M::P& q) { return M::positive_pressure(q); }
};

// The pressure at or below which a state has no real sound speed: -p_inf for the stiffened-gas models whose
// parameters carry p_inf (c^2 = gamma (p + p_inf) / rho, Euler/eulerequationofstate.cpp:23-29), 0 for the others.
template <class P, class = void>
struct pressure_floor {
    __device__ static double of(const P&) { return 0.0; }
};
template <class P>
struct pressure_floor<P, decltype((void)std::declval<P>().pinf)> {
    __device__ static double of(const P& q) { return -q.pinf; }
};

template <class M>
__device__ __forceinline__ bool bad_state(const double* W, const typename M::P& q) {
    double rho = M::density(W), p = M::pressure(W);
    if (!pressure_rule<M>::positive(q)) return !(rho > 0.0) || !isfinite(rho) || !isfinite(p);
    return !(rho > 0.0) || !(p > pressure_floor<typename M::P>::of(q)) || !isfinite(rho) || !isfinite(p);
}

// ----------------------------------------------------------------------------------------- X sweep
template <class M, int P, int LPB, int MINB>
__global__ void __launch_bounds__(P* LPB, MINB) sweep_x_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW;
    constexpr int NT = P * LPB;
    __shared__ double Us[NU][LPB][P + 2];
    __shared__ double Es[NU][LPB][P];
    __shared__ double Fs[NU][LPB][P];

    const int p = threadIdx.x % P, l = threadIdx.x / P;
    const int row = blockIdx.y * LPB + l;
    const int len = a.nx;
    const int s0 = blockIdx.x * (P - 2);           // first output cell of this segment
    const int cell = s0 - 1 + p;                   // cell owned by this thread (halo at p = 0, P-1)
    const bool row_ok = row < a.ny;
    const bool out_ok = row_ok && p >= 1 && p <= P - 2 && cell < len;
    const long rowbase = (long)(row_ok ? row : 0) * a.pitch;

    if (a.ctrl && !a.ctrl->active) {               // step past the end: carry the state over unchanged
        if (out_ok)
            for (int v = 0; v < NW; v++) a.out[v * a.plane + rowbase + cell] = a.in[v * a.plane + rowbase + cell];
        return;
    }
    double ts;
    const SweepConst k = sweep_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);

    // stage 1: conserved vectors of cells s0-2 .. s0+P-1 (slot = cell - s0 + 2)
    auto conserve = [&](int slot) {
        int c = ghost_index(s0 - 2 + slot, len, a.periodic);
        double W[NW], U[NU];
        load_w<M>(a, rowbase + c, W);
        M::cons(W, q, U);
#pragma unroll
        for (int v = 0; v < NU; v++) Us[v][l][slot] = U[v];
    };
    conserve(p + 1);
    if (p == 0) conserve(0);
    if (p == P - 1) conserve(P + 1);
    __syncthreads();

    // stage 2: evolved edge states of the owned cell
    double ub[NU];  // conserved left-side edge state of the owned cell (right state of interface cell-1/2)
    {
        double uL[NU], u[NU], uR[NU], ua[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) {
            uL[v] = Us[v][l][p];
            u[v] = Us[v][l][p + 1];
            uR[v] = Us[v][l][p + 2];
        }
        evolve_edges<M, 0>(uL, u, uR, k, q, ub, ua, p >= 1, p <= P - 2);
#pragma unroll
        for (int v = 0; v < NU; v++) Es[v][l][p] = ua[v];
    }
    __syncthreads();

    // stage 3: FORCE flux at the interface left of the owned cell
    if (p >= 1) {
        double ua[NU], F[NU];
#pragma unroll
        for (int v = 0; v < NU; v++) ua[v] = Es[v][l][p - 1];
        force_flux<M, 0>(ua, ub, k, q, F);
#pragma unroll
        for (int v = 0; v < NU; v++) Fs[v][l][p] = F[v];
    }
    __syncthreads();

    // stage 4: conservative update (FirstOrderSolver::computeFORCEUpdate, Solvers/firstordersolver.cpp:428-433)
    double wave = 0.0;
    if (out_ok) {
        double Un[NU], W[NW];
#pragma unroll
        for (int v = 0; v < NU; v++) Un[v] = Us[v][l][p + 1] + (k.r * (Fs[v][l][p] - Fs[v][l][p + 1]));
        keep_fields<M>(a, rowbase + cell, q, W);
        M::setcons(Un, q, W);
        store_w<M>(a, rowbase + cell, W);
        if (bad_state<M>(W, q)) atomicOr(a.err, ERR_STATE);
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
__global__ void __launch_bounds__(TX, MINB) sweep_y_kernel(SweepArgs a) {
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
    const SweepConst k = sweep_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);

    auto conserve = [&](int r, double* U) {
        int rr = ghost_index(r, len, a.periodic);
        double W[NW];
        load_w<M>(a, (long)rr * a.pitch + c, W);
        M::cons(W, q, U);
    };

    double um1[NU], u0[NU], up1[NU], ua_prev[NU], f_prev[NU], dummy[NU];
    double wave = 0.0;
    conserve(r0 - 2, up1);   // temporarily holds row r0-2
    conserve(r0 - 1, um1);
    conserve(r0, u0);
    evolve_edges<M, 1>(up1, um1, u0, k, q, dummy, ua_prev, false, true);   // right edge of row r0-1
    for (int r = r0; r <= r1; r++) {
        conserve(r + 1, up1);
        double ub[NU], ua_next[NU];
        evolve_edges<M, 1>(um1, u0, up1, k, q, ub, ua_next, true, r < r1);
        double F[NU];
        force_flux<M, 1>(ua_prev, ub, k, q, F);     // flux at r - 1/2
        if (r > r0 && col_ok) {                      // update row r-1 with fluxes at r-3/2 and r-1/2
            double Un[NU], W[NW];
#pragma unroll
            for (int v = 0; v < NU; v++) Un[v] = um1[v] + (k.r * (f_prev[v] - F[v]));
            keep_fields<M>(a, (long)(r - 1) * a.pitch + c, q, W);
            M::setcons(Un, q, W);
            store_w<M>(a, (long)(r - 1) * a.pitch + c, W);
            if (bad_state<M>(W, q)) atomicOr(a.err, ERR_STATE);
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

// ------------------------------------------------------------------------------- CFL and time step
// Maximum wave speed of the current state into ctrl->smax_next (grid-stride, block reduce, one atomic per
// block; the maximum of exact values does not depend on the order, unlike the reference's racy OpenMP max).
template <class M, int NT>
__global__ void __launch_bounds__(NT) max_wave_kernel(const double* __restrict__ in, long plane, long pitch, int nx, int ny,
                                                      Ctrl* ctrl, SweepArgs a) {
    const typename M::P q = M::params(a.params, 0.0);
    double best = 0.0;
    long n = (long)nx * ny;
    for (long i = blockIdx.x * (long)NT + threadIdx.x; i < n; i += (long)gridDim.x * NT) {
        long r = i / nx, cidx = i - r * nx;
        double W[M::NW];
#pragma unroll
        for (int v = 0; v < M::NW; v++) W[v] = in[v * plane + r * pitch + cidx];
        double s = M::wave(W, q, a.dims);
        if (s > best) best = s;
    }
    block_max_to<NT>(best, &ctrl->smax_next);
}

// Solvers::computeStableTimeStep{,2D} (Solvers/solvers.cpp:388-452): dt = CFL * (dx / S), x0.2 for the first six
// steps, clamped to t_end.  In 2D S also covers the default-constructed corner ghosts of insertBoundaryCells2D
// (Solvers/solvers.cpp:92).  For MHD, c_h = S for this step (Solvers/mhdsecondordersolver.cpp:513-515).
template <class M>
__global__ void step_begin_kernel(Ctrl* c, SweepArgs a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int it = c->it;
    int active = (c->t < c->t_end) && (it < c->max_steps);
    c->active = active;
    double S = __longlong_as_double((long long)c->smax_next);
    if (c->dims == 2) {
        double W[M::NW];
        M::default_state(W);
        const typename M::P q = M::params(a.params, 0.0);
        double sd = M::wave(W, q, 2);
        if (sd > S) S = sd;
    }
    if (active) {
        double dt = c->cfl * (c->dx / S);
        if (it <= 5) dt *= 0.2;
        if ((c->t + dt) > c->t_end) dt = c->t_end - c->t;
        c->dt = dt;
        c->ch = a.ch_fixed ? a.ch_host : S;
        for (int i = 0; i < 2; i++) {
            sweep_scale(dt * (i == 0 ? 0.5 : 1.0), c->dx, c->kr[i], c->krinv[i], c->khalf_r[i]);
            c->kr_f[i] = (float)c->kr[i];
            c->krinv_f[i] = (float)c->krinv[i];
            c->khalf_r_f[i] = (float)c->khalf_r[i];
        }
    }
    c->smax_next = 0ull;
}

// Copy of the host-visible result of vg_max_wave_speed: S including corner ghosts.
template <class M>
__global__ void max_wave_finish_kernel(Ctrl* c, SweepArgs a, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double S = __longlong_as_double((long long)c->smax_next);
    if (c->dims == 2) {
        double W[M::NW];
        M::default_state(W);
        const typename M::P q = M::params(a.params, 0.0);
        double sd = M::wave(W, q, 2);
        if (sd > S) S = sd;
    }
    *out = S;
}

}  // namespace vg
