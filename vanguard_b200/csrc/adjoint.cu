// Discrete adjoint of the batched 1D Euler SLIC step, with binomial checkpointing (no counterpart in the
// reference, which has no derivatives).
//
// Loss  L = sum_k sum_i (rho_k,i(T) - target_k,i)^2  after `steps` steps of every instance's own solve() loop.
// Output dL/dW^0 (primitive planes rho, u, p of every cell) and dL/dgamma_k.
//
// One reverse step s maps lambda^{s+1} = dL/dW^{s+1} to lambda^s through the forward step of batch.cu:
//   W^{s+1}_i = setcons(U_i + r (F_{i-1/2} - F_{i+1/2})),  U_i = cons(W^s_i),  r = dt / dx,
//   F_{j+1/2} = FORCE(evolve_R(W_{j-1}, W_j, W_{j+1}), evolve_L(W_j, W_{j+1}, W_{j+2})),
//   dt = CFL dx / S (x0.2 for s <= 5),  S = max_i (|u_i| + c_i).
// Vector-Jacobian products are written by hand for cons / setcons / the x flux (the primitive round trips of the
// reference are identities and drop out), the slope limiter, the half-step evolution, the Lax-Friedrichs /
// Richtmyer / FORCE combination and the update.  Subgradients:
//   * limiter: the derivative of the branch the forward step took (one-sided at r = 0, 1/2, 1 and where the
//     minimum switches between r, xi_R and 2), decided by the forward's own comparisons on bit-equal operands;
//   * the |delta| < 1e-5 floor: zero derivative of the floored ratio operand;
//   * the CFL maximum: only the first cell attaining the maximum receives dS; |u| has derivative sign(u), 0 at 0.
// The dt dependence is propagated (dt -> S -> that cell's state and gamma), so the result is the gradient of the
// scheme that adapts its step, which is what central finite differences measure where the loss is smooth.
//
// Arithmetic: the values that select a branch (cons, the slope ratio and xi_R, the wave speed) are recomputed
// with uncontracted IEEE operations (__dmul_rn & co.) exactly as the forward step forms them, so every branch
// matches it; everything else (edge states, fluxes, the derivative formulas) uses reciprocals refined to full
// double precision and FMA contraction, which moves the gradient by round-off only.
//
// Tiles: AP = 128 positions per block, AH = 5 halo cells each side, AP - 2 AH outputs.  Every contribution to
// r-bar and gamma-bar is owned by exactly one tile (interfaces by their right cell, or the last cell at the right
// end; ghost-cell edges by the instance's end cells), so the per-instance sums are deterministic.  Ghost cells
// (transmissive mirror copies, Solvers/solvers.cpp:17-23) fold their adjoints into the cells they copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/vanguard_slic.h"
#include "batch_internal.cuh"
#include "physics_mixed.cuh"
#include "vg_ops.h"

namespace vg {
namespace {

constexpr int AP = 128;
constexpr int AH = 5;
constexpr int AOUT = AP - 2 * AH;

__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

struct Gas {
    double g, pinf, gm1, igm1, gpinf;
};

// EulerStateVector::computeConservedVariableVector (Euler/eulerstatevector.cpp:78-91), operation for operation
__device__ __forceinline__ void cons_exact(const double* W, const Gas& q, double* U) {
    const double rho = W[0], u = W[1], p = W[2];
    const double e = xdiv(xadd(p, xmul(q.g, q.pinf)), xmul(xsub(q.g, 1.0), rho));
    U[0] = rho;
    U[1] = xmul(rho, u);
    U[2] = xmul(rho, xadd(xmul(0.5, xmul(u, u)), e));
}
// |u| + c of Solvers::computeMaximumWaveSpeed (Solvers/solvers.cpp:259-276), operation for operation
__device__ __forceinline__ double wave_exact(double rho, double u, double p, double g, double pinf) {
    return xadd(fabs(u), __dsqrt_rn(xdiv(xmul(g, xadd(p, pinf)), rho)));
}

// xi(r) of SlopeLimiters::computeSlopeLimiter (Solvers/slopelimiters.cpp:7-74) with the derivative of the branch
// taken; the comparisons see the forward's operands bit for bit (std::min(a, b) = b < a ? b : a).
__device__ __forceinline__ void limiter_d(double r, double w, int id, double& xi, double& dxi) {
    const double xr = xdiv(2.0, xadd(1.0 - w, xmul(1.0 + w, r)));
    const double dxr = -0.5 * (1.0 + w) * xr * xr;  // d(2 / den)/dr = -2 (1 + w) / den^2
    xi = 0.0;
    dxi = 0.0;
    if (r < 0.0) return;
    if (id == 0) {
        if (r < 0.5) {
            xi = xmul(2.0, r);
            dxi = 2.0;
        } else if (r < 1.0) {
            xi = 1.0;
        } else {
            const bool t = xr < r;
            const double m1 = t ? xr : r;
            if (!(2.0 < m1)) {
                xi = m1;
                dxi = t ? dxr : 1.0;
            } else {
                xi = 2.0;
            }
        }
    } else if (id == 1) {
        const double a = xdiv(xmul(2.0, r), xadd(1.0, r));
        if (xr < a) {
            xi = xr;
            dxi = dxr;
        } else {
            const double ip = rcp_nr2(1.0 + r);
            xi = a;
            dxi = 2.0 * ip * ip;
        }
    } else {
        if (r < 1.0) {
            xi = r;
            dxi = 1.0;
        } else if (xr < 1.0) {
            xi = xr;
            dxi = dxr;
        } else {
            xi = 1.0;
        }
    }
}

struct K {
    double r, rinv, half_r, cm, cp, bias, floor5;
    int limiter;
};

// One slope component (SlopeLimiters::computeSlopeVector, Solvers/slopelimiters.cpp:217-246) and its partial
// derivatives with respect to delta- = u - uL and delta+ = uR - u.
__device__ __forceinline__ double slope_d(double uL, double u, double uR, const K& k, double& sdm, double& sdp) {
    const double dm = u - uL, dp = uR - u;
    const bool nf = fabs(dm) < k.floor5, df = fabs(dp) < k.floor5;
    const double num = nf ? k.floor5 : dm, den = df ? k.floor5 : dp;
    const double r = xdiv(num, den);
    double xi, dxi;
    limiter_d(r, k.bias, k.limiter, xi, dxi);
    const double base = k.cm * dm + k.cp * dp;
    const double t = base * dxi * rcp_nr2(den);  // base * dxi * dr/dnum
    sdm = k.cm * xi + (nf ? 0.0 : t);
    sdp = k.cp * xi - (df ? 0.0 : t * r);  // dr/dden = -r / den
    return base * xi;
}

// x flux of a conserved state with 1/rho kept for the vector-Jacobian product
__device__ __forceinline__ void flux_a(const double* U, const Gas& q, double* F, double& ir) {
    ir = rcp_nr2(U[0]);
    const double u = U[1] * ir;
    const double p = q.gm1 * (U[2] - 0.5 * U[1] * u) - q.gpinf;
    F[0] = U[1];
    F[1] = U[1] * u + p;
    F[2] = u * (U[2] + p);
}
// Ub += (dF/dU)^T Fb, gb += (dF/dgamma) . Fb, for F = (m, m u + p, u (E + p)), u = m / rho,
// p = (gamma - 1)(E - m u / 2) - gamma p_inf
__device__ __forceinline__ void flux_vjp(const double* U, double ir, const Gas& q, const double* Fb, double* Ub,
                                         double& gb) {
    const double u = U[1] * ir;
    const double X = U[2] - 0.5 * U[1] * u;
    const double p = q.gm1 * X - q.gpinf;
    const double ub = U[1] * Fb[1] + (U[2] + p) * Fb[2];
    const double pb = Fb[1] + u * Fb[2];
    Ub[0] += q.gm1 * 0.5 * u * u * pb - u * ir * ub;
    Ub[1] += Fb[0] + u * Fb[1] + ir * ub - q.gm1 * u * pb;
    Ub[2] += u * Fb[2] + q.gm1 * pb;
    gb += (X - q.pinf) * pb;
}

struct AdjArgs {
    const double* W;        // state W^s (rho, u, p planes)
    const double* lam_in;   // dL/dW^{s+1}
    double* lam_out;        // dL/dW^s (cells owned by the tiles)
    long plane;
    const long* offset;
    const int* ncell;
    const double* dx;
    const double* gam;
    const Tile* tiles;      // adjoint tiles: AOUT outputs each
    int ntiles;
    const unsigned long long* S;  // max |u| + c of W^s per instance (double bit patterns)
    int* arg;               // first cell attaining S per instance (atomicMin; reset by the dt adjoint kernel)
    double* tile_part;      // per tile: r-bar (dL/dr) and gamma-bar
    double cfl, bias, floor5;
    int limiter;
    int step;               // s
};

// dt of step s from S, operation for operation as the forward step forms it (Solvers/solvers.cpp:437-452)
__device__ __forceinline__ double step_dt(double cfl, double dx, double S, int s) {
    double d = xmul(cfl, xdiv(dx, S));
    if (s <= 5) d = xmul(d, 0.2);
    return d;
}

__global__ void __launch_bounds__(AP, 4) adjoint_step_kernel(AdjArgs a) {
    // stage-aliased shared arrays: Us -> UL, Ea -> AB, Eb -> BB, Fs -> US
    __shared__ double S0[3][AP], S1[3][AP], S2[3][AP], S3[3][AP], MU[3][AP], UR[3][AP];
    __shared__ double red[2][AP / 32];
    __shared__ double tile_k[4];  // dt/dx, dx/dt, 1/(gamma - 1) of the tile's instance, formed by one thread
    auto& Us = S0;
    auto& UL = S0;
    auto& Ea = S1;
    auto& AB = S1;
    auto& Eb = S2;
    auto& BB = S2;
    auto& Fs = S3;
    auto& US = S3;
    const int p = threadIdx.x;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int k = tile.inst, n = a.ncell[k], s0 = tile.s0;
        const long base = a.offset[k];
        const int c = s0 - AH + p;  // cell of this position (may be a ghost or beyond)
        const bool real = c >= 0 && c < n;
        const bool out = p >= AH && p < AP - AH && real;
        const bool owns_first = s0 == 0;                          // tile owning cell 0
        const bool owns_last = s0 <= n - 1 && n - 1 < s0 + AOUT;  // tile owning cell n-1
        const double dxk = a.dx[k];
        const double Sk = __longlong_as_double((long long)a.S[k]);
        if (p == 0) {
            const double dt = step_dt(a.cfl, dxk, Sk, a.step);
            tile_k[0] = xdiv(dt, dxk);
            tile_k[1] = dxk / dt;
            tile_k[2] = 1.0 / (a.gam[2 * k] - 1.0);
        }
        K kc;
        kc.cm = 0.5 * (1.0 + a.bias);
        kc.cp = 0.5 * (1.0 - a.bias);
        kc.bias = a.bias;
        kc.floor5 = a.floor5;
        kc.limiter = a.limiter;
        Gas q;
        q.g = a.gam[2 * k];
        q.pinf = a.gam[2 * k + 1];
        q.gm1 = q.g - 1.0;
        q.gpinf = q.g * q.pinf;
        // stage A: conserved vectors of every position (ghosts by the transmissive mirror); the adjoint input of
        // the cells reverse 1 needs is loaded here so its latency hides behind stages B and C
        double W[3], lam[3] = {0.0, 0.0, 0.0};
        const bool upd = p >= 2 && p < AP - 2 && real;
        {
            const int gi = ghost_index(c, n, 0);
            for (int v = 0; v < 3; v++) W[v] = a.W[v * a.plane + base + gi];
            if (upd)
                for (int v = 0; v < 3; v++) lam[v] = a.lam_in[v * a.plane + base + c];
            double U[3];
            cons_exact(W, q, U);
            for (int v = 0; v < 3; v++) Us[v][p] = U[v];
        }
        // first cell of the instance attaining S (the CFL maximum's argmax)
        {
            const unsigned hit = (out && wave_exact(W[0], W[1], W[2], q.g, q.pinf) == Sk) ? (unsigned)c : 0xffffffffu;
            const unsigned m = __reduce_min_sync(0xffffffffu, hit);
            if ((p & 31) == 0 && m != 0xffffffffu) atomicMin(&a.arg[k], (int)m);
        }
        __syncthreads();
        kc.r = tile_k[0];
        kc.rinv = tile_k[1];
        kc.half_r = 0.5 * kc.r;
        q.igm1 = tile_k[2];
        // stage B: slopes (with their derivatives) and the evolved edge states of positions [1, AP-1)
        double xl[3], xr[3], dF[3], sdm[3], sdp[3], irl = 1.0, irr = 1.0;
        if (p >= 1 && p < AP - 1) {
            for (int v = 0; v < 3; v++) {
                const double u = Us[v][p];
                const double s = slope_d(Us[v][p - 1], u, Us[v][p + 1], kc, sdm[v], sdp[v]);
                xl[v] = u - 0.5 * s;
                xr[v] = u + 0.5 * s;
            }
            double fl[3], fr[3];
            flux_a(xl, q, fl, irl);
            flux_a(xr, q, fr, irr);
            for (int v = 0; v < 3; v++) {
                dF[v] = fl[v] - fr[v];
                const double ev = kc.half_r * dF[v];
                Ea[v][p] = xl[v] + ev;
                Eb[v][p] = xr[v] + ev;
            }
        }
        __syncthreads();
        // stage C: FORCE flux at the interface left of positions [2, AP-1)
        double ua[3], ub[3], uri[3], dfab[3], ira = 1.0, irb = 1.0, iri = 1.0;
        if (p >= 2 && p < AP - 1) {
            double fa[3], fb[3], fri[3];
            for (int v = 0; v < 3; v++) {
                ua[v] = Eb[v][p - 1];
                ub[v] = Ea[v][p];
            }
            flux_a(ua, q, fa, ira);
            flux_a(ub, q, fb, irb);
            for (int v = 0; v < 3; v++) {
                dfab[v] = fa[v] - fb[v];
                uri[v] = 0.5 * ((ua[v] + ub[v]) + kc.r * dfab[v]);
            }
            flux_a(uri, q, fri, iri);
            for (int v = 0; v < 3; v++) Fs[v][p] = 0.5 * (0.5 * ((fa[v] + fb[v]) + kc.rinv * (ua[v] - ub[v])) + fri[v]);
        }
        __syncthreads();
        double rb = 0.0, rinvb = 0.0, halfrb = 0.0, gb = 0.0;
        // reverse 1: update and setcons; mu = dL/dU'_c for real cells of positions [2, AP-2)
        {
            double mu[3] = {0.0, 0.0, 0.0};
            if (upd) {
                double Un[3];
                for (int v = 0; v < 3; v++) Un[v] = Us[v][p] + kc.r * (Fs[v][p] - Fs[v][p + 1]);
                // W = (rho, m / rho, (gamma - 1)(E - m u / 2) - gamma p_inf)
                const double ir = rcp_nr2(Un[0]);
                const double u = Un[1] * ir;
                const double X = Un[2] - 0.5 * Un[1] * u;
                mu[0] = lam[0] - u * ir * lam[1] + q.gm1 * 0.5 * u * u * lam[2];
                mu[1] = ir * lam[1] - q.gm1 * u * lam[2];
                mu[2] = q.gm1 * lam[2];
                if (out) {
                    gb += (X - q.pinf) * lam[2];
                    for (int v = 0; v < 3; v++) rb += mu[v] * (Fs[v][p] - Fs[v][p + 1]);
                }
            }
            for (int v = 0; v < 3; v++) MU[v][p] = mu[v];
        }
        __syncthreads();
        // reverse 2: interface left of positions [3, AP-2); real for right cell c in [0, n]
        {
            double uab[3] = {0.0, 0.0, 0.0}, ubb[3] = {0.0, 0.0, 0.0};
            const bool live = p >= 3 && p < AP - 2 && c >= 0 && c <= n;
            if (live) {
                double lf_b[3], urib[3] = {0.0, 0.0, 0.0}, lrb = 0.0, lrinvb = 0.0, lgb = 0.0;
                for (int v = 0; v < 3; v++) lf_b[v] = 0.5 * kc.r * (MU[v][p] - MU[v][p - 1]);  // lf-bar = fri-bar = F-bar / 2
                flux_vjp(uri, iri, q, lf_b, urib, lgb);
                double fab[3], fbb[3];
                for (int v = 0; v < 3; v++) {
                    fab[v] = 0.5 * lf_b[v] + 0.5 * kc.r * urib[v];
                    fbb[v] = 0.5 * lf_b[v] - 0.5 * kc.r * urib[v];
                    uab[v] = 0.5 * kc.rinv * lf_b[v] + 0.5 * urib[v];
                    ubb[v] = -0.5 * kc.rinv * lf_b[v] + 0.5 * urib[v];
                    lrb += 0.5 * urib[v] * dfab[v];
                    lrinvb += 0.5 * lf_b[v] * (ua[v] - ub[v]);
                }
                flux_vjp(ua, ira, q, fab, uab, lgb);
                flux_vjp(ub, irb, q, fbb, ubb, lgb);
                const bool own = c < n ? out : (p - 1 >= AH && p - 1 < AP - AH);
                if (own) {
                    rb += lrb;
                    rinvb += lrinvb;
                    gb += lgb;
                }
            }
            // edge adjoints of positions [2, AP-3); interfaces outside [0, n] contribute nothing
            if (p >= 3 && p < AP - 2) {
                for (int v = 0; v < 3; v++) {
                    BB[v][p - 1] = uab[v];
                    AB[v][p] = ubb[v];
                }
            }
        }
        __syncthreads();
        // reverse 3: edge adjoints of positions [3, AP-3) -> contributions to cells p-1, p, p+1
        {
            double l[3] = {0.0, 0.0, 0.0}, m[3] = {0.0, 0.0, 0.0}, rr[3] = {0.0, 0.0, 0.0};
            if (p >= 3 && p < AP - 3) {
                double xlb[3], xrb[3], flb[3], frb[3], lh = 0.0, lgb = 0.0;
                for (int v = 0; v < 3; v++) {
                    const double evb = AB[v][p] + BB[v][p];
                    xlb[v] = AB[v][p];
                    xrb[v] = BB[v][p];
                    flb[v] = kc.half_r * evb;
                    frb[v] = -kc.half_r * evb;
                    lh += evb * dF[v];
                }
                flux_vjp(xl, irl, q, flb, xlb, lgb);
                flux_vjp(xr, irr, q, frb, xrb, lgb);
                for (int v = 0; v < 3; v++) {
                    const double sb = 0.5 * (xrb[v] - xlb[v]);
                    const double dmb = sb * sdm[v], dpb = sb * sdp[v];
                    l[v] = -dmb;
                    m[v] = xlb[v] + xrb[v] + dmb - dpb;
                    rr[v] = dpb;
                }
                const bool own = real ? out : (c < 0 ? owns_first : owns_last);
                if (own) {
                    halfrb += lh;
                    gb += lgb;
                }
            }
            for (int v = 0; v < 3; v++) {
                UL[v][p] = l[v];
                US[v][p] = m[v];
                UR[v][p] = rr[v];
            }
        }
        __syncthreads();
        // reverse 4: dL/dU of output cells (direct path + three neighbouring edges + folded ghost copies), then cons
        if (out) {
            double Ub[3];
            for (int v = 0; v < 3; v++) {
                Ub[v] = MU[v][p] + US[v][p] + UR[v][p - 1] + UL[v][p + 1];
                // ghost g mirrors cell c when g = -1 - c (c <= 1) or g = 2n - 1 - c (c >= n - 2); its dL/dU is
                // US[g] + UR[g-1] + UL[g+1], where only the edges of ghosts -1 and n and of the real cells are live
                if (c == 0) Ub[v] += US[v][p - 1] + UL[v][p];      // ghost -1: own edges, cell 0's left operand
                if (c == 1) Ub[v] += UL[v][p - 2];                  // ghost -2: ghost -1's left operand
                if (c == n - 1) Ub[v] += US[v][p + 1] + UR[v][p];  // ghost n: own edges, cell n-1's right operand
                if (c == n - 2) Ub[v] += UR[v][p + 2];              // ghost n+1: ghost n's right operand
            }
            // U = (rho, rho u, rho u^2 / 2 + (p + gamma p_inf) / (gamma - 1))
            const double rho = W[0], u = W[1], pr = W[2];
            a.lam_out[base + c] = Ub[0] + u * Ub[1] + 0.5 * u * u * Ub[2];
            a.lam_out[a.plane + base + c] = rho * Ub[1] + rho * u * Ub[2];
            a.lam_out[2 * a.plane + base + c] = q.igm1 * Ub[2];
            gb += -(pr + q.pinf) * q.igm1 * q.igm1 * Ub[2];
        }
        // r-bar of this tile: r, half_r = r / 2 and rinv = 1 / r all depend on dt
        double tr = rb + 0.5 * halfrb - rinvb * (kc.rinv * kc.rinv);
        for (int o = 16; o > 0; o >>= 1) {
            tr += __shfl_xor_sync(0xffffffffu, tr, o);
            gb += __shfl_xor_sync(0xffffffffu, gb, o);
        }
        if ((p & 31) == 0) {
            red[0][p >> 5] = tr;
            red[1][p >> 5] = gb;
        }
        __syncthreads();
        if (p == 0) {
            double s1 = 0.0, s2 = 0.0;
            for (int w = 0; w < AP / 32; w++) {
                s1 += red[0][w];
                s2 += red[1][w];
            }
            a.tile_part[2 * t] = s1;
            a.tile_part[2 * t + 1] = s2;
        }
        __syncthreads();
    }
}

// Per instance: sum the tile partials in tile order, propagate dt-bar through the CFL maximum to the argmax cell.
__global__ void instance_dt_adjoint_kernel(double* lam, const double* W, long plane, const long* offset, const int* ncell,
                                           const double* dx, const double* gam, const int* tile_first,
                                           const int* tile_count, const double* tile_part,
                                           const unsigned long long* Sbits, double cfl, int s, int* arg, double* ggam,
                                           int ninst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ninst) return;
    double rbar = 0.0, gbar = 0.0;
    for (int t = tile_first[k]; t < tile_first[k] + tile_count[k]; t++) {
        rbar += tile_part[2 * t];
        gbar += tile_part[2 * t + 1];
    }
    const int ai = arg[k];
    arg[k] = 0x7fffffff;  // ready for the next reversed step
    if (ai < 0 || ai >= ncell[k]) {  // no cell attains S: cannot happen for a state whose S was taken from it
        ggam[k] += gbar;
        return;
    }
    // r = dt / dx, dt = CFL dx / S (x0.2):  S-bar = -(dt / S) dt-bar
    const double S = __longlong_as_double((long long)Sbits[k]);
    const double dtb = rbar / dx[k];
    const double Sb = -(step_dt(cfl, dx[k], S, s) / S) * dtb;
    const long i = offset[k] + ai;
    const double rho = W[i], u = W[plane + i], p = W[2 * plane + i];
    const double g = gam[2 * k], pinf = gam[2 * k + 1];
    const double c = sqrt((g * (p + pinf)) / rho);
    lam[i] += (-c / (2.0 * rho)) * Sb;
    lam[plane + i] += (u > 0.0 ? 1.0 : (u < 0.0 ? -1.0 : 0.0)) * Sb;
    lam[2 * plane + i] += (g / (2.0 * rho * c)) * Sb;
    ggam[k] += gbar + ((p + pinf) / (2.0 * rho * c)) * Sb;
}

// Loss and its gradient at the final state: lambda = (2 (rho - target), 0, 0); per-block partial losses.
__global__ void __launch_bounds__(256) loss_kernel(const double* W, const double* target, long plane, double* lam,
                                                   double* block_loss) {
    double acc = 0.0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < plane; i += (long)gridDim.x * 256) {
        const double d = W[i] - target[i];
        acc += d * d;
        lam[i] = 2.0 * d;
        lam[plane + i] = 0.0;
        lam[2 * plane + i] = 0.0;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_loss[blockIdx.x] = red[0];
}

}  // namespace
}  // namespace vg

namespace {

vg_status afail(vg_status st, const std::string& m) {
    vg::set_last_error(m);
    return st;
}

#define VA_CUDA(call)                                                                                \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return afail(e_ == cudaErrorMemoryAllocation ? VG_ENOMEM : VG_ECUDA,   \
                                            std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

// beta(s, t) = C(s + t, s): the most steps that s stored states (the starting state included) reverse when no
// step is advanced more than t times (Griewank's binomial bound)
double beta(int s, int t) {
    double v = 1.0;
    for (int i = 1; i <= t; i++) v = v * (s + i) / i;
    return v;
}

// Workspace that depends only on the batch's instance sizes: adjoint tiles, per-tile partials, per-instance scalars.
cudaError_t ensure_workspace(vg_batch* b, int checkpoints) {
    const long n = b->total;
    const size_t sbytes = sizeof(double) * 3 * n;
    cudaError_t e = cudaSuccess;
    if (b->ckpt_slots != checkpoints) {
        if (b->ckpt) cudaFree(b->ckpt);
        if (b->ckptS) cudaFree(b->ckptS);
        b->ckpt = nullptr;
        b->ckptS = nullptr;
        b->ckpt_slots = 0;
        e = cudaMalloc(&b->ckpt, sbytes * (checkpoints + 1));  // + 1: the recomputation buffer
        if (e == cudaSuccess) e = cudaMalloc(&b->ckptS, sizeof(unsigned long long) * b->ninst * (checkpoints + 1));
        if (e != cudaSuccess) return e;
        b->ckpt_slots = checkpoints;
    }
    if (b->lam[0]) return cudaSuccess;
    std::vector<vg::Tile> at;
    std::vector<int> af(b->ninst), ac(b->ninst), order(b->ninst);
    for (int k = 0; k < b->ninst; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->ncell[x] > b->ncell[y]; });
    for (int k : order) {
        af[k] = (int)at.size();
        for (int s0 = 0; s0 < b->ncell[k]; s0 += vg::AOUT) at.push_back({k, s0});
        ac[k] = (int)at.size() - af[k];
    }
    b->natiles = (int)at.size();
    b->loss_blocks = (int)std::min<long>((n + 255) / 256, 1024);
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vg::adjoint_step_kernel, vg::AP, 0);
    b->agrid = std::max(1, std::min(b->natiles, sms * std::max(per_sm, 1)));
    if (e == cudaSuccess) e = cudaMalloc(&b->lam[0], sbytes);
    if (e == cudaSuccess) e = cudaMalloc(&b->lam[1], sbytes);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_target, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_atiles, sizeof(vg::Tile) * at.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tile_part, sizeof(double) * 2 * at.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tile_first, sizeof(int) * b->ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tile_count, sizeof(int) * b->ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ggam, sizeof(double) * b->ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_arg, sizeof(int) * b->ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_loss, sizeof(double) * b->loss_blocks);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_atiles, at.data(), sizeof(vg::Tile) * at.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_tile_first, af.data(), sizeof(int) * b->ninst, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_tile_count, ac.data(), sizeof(int) * b->ninst, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        std::vector<int> none(b->ninst, 0x7fffffff);
        e = cudaMemcpy(b->d_arg, none.data(), sizeof(int) * b->ninst, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {  // leave the workspace absent so the next call retries
        for (double** p : {&b->lam[0], &b->lam[1], &b->d_target, &b->d_tile_part, &b->d_ggam, &b->d_loss}) {
            cudaFree(*p);
            *p = nullptr;
        }
        cudaFree(b->d_atiles);
        cudaFree(b->d_tile_first);
        cudaFree(b->d_tile_count);
        cudaFree(b->d_arg);
        b->d_atiles = nullptr;
        b->d_tile_first = b->d_tile_count = b->d_arg = nullptr;
    }
    return e;
}

// Reverse sweep over the time steps with a binomial checkpoint schedule.
struct Reverser {
    vg_batch* b;
    double cfl, bias, floor5;
    int limiter, steps;
    cudaStream_t st;
    std::vector<double*> slots;  // checkpoint buffers; slot 0 holds W^0 throughout
    std::vector<unsigned long long*> slotsS;  // their per-instance maxima |u| + c
    std::vector<bool> used;
    double* tmp;                 // recomputed state
    unsigned long long* tmpS;
    int lam_cur = 0;             // lam[lam_cur] holds dL/dW^{s+1} before reversing step s
    bool started = false;

    int take() {
        for (size_t i = 0; i < used.size(); i++)
            if (!used[i]) {
                used[i] = true;
                return (int)i;
            }
        return -1;
    }

    // W^steps from W^{steps-1} (into the idle adjoint buffer), then the loss and dL/dW^steps
    cudaError_t init_final(const double* Wprev, const unsigned long long* WprevS) {
        double* Wfin = b->lam[1 - lam_cur];
        cudaError_t e = vg::batch_advance(b, Wprev, WprevS, Wfin, nullptr, steps - 1, 1, cfl, bias, limiter, st);
        if (e != cudaSuccess) return e;
        vg::loss_kernel<<<b->loss_blocks, 256, 0, st>>>(Wfin, b->d_target, b->total, b->lam[lam_cur], b->d_loss);
        started = true;
        return cudaGetLastError();
    }

    // dL/dW^s from dL/dW^{s+1} and W^s
    cudaError_t adjoint_step(const double* Ws, const unsigned long long* WsS, int s) {
        if (s == steps - 1 && !started) {
            cudaError_t e = init_final(Ws, WsS);
            if (e != cudaSuccess) return e;
        }
        vg::AdjArgs a{};
        a.W = Ws;
        a.lam_in = b->lam[lam_cur];
        a.lam_out = b->lam[1 - lam_cur];
        a.plane = b->total;
        a.offset = b->d_offset;
        a.ncell = b->d_ncell;
        a.dx = b->d_dx;
        a.gam = b->d_gam;
        a.tiles = b->d_atiles;
        a.ntiles = b->natiles;
        a.S = WsS;
        a.arg = b->d_arg;
        a.tile_part = b->d_tile_part;
        a.cfl = cfl;
        a.bias = bias;
        a.floor5 = floor5;
        a.limiter = limiter;
        a.step = s;
        vg::adjoint_step_kernel<<<b->agrid, vg::AP, 0, st>>>(a);
        vg::instance_dt_adjoint_kernel<<<(b->ninst + 127) / 128, 128, 0, st>>>(
            b->lam[1 - lam_cur], Ws, b->total, b->d_offset, b->d_ncell, b->d_dx, b->d_gam, b->d_tile_first,
            b->d_tile_count, b->d_tile_part, WsS, cfl, s, b->d_arg, b->d_ggam, b->ninst);
        lam_cur = 1 - lam_cur;
        b->last_adjoint_steps++;
        return cudaGetLastError();
    }

    // Reverse steps [s0, s1) given W^{s0} in slots[slot] and c free slots besides it.  Split (Griewank's
    // binomial rule): t = least repetition count with beta(c + 1, t) >= n; advance to m so that the right part
    // [m, s1) is reversible with c slots (c - 1 free) and t repetitions, reverse it, then the left part with
    // one repetition fewer.
    cudaError_t reverse(int s0, int s1, int c, int slot) {
        cudaError_t e = cudaSuccess;
        const int n = s1 - s0;
        if (n == 1) return adjoint_step(slots[slot], slotsS[slot], s0);
        if (c == 0) {  // only the starting state: recompute every step from it
            for (int s = s1 - 1; s > s0 && e == cudaSuccess; s--) {
                e = vg::batch_advance(b, slots[slot], slotsS[slot], tmp, tmpS, s0, s - s0, cfl, bias, limiter, st);
                if (e == cudaSuccess) e = adjoint_step(tmp, tmpS, s);
            }
            if (e == cudaSuccess) e = adjoint_step(slots[slot], slotsS[slot], s0);
            return e;
        }
        int t = 1;
        while (beta(c + 1, t) < n) t++;
        const int right = (int)std::min<double>(n - 1, beta(c, t));
        const int m = s1 - right;
        const int ns = take();
        e = vg::batch_advance(b, slots[slot], slotsS[slot], slots[ns], slotsS[ns], s0, m - s0, cfl, bias, limiter, st);
        if (e == cudaSuccess) e = reverse(m, s1, c - 1, ns);
        used[ns] = false;
        if (e == cudaSuccess) e = reverse(s0, m, c, slot);
        return e;
    }
};

}  // namespace

extern "C" vg_status vg_batch_gradient(vg_batch* b, const double* target_rho, double cfl, int steps, double bias,
                                       int limiter, int checkpoints, double* loss, double* grad_planes,
                                       double* grad_gamma, int is_device, long* forward_steps, long* adjoint_steps,
                                       void* stream) {
    if (!b || !target_rho || steps < 1 || !(cfl > 0.0) || limiter < 0 || limiter > 2)
        return afail(VG_EINVAL, "bad vg_batch_gradient argument");
    if (checkpoints < 1) return afail(VG_EINVAL, "need at least one checkpoint slot (the initial state)");
    if (!b->has_state) return afail(VG_EINVAL, "no state uploaded");
    checkpoints = std::min(checkpoints, steps);
    cudaStream_t st = (cudaStream_t)stream;
    VA_CUDA(cudaSetDevice(b->device));
    VA_CUDA(ensure_workspace(b, checkpoints));
    const long n = b->total;
    const size_t sbytes = sizeof(double) * 3 * n;
    const cudaMemcpyKind in_kind = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out_kind = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    VA_CUDA(cudaMemcpyAsync(b->d_target, target_rho, sizeof(double) * n, in_kind, st));
    VA_CUDA(cudaMemsetAsync(b->d_ggam, 0, sizeof(double) * b->ninst, st));
    VA_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(unsigned int), st));

    Reverser R;
    R.b = b;
    R.cfl = cfl;
    R.bias = bias;
    R.floor5 = std::pow(10.0, -5.0);
    R.limiter = limiter;
    R.steps = steps;
    R.st = st;
    for (int i = 0; i < checkpoints; i++) {
        R.slots.push_back(b->ckpt + (long)i * 3 * n);
        R.slotsS.push_back(b->ckptS + (long)i * b->ninst);
    }
    R.used.assign(checkpoints, false);
    R.tmp = b->ckpt + (long)checkpoints * 3 * n;
    R.tmpS = b->ckptS + (long)checkpoints * b->ninst;
    b->last_forward_steps = 0;
    b->last_adjoint_steps = 0;
    VA_CUDA(cudaMemcpyAsync(R.slots[0], b->buf[b->cur], sbytes, cudaMemcpyDeviceToDevice, st));
    VA_CUDA(vg::batch_wave_max(b, R.slots[0], R.slotsS[0], st));
    R.used[0] = true;
    cudaError_t e = R.reverse(0, steps, checkpoints - 1, 0);
    // the batch keeps its initial state
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->buf[0], R.slots[0], sbytes, cudaMemcpyDeviceToDevice, st);
    b->cur = 0;
    std::vector<double> bl(b->loss_blocks);
    unsigned int err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(bl.data(), b->d_loss, sizeof(double) * bl.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, b->d_err, sizeof(err), cudaMemcpyDeviceToHost, st);
    // gradient planes in the 6-plane Euler layout: rho, u, v, w, p, lambda (v, w, lambda are held fixed: 0)
    const double* lam0 = b->lam[R.lam_cur];
    const int ref[3] = {0, 1, 4};
    for (int v = 0; v < 3 && e == cudaSuccess && grad_planes; v++)
        e = cudaMemcpyAsync(grad_planes + ref[v] * n, lam0 + v * n, sizeof(double) * n, out_kind, st);
    for (int v : {2, 3, 5})
        if (e == cudaSuccess && grad_planes && is_device) e = cudaMemsetAsync(grad_planes + v * n, 0, sizeof(double) * n, st);
    if (e == cudaSuccess && grad_gamma)
        e = cudaMemcpyAsync(grad_gamma, b->d_ggam, sizeof(double) * b->ninst, out_kind, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return afail(VG_ECUDA, std::string("vg_batch_gradient: ") + cudaGetErrorString(e));
    if (err) return afail(VG_ENAN, "non-finite value, non-positive density or pressure at or below -p_inf produced");
    if (grad_planes && !is_device)
        for (long i = 0; i < n; i++) grad_planes[2 * n + i] = grad_planes[3 * n + i] = grad_planes[5 * n + i] = 0.0;
    if (loss) {
        double sum = 0.0;
        for (double x : bl) sum += x;
        *loss = sum;
    }
    if (forward_steps) *forward_steps = b->last_forward_steps;
    if (adjoint_steps) *adjoint_steps = b->last_adjoint_steps;
    return VG_OK;
}
