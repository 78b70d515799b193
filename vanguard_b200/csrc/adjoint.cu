// Discrete adjoint of the batched 1D Euler SLIC step, with binomial checkpointing (no counterpart in the
// reference, which has no derivatives).
//
// Loss  L = sum_k sum_i (rho_k,i(T) - target_k,i)^2  after `steps` steps of every instance's own solve() loop.
// Output dL/dW^0 (primitive planes rho, u, p of every cell) and dL/dgamma_k.
//
// One reverse step s maps lambda^{s+1} = dL/dW^{s+1} to lambda^s through the exact-FP64 forward step of
// batch.cu, recomputed from W^s with the same device functions (so the limiter takes the same branches):
//   W^{s+1}_i = setcons(U_i + r (F_{i-1/2} - F_{i+1/2})),  U_i = cons(W^s_i),  r = dt / dx,
//   F_{j+1/2} = FORCE(evolve_R(W_{j-1}, W_j, W_{j+1}), evolve_L(W_j, W_{j+1}, W_{j+2})),
//   dt = CFL dx / S (x0.2 for s <= 5),  S = max_i (|u_i| + c_i).
// Vector-Jacobian products are written by hand for cons / setcons / the x flux (exact identities of the ideal
// stiffened gas, the primitive round trips of the reference are identities), the slope limiter, the half-step
// evolution, the Lax-Friedrichs / Richtmyer / FORCE combination and the update.  Subgradients:
//   * limiter: the derivative of the branch the forward pass took (one-sided at r = 0, 1/2, 1 and where the
//     minimum switches between r, xi_R and 2), computed with the forward's own comparisons;
//   * the |delta| < 1e-5 floor: zero derivative of the floored ratio operand;
//   * the CFL maximum: only the first cell attaining the maximum receives dS; |u| has derivative sign(u), 0 at 0.
// The dt dependence is propagated (dt -> S -> that cell's state and gamma), so the gradient is that of the
// scheme that adapts its step, which is what central finite differences measure.
//
// Tiles: AP = 128 positions per block, AH = 5 halo cells each side, AP - 2 AH outputs.  Every contribution to r-bar
// and gamma-bar is owned by exactly one tile (interfaces by their right cell, or the last cell at the right end;
// ghost-cell edges by the instance's end cells), so the per-instance sums are deterministic.  Ghost cells
// (transmissive mirror copies, Solvers/solvers.cpp:17-23) fold their adjoints into the cells they copy.
// Compiled with -fmad=false so the recomputed forward matches the stored one bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/vanguard_slic.h"
#include "batch_internal.cuh"
#include "physics_fp64.cuh"
#include "slic_kernels.cuh"
#include "vg_ops.h"

namespace vg {
namespace {

using M1 = EulerF64<1>;
constexpr int AP = 128;
constexpr int AH = 5;
constexpr int AOUT = AP - 2 * AH;

struct Q1 {
    double g, pinf;
};

// ---------------------------------------------------------------------------- vector-Jacobian products
// U = (rho, rho u, rho u^2 / 2 + (p + g pinf) / (g - 1))
__device__ __forceinline__ void cons_vjp(const double* W, const Q1& q, const double* Ub, double* Wb, double& gb) {
    double rho = W[0], u = W[1], p = W[2], gm1 = q.g - 1.0;
    Wb[0] += Ub[0] + u * Ub[1] + 0.5 * u * u * Ub[2];
    Wb[1] += rho * Ub[1] + rho * u * Ub[2];
    Wb[2] += Ub[2] / gm1;
    gb += (-(p + q.pinf) / (gm1 * gm1)) * Ub[2];
}
// p = (g - 1)(U2 - U1 u / 2) - g pinf with u = U1 / U0
__device__ __forceinline__ void pressure_vjp(const double* U, const Q1& q, double u, double pb, double* Ub, double& gb) {
    double gm1 = q.g - 1.0;
    Ub[0] += gm1 * 0.5 * u * u * pb;
    Ub[1] += -gm1 * u * pb;
    Ub[2] += gm1 * pb;
    gb += ((U[2] - 0.5 * U[1] * u) - q.pinf) * pb;
}
__device__ __forceinline__ void setcons_vjp(const double* U, const Q1& q, const double* Wb, double* Ub, double& gb) {
    double rho = U[0], u = U[1] / rho;
    Ub[0] += Wb[0] - (u / rho) * Wb[1];
    Ub[1] += Wb[1] / rho;
    pressure_vjp(U, q, u, Wb[2], Ub, gb);
}
// F = (U1, U1 u + p, u (U2 + p))
__device__ __forceinline__ void flux_vjp(const double* U, const Q1& q, const double* Fb, double* Ub, double& gb) {
    double rho = U[0], u = U[1] / rho;
    double p = (q.g - 1.0) * (U[2] - 0.5 * U[1] * u) - q.g * q.pinf;
    double ub = U[1] * Fb[1] + (U[2] + p) * Fb[2];
    double pb = Fb[1] + u * Fb[2];
    Ub[1] += Fb[0] + u * Fb[1];
    Ub[2] += u * Fb[2];
    Ub[0] += -(u / rho) * ub;
    Ub[1] += ub / rho;
    pressure_vjp(U, q, u, pb, Ub, gb);
}
// d xi / d r of the branch SlopeLimiters::computeSlopeLimiter takes (Solvers/slopelimiters.cpp:7-74), with the
// forward's own comparisons and std::min tie rule
__device__ __forceinline__ double limiter_deriv(double r, double w, int id) {
    double den = (1.0 - w) + ((1.0 + w) * r);
    double xr = 2.0 / den, dxr = -2.0 * (1.0 + w) / (den * den);
    if (id == 0) {
        if (r < 0.0) return 0.0;
        if (r < 0.5) return 2.0;
        if (r < 1.0) return 0.0;
        double m1 = (xr < r) ? xr : r, dm1 = (xr < r) ? dxr : 1.0;
        return (2.0 < m1) ? 0.0 : dm1;
    } else if (id == 1) {
        if (r < 0.0) return 0.0;
        double a = (2.0 * r) / (1.0 + r);
        return (xr < a) ? dxr : 2.0 / ((1.0 + r) * (1.0 + r));
    }
    if (r < 0.0) return 0.0;
    if (r < 1.0) return 1.0;
    return (xr < 1.0) ? dxr : 0.0;
}
__device__ __forceinline__ void slope_vjp(double uL, double u, double uR, const SweepConst& k, double sb, double& uLb,
                                          double& ub, double& uRb) {
    double dm = u - uL, dp = uR - u;
    double base = (k.cm * dm) + (k.cp * dp);
    bool nf = fabs(dm) < k.floor5, df = fabs(dp) < k.floor5;
    double num = nf ? k.floor5 : dm, den = df ? k.floor5 : dp;
    double r = num / den;
    double xi = limiter_f64(r, k.bias, k.limiter), dxi = limiter_deriv(r, k.bias, k.limiter);
    double dmb = sb * (k.cm * xi) + (nf ? 0.0 : sb * base * dxi / den);
    double dpb = sb * (k.cp * xi) + (df ? 0.0 : -sb * base * dxi * num / (den * den));
    uLb -= dmb;
    ub += dmb - dpb;
    uRb += dpb;
}
// adjoint of evolve_edges for one cell: ab / bb adjoints of its left-side / right-side evolved states
__device__ void evolve_vjp(const double* uL, const double* u, const double* uR, const SweepConst& k, const Q1& q1,
                           const M1::P& q, const double* ab, const double* bb, double* uLb, double* ub, double* uRb,
                           double& halfrb, double& gb) {
    double xl[3], xr[3], fl[3], fr[3];
    for (int i = 0; i < 3; i++) {
        double s = slope_f64(uL[i], u[i], uR[i], k);
        xl[i] = u[i] - (0.5 * s);
        xr[i] = u[i] + (0.5 * s);
    }
    M1::flux<0>(xl, q, fl);
    M1::flux<0>(xr, q, fr);
    double xlb[3], xrb[3], flb[3], frb[3];
    for (int i = 0; i < 3; i++) {
        double evb = ab[i] + bb[i];
        xlb[i] = ab[i];
        xrb[i] = bb[i];
        flb[i] = k.half_r * evb;
        frb[i] = -k.half_r * evb;
        halfrb += evb * (fl[i] - fr[i]);
    }
    flux_vjp(xl, q1, flb, xlb, gb);
    flux_vjp(xr, q1, frb, xrb, gb);
    for (int i = 0; i < 3; i++) {
        ub[i] += xlb[i] + xrb[i];
        slope_vjp(uL[i], u[i], uR[i], k, 0.5 * (xrb[i] - xlb[i]), uLb[i], ub[i], uRb[i]);
    }
}
// adjoint of force_flux(ua, ub)
__device__ void force_vjp(const double* ua, const double* ubv, const SweepConst& k, const Q1& q1, const M1::P& q,
                          const double* Fb, double* uab, double* ubb, double& rb, double& rinvb, double& gb) {
    double fa[3], fb[3], uri[3];
    M1::flux<0>(ua, q, fa);
    M1::flux<0>(ubv, q, fb);
    for (int i = 0; i < 3; i++) uri[i] = 0.5 * ((ua[i] + ubv[i]) + (k.r * (fa[i] - fb[i])));
    double urib[3] = {0.0, 0.0, 0.0}, frib[3], lfb[3], fab[3], fbb[3];
    for (int i = 0; i < 3; i++) {
        lfb[i] = 0.5 * Fb[i];
        frib[i] = 0.5 * Fb[i];
    }
    flux_vjp(uri, q1, frib, urib, gb);
    for (int i = 0; i < 3; i++) {
        fab[i] = 0.5 * lfb[i] + 0.5 * k.r * urib[i];
        fbb[i] = 0.5 * lfb[i] - 0.5 * k.r * urib[i];
        uab[i] += 0.5 * k.rinv * lfb[i] + 0.5 * urib[i];
        ubb[i] += -0.5 * k.rinv * lfb[i] + 0.5 * urib[i];
        rb += 0.5 * urib[i] * (fa[i] - fb[i]);
        rinvb += 0.5 * lfb[i] * (ua[i] - ubv[i]);
    }
    flux_vjp(ua, q1, fab, uab, gb);
    flux_vjp(ubv, q1, fbb, ubb, gb);
}

// ------------------------------------------------------------------------------------------------ kernels
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
    const double* dts;      // dt and S of step s, 2 per instance
    double* tile_part;      // per tile: r-bar (dL/dr) and gamma-bar
    double bias, floor5;
    int limiter;
};

__global__ void __launch_bounds__(AP) adjoint_step_kernel(AdjArgs a) {
    __shared__ double Us[3][AP], Ea[3][AP], Eb[3][AP], Fs[3][AP + 1], MU[3][AP], AB[3][AP], BB[3][AP], UL[3][AP],
        US[3][AP], UR[3][AP];
    __shared__ double red[2][AP / 32];
    const int p = threadIdx.x;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int k = tile.inst, n = a.ncell[k], s0 = tile.s0;
        const long base = a.offset[k];
        const int c = s0 - AH + p;  // cell of this position (may be a ghost or beyond)
        const bool real = c >= 0 && c < n;
        const bool out = p >= AH && p < AP - AH && real;
        const bool owns_first = s0 == 0;                       // tile owning cell 0
        const bool owns_last = s0 <= n - 1 && n - 1 < s0 + AOUT;  // tile owning cell n-1
        const double dt = a.dts[2 * k], dxk = a.dx[k];
        SweepConst kc;
        kc.r = dt / dxk;
        kc.rinv = dxk / dt;
        kc.half_r = 0.5 * (dt / dxk);
        kc.cm = 0.5 * (1.0 + a.bias);
        kc.cp = 0.5 * (1.0 - a.bias);
        kc.bias = a.bias;
        kc.floor5 = a.floor5;
        kc.limiter = a.limiter;
        const M1::P q{a.gam[2 * k], a.gam[2 * k + 1], 0.0};
        const Q1 q1{a.gam[2 * k], a.gam[2 * k + 1]};
        double W[3];
        {
            const int gi = ghost_index(c, n, 0);
            for (int v = 0; v < 3; v++) W[v] = a.W[v * a.plane + base + gi];
            double U[3];
            M1::cons(W, q, U);
            for (int v = 0; v < 3; v++) {
                Us[v][p] = U[v];
                MU[v][p] = AB[v][p] = BB[v][p] = UL[v][p] = US[v][p] = UR[v][p] = 0.0;
            }
        }
        __syncthreads();
        // forward: evolved edge states of positions [1, AP-1)
        if (p >= 1 && p < AP - 1) {
            double uL[3], u[3], uR[3], ea[3], eb[3];
            for (int v = 0; v < 3; v++) {
                uL[v] = Us[v][p - 1];
                u[v] = Us[v][p];
                uR[v] = Us[v][p + 1];
            }
            evolve_edges<M1, 0>(uL, u, uR, kc, q, ea, eb, true, true);
            for (int v = 0; v < 3; v++) {
                Ea[v][p] = ea[v];
                Eb[v][p] = eb[v];
            }
        }
        __syncthreads();
        // forward: FORCE flux at the interface left of positions [2, AP-1)
        if (p >= 2 && p < AP - 1) {
            double ua[3], ub[3], F[3];
            for (int v = 0; v < 3; v++) {
                ua[v] = Eb[v][p - 1];
                ub[v] = Ea[v][p];
            }
            force_flux<M1, 0>(ua, ub, kc, q, F);
            for (int v = 0; v < 3; v++) Fs[v][p] = F[v];
        }
        __syncthreads();
        double rb = 0.0, rinvb = 0.0, halfrb = 0.0, gb = 0.0;
        // reverse 1: update and setcons, mu = dL/dU'_c for real cells of positions [2, AP-2)
        if (p >= 2 && p < AP - 2 && real) {
            double Un[3], lam[3], mu[3] = {0.0, 0.0, 0.0}, g0 = 0.0;
            for (int v = 0; v < 3; v++) {
                Un[v] = Us[v][p] + (kc.r * (Fs[v][p] - Fs[v][p + 1]));
                lam[v] = a.lam_in[v * a.plane + base + c];
            }
            setcons_vjp(Un, q1, lam, mu, g0);
            for (int v = 0; v < 3; v++) MU[v][p] = mu[v];
            if (out) {
                gb += g0;
                for (int v = 0; v < 3; v++) rb += mu[v] * (Fs[v][p] - Fs[v][p + 1]);
            }
        }
        __syncthreads();
        // reverse 2: interface left of positions [3, AP-2); real for right cell c in [0, n]
        if (p >= 3 && p < AP - 2 && c >= 0 && c <= n) {
            double Fb[3], uab[3] = {0.0, 0.0, 0.0}, ubb[3] = {0.0, 0.0, 0.0}, ua[3], ub[3];
            double lrb = 0.0, lrinvb = 0.0, lgb = 0.0;
            for (int v = 0; v < 3; v++) {
                Fb[v] = kc.r * (MU[v][p] - MU[v][p - 1]);
                ua[v] = Eb[v][p - 1];
                ub[v] = Ea[v][p];
            }
            force_vjp(ua, ub, kc, q1, q, Fb, uab, ubb, lrb, lrinvb, lgb);
            for (int v = 0; v < 3; v++) {
                BB[v][p - 1] = uab[v];
                AB[v][p] = ubb[v];
            }
            const bool own = c < n ? out : (p - 1 >= AH && p - 1 < AP - AH);
            if (own) {
                rb += lrb;
                rinvb += lrinvb;
                gb += lgb;
            }
        }
        __syncthreads();
        // reverse 3: edge adjoints of positions [3, AP-3) -> contributions to cells p-1, p, p+1
        if (p >= 3 && p < AP - 3) {
            double uL[3], u[3], uR[3], ab[3], bb[3], uLb[3] = {0, 0, 0}, ub[3] = {0, 0, 0}, uRb[3] = {0, 0, 0};
            double lh = 0.0, lgb = 0.0;
            for (int v = 0; v < 3; v++) {
                uL[v] = Us[v][p - 1];
                u[v] = Us[v][p];
                uR[v] = Us[v][p + 1];
                ab[v] = AB[v][p];
                bb[v] = BB[v][p];
            }
            evolve_vjp(uL, u, uR, kc, q1, q, ab, bb, uLb, ub, uRb, lh, lgb);
            for (int v = 0; v < 3; v++) {
                UL[v][p] = uLb[v];
                US[v][p] = ub[v];
                UR[v][p] = uRb[v];
            }
            const bool own = real ? out : (c < 0 ? owns_first : owns_last);
            if (own) {
                halfrb += lh;
                gb += lgb;
            }
        }
        __syncthreads();
        // reverse 4: dL/dU of output cells (direct path + three neighbouring edges + folded ghost copies), then cons
        if (out) {
            double Ub[3];
            for (int v = 0; v < 3; v++) {
                Ub[v] = MU[v][p] + US[v][p] + UR[v][p - 1] + UL[v][p + 1];
                // ghost g mirrors cell c when g = -1 - c (c <= 1) or g = 2n - 1 - c (c >= n - 2); its dL/dU is
                // US[g] + UR[g-1] + UL[g+1], where only edges of the ghosts -1 and n and the real end cells are non-zero
                if (c == 0) Ub[v] += US[v][p - 1] + UL[v][p];                      // ghost -1: own edge, cell 0's left
                if (c == 1) Ub[v] += UL[v][p - 2];                                  // ghost -2: ghost -1's left
                if (c == n - 1) Ub[v] += US[v][p + 1] + UR[v][p];                   // ghost n: own edge, cell n-1's right
                if (c == n - 2) Ub[v] += UR[v][p + 2];                              // ghost n+1: ghost n's right
            }
            double Wb[3] = {0.0, 0.0, 0.0};
            cons_vjp(W, q1, Ub, Wb, gb);
            for (int v = 0; v < 3; v++) a.lam_out[v * a.plane + base + c] = Wb[v];
        }
        // r-bar of this tile: r, half_r = r / 2 and rinv = 1 / r all depend on dt
        double tr = rb + 0.5 * halfrb - rinvb / (kc.r * kc.r);
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

// Per instance: S = max (|u| + c) with its first argmax, and dt of step s (one block per instance).
__global__ void __launch_bounds__(256) instance_dt_kernel(const double* W, long plane, const long* offset, const int* ncell,
                                                          const double* dx, const double* gam, double cfl, int s,
                                                          double* dts, int* arg_out) {
    const int k = blockIdx.x;
    const long base = offset[k];
    const int n = ncell[k];
    const M1::P q{gam[2 * k], gam[2 * k + 1], 0.0};
    double best = 0.0;
    int arg = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += 256) {
        double w[3] = {W[base + i], W[plane + base + i], W[2 * plane + base + i]};
        double sw = M1::wave(w, q, 1);
        if (sw > best) {  // per thread the indices increase, so the first maximum is kept
            best = sw;
            arg = i;
        }
    }
    __shared__ double bv[256];
    __shared__ int bi[256];
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = arg;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            double ov = bv[threadIdx.x + o];
            int oi = bi[threadIdx.x + o];
            if (ov > bv[threadIdx.x] || (ov == bv[threadIdx.x] && oi < bi[threadIdx.x])) {
                bv[threadIdx.x] = ov;
                bi[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double S = bv[0];
        double d = cfl * (dx[k] / S);
        if (s <= 5) d *= 0.2;
        dts[2 * k] = d;
        dts[2 * k + 1] = S;
        arg_out[k] = bi[0];
    }
}

// Per instance: sum the tile partials in tile order, propagate dt-bar through the CFL maximum to the argmax cell.
__global__ void instance_dt_adjoint_kernel(double* lam, const double* W, long plane, const long* offset, const double* dx,
                                           const double* gam, const int* tile_first, const int* tile_count,
                                           const double* tile_part, const double* dts, const int* arg, double* ggam,
                                           int ninst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ninst) return;
    double rbar = 0.0, gbar = 0.0;
    for (int t = tile_first[k]; t < tile_first[k] + tile_count[k]; t++) {
        rbar += tile_part[2 * t];
        gbar += tile_part[2 * t + 1];
    }
    // r = dt / dx, dt = CFL dx / S (x0.2):  dS-bar = -(dt / S) dt-bar
    const double dtb = rbar / dx[k];
    const double Sb = -(dts[2 * k] / dts[2 * k + 1]) * dtb;
    const long i = offset[k] + arg[k];
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
        double d = W[i] - target[i];
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
        b->ckpt = nullptr;
        b->ckpt_slots = 0;
        e = cudaMalloc(&b->ckpt, sbytes * (checkpoints + 1));  // + 1: the recomputation buffer
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
    if (e == cudaSuccess) e = cudaMalloc(&b->d_stepdt, sizeof(double) * 2 * b->ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_arg, sizeof(int) * b->ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_loss, sizeof(double) * b->loss_blocks);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_atiles, at.data(), sizeof(vg::Tile) * at.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_tile_first, af.data(), sizeof(int) * b->ninst, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_tile_count, ac.data(), sizeof(int) * b->ninst, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {  // leave the workspace absent so the next call retries
        for (double** p : {&b->lam[0], &b->lam[1], &b->d_target, &b->d_tile_part, &b->d_ggam, &b->d_stepdt, &b->d_loss}) {
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
    std::vector<bool> used;
    double* tmp;                 // recomputed state
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
    cudaError_t init_final(const double* Wprev) {
        double* Wfin = b->lam[1 - lam_cur];
        cudaError_t e = vg::batch_advance(b, Wprev, Wfin, steps - 1, 1, cfl, bias, limiter, st);
        if (e != cudaSuccess) return e;
        vg::loss_kernel<<<b->loss_blocks, 256, 0, st>>>(Wfin, b->d_target, b->total, b->lam[lam_cur], b->d_loss);
        started = true;
        return cudaGetLastError();
    }

    // dL/dW^s from dL/dW^{s+1} and W^s
    cudaError_t adjoint_step(const double* Ws, int s) {
        if (s == steps - 1 && !started) {
            cudaError_t e = init_final(Ws);
            if (e != cudaSuccess) return e;
        }
        vg::instance_dt_kernel<<<b->ninst, 256, 0, st>>>(Ws, b->total, b->d_offset, b->d_ncell, b->d_dx, b->d_gam, cfl, s,
                                                          b->d_stepdt, b->d_arg);
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
        a.dts = b->d_stepdt;
        a.tile_part = b->d_tile_part;
        a.bias = bias;
        a.floor5 = floor5;
        a.limiter = limiter;
        vg::adjoint_step_kernel<<<b->agrid, vg::AP, 0, st>>>(a);
        vg::instance_dt_adjoint_kernel<<<(b->ninst + 127) / 128, 128, 0, st>>>(
            b->lam[1 - lam_cur], Ws, b->total, b->d_offset, b->d_dx, b->d_gam, b->d_tile_first, b->d_tile_count,
            b->d_tile_part, b->d_stepdt, b->d_arg, b->d_ggam, b->ninst);
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
        if (n == 1) return adjoint_step(slots[slot], s0);
        if (c == 0) {  // only the starting state: recompute every step from it
            for (int s = s1 - 1; s >= s0 && e == cudaSuccess; s--) {
                e = vg::batch_advance(b, slots[slot], tmp, s0, s - s0, cfl, bias, limiter, st);
                if (e == cudaSuccess) e = adjoint_step(tmp, s);
            }
            return e;
        }
        int t = 1;
        while (beta(c + 1, t) < n) t++;
        const int right = (int)std::min<double>(n - 1, beta(c, t));
        const int m = s1 - right;
        const int ns = take();
        e = vg::batch_advance(b, slots[slot], slots[ns], s0, m - s0, cfl, bias, limiter, st);
        if (e == cudaSuccess) e = reverse(m, s1, c - 1, ns);
        used[ns] = false;
        if (e == cudaSuccess) e = reverse(s0, m, c, slot);
        return e;
    }
};

}  // namespace

extern "C" vg_status vg_batch_gradient(vg_batch* b, const double* target_rho, double cfl, int steps, double bias,
                                       int limiter, int checkpoints, double* loss, double* grad_planes,
                                       double* grad_gamma, long* forward_steps, long* adjoint_steps, void* stream) {
    if (!b || !target_rho || steps < 1 || !(cfl > 0.0) || limiter < 0 || limiter > 2)
        return afail(VG_EINVAL, "bad vg_batch_gradient argument");
    if (checkpoints < 1) return afail(VG_EINVAL, "need at least one checkpoint slot (the initial state)");
    checkpoints = std::min(checkpoints, steps);
    cudaStream_t st = (cudaStream_t)stream;
    VA_CUDA(cudaSetDevice(b->device));
    VA_CUDA(ensure_workspace(b, checkpoints));
    const long n = b->total;
    const size_t sbytes = sizeof(double) * 3 * n;
    VA_CUDA(cudaMemcpyAsync(b->d_target, target_rho, sizeof(double) * n, cudaMemcpyHostToDevice, st));
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
    for (int i = 0; i < checkpoints; i++) R.slots.push_back(b->ckpt + (long)i * 3 * n);
    R.used.assign(checkpoints, false);
    R.tmp = b->ckpt + (long)checkpoints * 3 * n;
    b->last_forward_steps = 0;
    b->last_adjoint_steps = 0;
    VA_CUDA(cudaMemcpyAsync(R.slots[0], b->buf[b->cur], sbytes, cudaMemcpyDeviceToDevice, st));
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
        e = cudaMemcpyAsync(grad_planes + ref[v] * n, lam0 + v * n, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && grad_gamma)
        e = cudaMemcpyAsync(grad_gamma, b->d_ggam, sizeof(double) * b->ninst, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return afail(VG_ECUDA, std::string("vg_batch_gradient: ") + cudaGetErrorString(e));
    if (err) return afail(VG_ENAN, "non-finite or non-positive density/pressure produced");
    if (grad_planes)
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
