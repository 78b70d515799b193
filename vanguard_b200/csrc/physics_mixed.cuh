// Mixed FP32/FP64 device models for the VG_MIXED form.
//
// Split of the arithmetic:
//   FP64  conserved cell states and every evolved edge / Richtmyer state (so no state is ever rounded to
//         float); the physical flux function with its pressure recovery from total energy
//         (E - |m|^2 / 2 rho, where the kinetic energy cancels); the limiter's slope ratio; the CFL wave
//         speed; and the cell-update accumulation U + (dt/dx)(F_L - F_R).
//   FP32  flux values, the half-step evolution increment (dt/2dx)(F(x_L) - F(x_R)), and the
//         Lax-Friedrichs, Richtmyer and FORCE combinations.  The update's flux difference F_L - F_R is
//         formed in FP64 from the two FP32 interface fluxes, so the interface terms telescope exactly
//         and mass, momentum and energy are conserved to FP64 round-off.
// No correctly rounded FP64 division is used: 1/rho starts from the hardware reciprocal approximation
// (PTX rcp.approx.ftz.f64, one XU operation and no precision conversion) and is refined by Newton-Raphson
// steps x <- x + x (1 - a x), each of which doubles the number of correct bits.
//
// On B200 the XU pipe that executes reciprocal approximations and every float<->double conversion has a
// quarter of the FP64 pipe's lanes.  The 9-component MHD variant and the HPR solids (EulerMixed's split) evaluate
// the physical flux function in FP64 with FMA and round only its outputs to FP32; the arithmetic that combines
// fluxes (half-step evolution increment, Lax-Friedrichs, Richtmyer and FORCE averages) runs in FP32.  Euler
// (EulerF32), MHD with w = Bz = 0 (MHDF32) and HPR gas (HPRF32) go further: the limited edge states, the evolved
// and Richtmyer states and their fluxes are FP32 (the states are rounded once, after the FP64 slope differences),
// which halves the sweeps' instruction count; FP64 stays in the cell states, the conserved/primitive conversion of
// the stored state with its pressure recovery, the wave speed and the update accumulation.  Each model's `R`
// names the type of its reconstructed states.
#pragma once

#include "physics_fp64.cuh"
#include "physics_hpr.cuh"
#include "vg_common.cuh"

namespace vg {

__device__ __forceinline__ double rcp_approx(double a) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
    return r;
}
__device__ __forceinline__ float rcp_approx_f(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}
// Two FP32 lanes processed by one packed Blackwell instruction (FADD2/FMUL2/FFMA2): the X sweep of the
// Euler mixed form carries two grid rows through its FP32 arithmetic this way, lane x = first row.  Each lane
// is rounded exactly as the scalar operation would be (a - b is fma(b, -1, a), which rounds once).
struct f2 {
    float2 v;
};
__device__ __forceinline__ f2 mk2(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ f2 splat2(float s) { return {make_float2(s, s)}; }
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return fma2(b, splat2(-1.0f), a); }
__device__ __forceinline__ f2 sel2(bool cx, bool cy, f2 a, f2 b) {
    return mk2(cx ? a.v.x : b.v.x, cy ? a.v.y : b.v.y);
}
__device__ __forceinline__ f2 rcp2(f2 a) { return mk2(rcp_approx_f(a.v.x), rcp_approx_f(a.v.y)); }

// 1/a refined by one Newton step: relative error ~2^-44, far below the FP32 rounding of a flux value.
__device__ __forceinline__ double rcp_nr1(double a) {
    double x = rcp_approx(a);
    double e = fma(-a, x, 1.0);
    return fma(x, e, x);
}
// 1/a refined by two Newton steps (full double precision), for the stored state.
__device__ __forceinline__ double rcp_nr2(double a) {
    double x = rcp_approx(a);
    double e = fma(-a, x, 1.0);
    x = fma(x, e, x);
    e = fma(-a, x, 1.0);
    return fma(x, e, x);
}

// ------------------------------------------------------------------------------------------- Euler
template <int NVEL>
struct EulerMixed {
    static constexpr int NW = NVEL + 2;
    static constexpr int NU = NW;
    static constexpr int IE = NU - 1;
    static constexpr bool HAS_Y = NVEL == 2;
    using R = double;  // type of the reconstructed, evolved and Richtmyer states
    static constexpr bool PAIR_X = false;  // X sweep carries two rows per thread in packed FP32 lanes
    struct P {
        double gm1, inv_gm1, gpinf, g, pinf, ch2;
    };
    __device__ static P params(const double* prm, double /*ch*/) {
        double g = prm[0], pinf = prm[1];
        return P{g - 1.0, prm[kInvGm1], g * pinf, g, pinf, 0.0};
    }
    // W -> U in FP64: E = rho |v|^2 / 2 + (p + gamma p_inf) / (gamma - 1)
    __device__ static void cons(const double* W, const P& q, double* U) {
        double rho = W[0], u = W[1], v = (NVEL == 2) ? W[2] : 0.0, p = W[IE];
        U[0] = rho;
        U[1] = rho * u;
        if constexpr (NVEL == 2) U[2] = rho * v;
        double v2 = (NVEL == 2) ? fma(u, u, v * v) : u * u;
        U[IE] = fma(0.5 * rho, v2, (p + q.gpinf) * q.inv_gm1);
    }
    // U -> W in FP64 (final cell update)
    __device__ static void setcons(const double* U, const P& q, double* W) {
        double rho = U[0], inv = rcp_nr2(rho);
        double u = U[1] * inv, v = (NVEL == 2) ? U[2] * inv : 0.0;
        double ke2 = (NVEL == 2) ? fma(U[1], u, U[2] * v) : U[1] * u;  // |m|^2 / rho
        W[0] = rho;
        W[1] = u;
        if constexpr (NVEL == 2) W[2] = v;
        W[IE] = fma(q.gm1, fma(-0.5, ke2, U[IE]), -q.gpinf);
    }
    // Flux of an FP64 state, evaluated in FP64 (pressure recovered from total energy where the kinetic energy
    // cancels) and rounded to FP32 on output.
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, float* F) {
        double inv = rcp_nr1(U[0]);
        double mxd = U[1], myd = (NVEL == 2) ? U[2] : 0.0;
        double un = (AXIS == 0 ? mxd : myd) * inv;
        double ke2 = (NVEL == 2) ? fma(mxd, mxd, myd * myd) * inv : mxd * mxd * inv;
        double p = fma(q.gm1, fma(-0.5, ke2, U[IE]), -q.gpinf);
        if constexpr (AXIS == 0) {
            F[0] = (float)mxd;
            F[1] = (float)fma(mxd, un, p);
            if constexpr (NVEL == 2) F[2] = (float)(myd * un);
        } else {
            F[0] = (float)myd;
            F[1] = (float)(mxd * un);
            F[2] = (float)fma(myd, un, p);
        }
        F[IE] = (float)((U[IE] + p) * un);
    }
    __device__ static double wave(const double* W, const P& q, int dims) {
        double c = sqrt((q.g * (W[IE] + q.pinf)) / W[0]);
        if (dims == 1) return fabs(W[1]) + c;
        double v = (NVEL == 2) ? W[2] : 0.0;
        return fmax(fabs(W[1]), fabs(v)) + c;
    }
    __device__ static void default_state(double* W) {
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 1.0;
        W[IE] = 1.0;
    }
    __device__ static double density(const double* W) { return W[0]; }
    __device__ static double pressure(const double* W) { return W[IE]; }
};

// Euler with FP32 reconstruction: the limited edge states, the half-step evolved states, the Richtmyer state
// and every flux evaluation are FP32 (the limiter works on FP64 slope differences rounded to FP32, since the
// slope floor 1e-5 is below the FP32 resolution of total energy); the cell states, the conserved/primitive
// conversions of the stored state (its pressure recovery from total energy), the wave speed and the update
// accumulation stay FP64 as in EulerMixed.
template <int NVEL>
struct EulerF32 : EulerMixed<NVEL> {
    using Base = EulerMixed<NVEL>;
    using Base::IE;
    using R = float;
    static constexpr bool PAIR_X = true;
    struct P : Base::P {
        float gm1_f, gpinf_f;
    };
    __device__ static P params(const double* prm, double ch) {
        P q;
        static_cast<typename Base::P&>(q) = Base::params(prm, ch);
        q.gm1_f = (float)q.gm1;
        q.gpinf_f = (float)q.gpinf;
        return q;
    }
    template <int AXIS>
    __device__ static void flux(const float* U, const P& q, float* F) {
        float inv = rcp_approx_f(U[0]);
        float mx = U[1], my = (NVEL == 2) ? U[2] : 0.0f;
        float un = (AXIS == 0 ? mx : my) * inv;
        float ke2 = (NVEL == 2) ? fmaf(mx, mx, my * my) * inv : mx * mx * inv;
        float p = fmaf(q.gm1_f, fmaf(-0.5f, ke2, U[IE]), -q.gpinf_f);
        if constexpr (AXIS == 0) {
            F[0] = mx;
            F[1] = fmaf(mx, un, p);
            if constexpr (NVEL == 2) F[2] = my * un;
        } else {
            F[0] = my;
            F[1] = mx * un;
            F[2] = fmaf(my, un, p);
        }
        F[IE] = (U[IE] + p) * un;
    }
    // flux of two states at once, one per lane, with the same operations as flux()
    template <int AXIS>
    __device__ static void flux2(const f2* U, const P& q, f2* F) {
        f2 inv = rcp2(U[0]);
        f2 mx = U[1], my = (NVEL == 2) ? U[2] : splat2(0.0f);
        f2 un = (AXIS == 0 ? mx : my) * inv;
        f2 ke2 = ((NVEL == 2) ? fma2(mx, mx, my * my) : mx * mx) * inv;
        f2 p = fma2(splat2(q.gm1_f), fma2(splat2(-0.5f), ke2, U[IE]), splat2(-q.gpinf_f));
        if constexpr (AXIS == 0) {
            F[0] = mx;
            F[1] = fma2(mx, un, p);
            if constexpr (NVEL == 2) F[2] = my * un;
        } else {
            F[0] = my;
            F[1] = mx * un;
            F[2] = fma2(my, un, p);
        }
        F[IE] = (U[IE] + p) * un;
    }
};

// --------------------------------------------------------------------------------------------- MHD
template <bool FULL>
struct MHDMixed {
    static constexpr int NW = FULL ? 9 : 7;
    static constexpr int NU = NW;
    static constexpr int IP = FULL ? 4 : 3;
    static constexpr int IBX = IP + 1;
    static constexpr int IBY = IP + 2;
    static constexpr int IPSI = NW - 1;
    static constexpr bool HAS_Y = true;
    using R = double;
    static constexpr bool PAIR_X = false;
    struct P {
        double gm1, inv_gm1, gpinf, g, pinf, ch2;
    };
    __device__ static P params(const double* prm, double ch) {
        double g = prm[0], pinf = prm[1];
        return P{g - 1.0, prm[kInvGm1], g * pinf, g, pinf, ch * ch};
    }
    __device__ static double sq3(double a, double b, double c) {
        if constexpr (FULL) return fma(a, a, fma(b, b, c * c));
        else return fma(a, a, b * b);
    }
    __device__ static void cons(const double* W, const P& q, double* U) {
        double rho = W[0], u = W[1], v = W[2], w = FULL ? W[3] : 0.0, p = W[IP];
        double bx = W[IBX], by = W[IBY], bz = FULL ? W[7] : 0.0;
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        if constexpr (FULL) U[3] = rho * w;
        U[IP] = fma(0.5 * rho, sq3(u, v, w), fma(0.5, sq3(bx, by, bz), (p + q.gpinf) * q.inv_gm1));
        U[IBX] = bx;
        U[IBY] = by;
        if constexpr (FULL) U[7] = bz;
        U[IPSI] = W[IPSI];
    }
    __device__ static double pressure_of(const double* U, const P& q, double inv, double& u, double& v, double& w) {
        u = U[1] * inv;
        v = U[2] * inv;
        w = FULL ? U[3] * inv : 0.0;
        double ke2 = FULL ? fma(U[1], u, fma(U[2], v, U[3] * w)) : fma(U[1], u, U[2] * v);
        double b2 = sq3(U[IBX], U[IBY], FULL ? U[7] : 0.0);
        return fma(q.gm1, fma(-0.5, ke2 + b2, U[IP]), -q.gpinf);
    }
    __device__ static void setcons(const double* U, const P& q, double* W) {
        double inv = rcp_nr2(U[0]), u, v, w;
        double p = pressure_of(U, q, inv, u, v, w);
        W[0] = U[0];
        W[1] = u;
        W[2] = v;
        if constexpr (FULL) W[3] = w;
        W[IP] = p;
        W[IBX] = U[IBX];
        W[IBY] = U[IBY];
        if constexpr (FULL) W[7] = U[7];
        W[IPSI] = U[IPSI];
    }
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, float* F) {
        double inv = rcp_nr1(U[0]), u, v, w;
        double p = pressure_of(U, q, inv, u, v, w);
        double bx = U[IBX], by = U[IBY], bz = FULL ? U[7] : 0.0, psi = U[IPSI];
        double pt = fma(0.5, sq3(bx, by, bz), p);  // total pressure
        double vb = FULL ? fma(u, bx, fma(v, by, w * bz)) : fma(u, bx, v * by);
        if constexpr (AXIS == 0) {
            double mx = U[1];
            F[0] = (float)mx;
            F[1] = (float)(fma(mx, u, pt) - bx * bx);
            F[2] = (float)fma(mx, v, -bx * by);
            if constexpr (FULL) F[3] = (float)fma(mx, w, -bx * bz);
            F[IP] = (float)fma(U[IP] + pt, u, -vb * bx);
            F[IBX] = (float)psi;
            F[IBY] = (float)fma(by, u, -bx * v);
            if constexpr (FULL) F[7] = (float)fma(bz, u, -bx * w);
            F[IPSI] = (float)(q.ch2 * bx);
        } else {
            double my = U[2];
            F[0] = (float)my;
            F[1] = (float)fma(my, u, -by * bx);
            F[2] = (float)(fma(my, v, pt) - by * by);
            if constexpr (FULL) F[3] = (float)fma(my, w, -by * bz);
            F[IP] = (float)fma(U[IP] + pt, v, -vb * by);
            F[IBX] = (float)fma(bx, v, -by * u);
            F[IBY] = (float)psi;
            if constexpr (FULL) F[7] = (float)fma(bz, v, -by * w);
            F[IPSI] = (float)(q.ch2 * by);
        }
    }
    __device__ static double fast(const double* W, const P& q, double bn) {
        double rho = W[0], bx = W[IBX], by = W[IBY], bz = FULL ? W[7] : 0.0;
        double c2 = (q.g * (W[IP] + q.pinf)) / rho;
        double a2 = sq3(bx, by, bz) / rho;
        double s = c2 + a2;
        return sqrt(0.5 * (s + sqrt(fmax(s * s - 4.0 * c2 * bn * bn / rho, 0.0))));
    }
    __device__ static double wave(const double* W, const P& q, int dims) {
        if (dims == 1) return fabs(W[1]) + fast(W, q, W[IBX]);
        return fmax(fabs(W[1]), fabs(W[2])) + fmax(fast(W, q, W[IBX]), fast(W, q, W[IBY]));
    }
    __device__ static void default_state(double* W) {
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 1.0;
        W[IP] = 1.0;
    }
    __device__ static double density(const double* W) { return W[0]; }
    __device__ static double pressure(const double* W) { return W[IP]; }
};

// MHD (GLM, w = Bz = 0) with FP32 reconstruction, as EulerF32 for Euler: the limited edge states, the half-step
// evolved states, the Richtmyer state and every flux evaluation (with its pressure p = (gamma - 1)(E - (|m|^2 / rho
// + |B|^2) / 2) - gamma p_inf) are FP32; the cell states, the conversions of the stored state (its pressure
// recovery from total energy), the fast-magnetosonic CFL speed and the update accumulation stay FP64 as in
// MHDMixed.  The X sweep carries two rows per thread through packed FP32x2 arithmetic (flux2).
struct MHDF32 : MHDMixed<false> {
    using Base = MHDMixed<false>;
    using R = float;
    static constexpr bool PAIR_X = true;
    struct P : Base::P {
        float gm1_f, gpinf_f, ch2_f;
    };
    __device__ static P params(const double* prm, double ch) {
        P q;
        static_cast<Base::P&>(q) = Base::params(prm, ch);
        q.gm1_f = (float)q.gm1;
        q.gpinf_f = (float)q.gpinf;
        q.ch2_f = (float)q.ch2;
        return q;
    }
    // W = (rho, u, v, p, Bx, By, psi), U = (rho, mx, my, E, Bx, By, psi)
    template <int AXIS>
    __device__ static void flux(const float* U, const P& q, float* F) {
        const float inv = rcp_approx_f(U[0]);
        const float mx = U[1], my = U[2], E = U[3], bx = U[4], by = U[5], psi = U[6];
        const float u = mx * inv, v = my * inv;
        const float ke2 = fmaf(mx, u, my * v);
        const float b2 = fmaf(bx, bx, by * by);
        const float p = fmaf(q.gm1_f, fmaf(-0.5f, ke2 + b2, E), -q.gpinf_f);
        const float pt = fmaf(0.5f, b2, p);
        const float vb = fmaf(u, bx, v * by);
        if constexpr (AXIS == 0) {
            F[0] = mx;
            F[1] = fmaf(mx, u, pt) - bx * bx;
            F[2] = fmaf(mx, v, -bx * by);
            F[3] = fmaf(E + pt, u, -vb * bx);
            F[4] = psi;
            F[5] = fmaf(by, u, -bx * v);
            F[6] = q.ch2_f * bx;
        } else {
            F[0] = my;
            F[1] = fmaf(my, u, -by * bx);
            F[2] = fmaf(my, v, pt) - by * by;
            F[3] = fmaf(E + pt, v, -vb * by);
            F[4] = fmaf(bx, v, -by * u);
            F[5] = psi;
            F[6] = q.ch2_f * by;
        }
    }
    // flux of two states at once, one per lane, with the same operations as flux()
    template <int AXIS>
    __device__ static void flux2(const f2* U, const P& q, f2* F) {
        const f2 inv = rcp2(U[0]);
        const f2 mx = U[1], my = U[2], E = U[3], bx = U[4], by = U[5], psi = U[6];
        const f2 u = mx * inv, v = my * inv;
        const f2 ke2 = fma2(mx, u, my * v);
        const f2 b2 = fma2(bx, bx, by * by);
        const f2 p = fma2(splat2(q.gm1_f), fma2(splat2(-0.5f), ke2 + b2, E), splat2(-q.gpinf_f));
        const f2 pt = fma2(splat2(0.5f), b2, p);
        const f2 vb = fma2(u, bx, v * by);
        const f2 neg = splat2(-1.0f);
        if constexpr (AXIS == 0) {
            F[0] = mx;
            F[1] = fma2(mx, u, pt) - bx * bx;
            F[2] = fma2(mx, v, neg * (bx * by));
            F[3] = fma2(E + pt, u, neg * (vb * bx));
            F[4] = psi;
            F[5] = fma2(by, u, neg * (bx * v));
            F[6] = splat2(q.ch2_f) * bx;
        } else {
            F[0] = my;
            F[1] = fma2(my, u, neg * (by * bx));
            F[2] = fma2(my, v, pt) - by * by;
            F[3] = fma2(E + pt, v, neg * (vb * by));
            F[4] = fma2(bx, v, neg * (by * u));
            F[5] = psi;
            F[6] = splat2(q.ch2_f) * by;
        }
    }
};

// ---------------------------------------------------------------------------------------------- HPR
// HPR (GPR) in the mixed form.  The state and its conversions, the pressure recovered from total energy inside the
// flux, the acoustic-tensor CFL speed and the relaxation source (run by the exact forcing kernel) are the exact
// model's FP64 formulas (here compiled with FMA contraction); each flux value leaves in FP32 for the FP32
// half-step and FORCE combinations.
template <bool SOLID>
struct HPRMixedT {
    static constexpr int NW = 17;
    static constexpr int NU = 17;
    static constexpr bool HAS_Y = true;
    static constexpr int J_PLANE = 14;
    using R = double;
    static constexpr bool PAIR_X = false;
    using P = typename HPRModel<SOLID>::P;
    __device__ static P params(const double* prm, double ch) { return HPRModel<SOLID>::params(prm, ch); }
    __device__ static bool positive_pressure(const P& q) { return HPRModel<SOLID>::positive_pressure(q); }
    __device__ static void cons(const double* W, const P& q, double* U) { HPRModel<SOLID>::cons(W, q, U); }
    __device__ static void setcons(const double* U, const P& q, double* W) { HPRModel<SOLID>::setcons(U, q, W); }
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, float* F) {
        double Fd[17];
        HPRModel<SOLID>::template flux<AXIS>(U, q, Fd);
#pragma unroll
        for (int i = 0; i < 17; i++) F[i] = (float)Fd[i];
    }
    __device__ static double wave(const double* W, const P& q, int dims) { return HPRModel<SOLID>::wave(W, q, dims); }
    __device__ static void default_state(double* W) { HPRModel<SOLID>::default_state(W); }
    __device__ static double density(const double* W) { return W[0]; }
    __device__ static double pressure(const double* W) { return W[1]; }
};
// HPR (GPR) gas with FP32 reconstruction, as EulerF32 and MHDF32: the limited edge states, the half-step evolved
// states, the Richtmyer state and every flux evaluation are FP32 -- the stress c_s^2 rho A^T A dev(A^T A), the
// pressure recovered inside the flux from total energy (StiffenedGas: p = (gamma - 1)(rho e - p_inf) - p_inf with
// e = E - |v|^2 / 2 - c_s^2 |dev(A^T A)|^2 / 4 [- alpha^2 |J|^2 / 2]) and the temperature of the heat flux.  The cell
// states, the conversions of the stored state (its pressure recovery), the acoustic-tensor CFL speed, the update
// accumulation and the relaxation source (the exact forcing and stiff-relaxation kernels) stay FP64
// (HPR/hprstatevector.cpp:164-298 for the fluxes).
struct HPRF32 : HPRMixedT<false> {
    using Base = HPRMixedT<false>;
    using R = float;
    static constexpr bool PAIR_X = false;
    struct P : Base::P {
        float gm1_f, pinf_f, cs2_f, qcs2_f, ha2_f, a2_f, tref_f, inv_gm1cv_f;
    };
    __device__ static P params(const double* prm, double ch) {
        P q;
        static_cast<Base::P&>(q) = Base::params(prm, ch);
        q.gm1_f = (float)(q.g - 1.0);
        q.pinf_f = (float)q.pinf;
        q.cs2_f = (float)(q.cs * q.cs);
        q.qcs2_f = (float)(0.25 * (q.cs * q.cs));
        q.ha2_f = (float)(0.5 * (q.alpha * q.alpha));
        q.a2_f = (float)(q.alpha * q.alpha);
        q.tref_f = (float)q.Tref;
        q.inv_gm1cv_f = (float)(1.0 / ((q.g - 1.0) * q.cv));
        return q;
    }
    // U = (rho, rho E, A (9, row-major), rho u, rho v, rho w, rho Jx, rho Jy, rho Jz)
    template <int AXIS>
    __device__ static void flux(const float* U, const P& q, float* F) {
        const float rho = U[0];
        const float inv = rcp_approx_f(rho);
        float A[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) A[i][j] = U[2 + 3 * i + j];
        // D = dev(A^T A)
        float D[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) D[i][j] = fmaf(A[0][i], A[0][j], fmaf(A[1][i], A[1][j], A[2][i] * A[2][j]));
        const float third = (D[0][0] + D[1][1] + D[2][2]) * (1.0f / 3.0f);
        D[0][0] -= third;
        D[1][1] -= third;
        D[2][2] -= third;
        // row AXIS of A^T (A D): (A^T A D)[AXIS][j] = sum_k G[AXIS][k] D[k][j], G = A^T A = D + third I
        float s[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            float acc = third * D[AXIS][j];
#pragma unroll
            for (int k = 0; k < 3; k++) acc = fmaf(D[AXIS][k], D[k][j], acc);
            s[j] = (q.cs2_f * rho) * acc;  // -sigma[AXIS][j]
        }
        float dd = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) dd = fmaf(D[i][j], D[i][j], dd);
        const float mx = U[11], my = U[12], mz = U[13];
        const float u = mx * inv, v = my * inv, w = mz * inv;
        const float E = U[1] * inv;
        float e = E - fmaf(0.5f, fmaf(u, u, fmaf(v, v, w * w)), q.qcs2_f * dd);
        float jx = 0.0f, jy = 0.0f, jz = 0.0f;
        if (q.thermal) {
            jx = U[14] * inv;
            jy = U[15] * inv;
            jz = U[16] * inv;
            e = e - q.ha2_f * fmaf(jx, jx, fmaf(jy, jy, jz * jz));
        }
        const float p = fmaf(q.gm1_f, fmaf(rho, e, -q.pinf_f), -q.pinf_f);
        const float un = AXIS == 0 ? u : v;
        const float mn = AXIS == 0 ? mx : my;
#pragma unroll
        for (int i = 0; i < 17; i++) F[i] = 0.0f;
        F[0] = mn;
        F[1] = fmaf(U[1] + p, un, fmaf(s[0], u, fmaf(s[1], v, s[2] * w)));
        F[11] = fmaf(mx, un, s[0]);
        F[12] = fmaf(my, un, s[1]);
        F[13] = fmaf(mz, un, s[2]);
        F[11 + AXIS] += p;
#pragma unroll
        for (int i = 0; i < 3; i++) F[2 + 3 * i + AXIS] = fmaf(A[i][0], u, fmaf(A[i][1], v, A[i][2] * w));
        if (q.thermal) {
            const float T = fmaf(p + q.pinf_f, inv * q.inv_gm1cv_f, q.tref_f);
            F[1] = fmaf(T * q.a2_f, AXIS == 0 ? jx : jy, F[1]);
            F[14] = U[14] * un;
            F[15] = U[15] * un;
            F[16] = U[16] * un;
            F[14 + AXIS] += T;
        }
    }
};

// The Euler two-material models in the mixed form: FP64 states and flux function (its pressure
// recovery from total energy), flux values rounded to FP32, FP32 flux combinations (EulerMixed's split for MHD
// and HPR).
template <class F64>
struct TwoMaterialMixed {
    static constexpr bool ROUNDTRIP_EVOLVED = true;  // the stored form clamps alpha1 and rebuilds rho
    static constexpr int NW = F64::NW;
    static constexpr int NU = F64::NU;
    static constexpr bool HAS_Y = true;
    using R = double;
    static constexpr bool PAIR_X = false;
    using P = typename F64::P;
    __device__ static P params(const double* prm, double ch) { return F64::params(prm, ch); }
    __device__ static void cons(const double* W, const P& q, double* U) { F64::cons(W, q, U); }
    __device__ static void setcons(const double* U, const P& q, double* W) { F64::setcons(U, q, W); }
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, float* F) {
        double Fd[NU];
        F64::template flux<AXIS>(U, q, Fd);
#pragma unroll
        for (int i = 0; i < NU; i++) F[i] = (float)Fd[i];
    }
    __device__ static double wave(const double* W, const P& q, int dims) { return F64::wave(W, q, dims); }
    __device__ static void default_state(double* W) { F64::default_state(W); }
    __device__ static double density(const double* W) { return F64::density(W); }
    __device__ static double pressure(const double* W) { return F64::pressure(W); }
};
using ReducedMixed = TwoMaterialMixed<EulerReducedF64>;

using HPRSolidMixed = HPRMixedT<true>;

}  // namespace vg
