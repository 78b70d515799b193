// Exact-FP64 device restatement of the Euler and ideal-MHD (GLM) models.
//
// Every expression keeps the reference's association order so that, compiled with -fmad=false (no
// FMA contraction) and IEEE division/sqrt, the device reproduces the reference's x86-64 results bit for
// bit.  Components that stay identically zero (Euler w, MHD w and Bz) or exactly 1 (Euler lambda) are not
// carried; the host only selects these reduced variants when the input satisfies that, and the dropped
// terms are exact additive zeros in every expression they appear in.
#pragma once

#include "vg_common.cuh"

namespace vg {

// ------------------------------------------------------------------------------------------- Euler
// Stored primitives W = (rho, u, [v], p); conserved U = (rho, rho u, [rho v], E).
// NVEL = 1 (1D with v == 0) or 2.  Params: params[0] = gamma, params[1] = p_inf.
template <int NVEL>
struct EulerF64 {
    static constexpr int NW = NVEL + 2;
    static constexpr int NU = NW;
    static constexpr int IE = NU - 1;  // energy / pressure slot
    static constexpr bool HAS_Y = NVEL == 2;
    static constexpr bool HAS_SOURCE = false;
    struct P {
        double g, pinf, ch2;
    };
    __device__ static P params(const double* prm, double /*ch*/) { return P{prm[0], prm[1], 0.0}; }

    // EulerEquationOfState::computeSpecificInternalEnergy (Euler/eulerequationofstate.cpp:7-13)
    __device__ static double e_of(double rho, double p, const P& q) { return (p + (q.g * q.pinf)) / ((q.g - 1) * rho); }
    // EulerEquationOfState::computePressure (Euler/eulerequationofstate.cpp:15-21)
    __device__ static double p_of(double rho, double e, const P& q) { return ((e * (q.g - 1)) * rho) - (q.g * q.pinf); }

    __device__ static double vsq(double u, double v) {
        if constexpr (NVEL == 2) return (u * u) + (v * v);
        else return u * u;
    }

    // EulerStateVector::computeConservedVariableVector / computeTotalEnergy (Euler/eulerstatevector.cpp:78-91, :192-198)
    __device__ static void cons(const double* W, const P& q, double* U) {
        double rho = W[0], u = W[1], v = (NVEL == 2) ? W[2] : 0.0, p = W[IE];
        U[0] = rho;
        U[1] = rho * u;
        if constexpr (NVEL == 2) U[2] = rho * v;
        U[IE] = rho * ((0.5 * vsq(u, v)) + e_of(rho, p, q));
    }
    // EulerStateVector::setConservedVariableVector (Euler/eulerstatevector.cpp:47-61)
    __device__ static void setcons(const double* U, const P& q, double* W) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = 0.0;
        if constexpr (NVEL == 2) v = U[2] / rho;
        double e = (U[IE] / rho) - (0.5 * vsq(u, v));
        W[0] = rho;
        W[1] = u;
        if constexpr (NVEL == 2) W[2] = v;
        W[IE] = p_of(rho, e, q);
    }
    // EulerStateVector::compute{X,Y}FluxVector (Euler/eulerstatevector.cpp:93-120, :127-154)
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        double rho = U[0];
        double u = U[1] / rho;
        double v = 0.0;
        if constexpr (NVEL == 2) v = U[2] / rho;
        double E = U[IE] / rho;
        double e = E - (0.5 * vsq(u, v));
        double p = p_of(rho, e, q);
        if constexpr (AXIS == 0) {
            F[0] = rho * u;
            F[1] = (rho * (u * u)) + p;
            if constexpr (NVEL == 2) F[2] = rho * (u * v);
            F[IE] = (rho * (u * E)) + (u * p);
        } else {
            F[0] = rho * v;
            F[1] = rho * (v * u);
            F[2] = (rho * (v * v)) + p;
            F[IE] = (rho * (v * E)) + (v * p);
        }
    }
    // Solvers::computeMaximumWaveSpeed{,2D} per-cell terms (Solvers/solvers.cpp:259-276, :318-339)
    __device__ static double wave(const double* W, const P& q, int dims) {
        double c = sqrt((q.g * (W[IE] + q.pinf)) / W[0]);
        if (dims == 1) return fabs(W[1]) + c;
        double v = (NVEL == 2) ? W[2] : 0.0;
        return std_max(fabs(W[1]), fabs(v)) + c;
    }
    // EulerStateVector() (Euler/eulerstatevector.cpp:3-12)
    __device__ static void default_state(double* W) {
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 1.0;
        W[IE] = 1.0;
    }
    __device__ static double density(const double* W) { return W[0]; }
    __device__ static double pressure(const double* W) { return W[IE]; }
};

// --------------------------------------------------------------------------------------------- MHD
// FULL: W = (rho, u, v, w, p, Bx, By, Bz, psi), U = (rho, mx, my, mz, E, Bx, By, Bz, psi).
// reduced: W = (rho, u, v, p, Bx, By, psi),    U = (rho, mx, my, E, Bx, By, psi)   (w == Bz == 0).
// Params: params[0] = gamma, params[1] = p_inf; c_h comes from the control block each step.
template <bool FULL>
struct MHDF64 {
    static constexpr int NW = FULL ? 9 : 7;
    static constexpr int NU = NW;
    static constexpr int IP = FULL ? 4 : 3;   // p / E slot
    static constexpr int IBX = IP + 1;
    static constexpr int IBY = IP + 2;
    static constexpr int IPSI = NW - 1;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = true;
    struct P {
        double g, pinf, ch2, ch;
    };
    __device__ static P params(const double* prm, double ch) { return P{prm[0], prm[1], ch * ch, ch}; }

    // MHDStateVector::computeSourceTermVector (MHD/mhdstatevector.cpp:222-234): GLM damping of psi with the
    // parabolic damping c_p = sqrt(c_h * 0.18) of MHDMaterialParameters::configureParabolicDamping
    // (MHD/mhdmaterialparameters.cpp:21-36), c_h being this step's maximum wave speed
    __device__ static void source(const double* U, const P& q, double* S) {
#pragma unroll
        for (int i = 0; i < NU; i++) S[i] = 0.0;
        const double cp = sqrt(q.ch * 0.18);
        S[IPSI] = (-(q.ch2 / (cp * cp))) * U[IPSI];
    }

    __device__ static double e_of(double rho, double p, const P& q) { return (p + (q.g * q.pinf)) / ((q.g - 1) * rho); }
    __device__ static double p_of(double rho, double e, const P& q) { return ((e * (q.g - 1)) * rho) - (q.g * q.pinf); }

    __device__ static double sq3(double a, double b, double c) {
        if constexpr (FULL) return ((a * a) + (b * b)) + (c * c);
        else return (a * a) + (b * b);
    }

    // MHDStateVector::computeConservedVariableVector + computeTotalEnergy (MHD/mhdstatevector.cpp:89-106, :236-245)
    __device__ static void cons(const double* W, const P& q, double* U) {
        double rho = W[0], u = W[1], v = W[2], w = FULL ? W[3] : 0.0, p = W[IP];
        double bx = W[IBX], by = W[IBY], bz = FULL ? W[7] : 0.0;
        double hydro = rho * ((0.5 * sq3(u, v, w)) + e_of(rho, p, q));
        U[0] = rho;
        U[1] = rho * u;
        U[2] = rho * v;
        if constexpr (FULL) U[3] = rho * w;
        U[IP] = hydro + (0.5 * sq3(bx, by, bz));
        U[IBX] = bx;
        U[IBY] = by;
        if constexpr (FULL) U[7] = bz;
        U[IPSI] = W[IPSI];
    }
    // MHDStateVector::setConservedVariableVector (MHD/mhdstatevector.cpp:49-68)
    __device__ static void setcons(const double* U, const P& q, double* W) {
        double rho = U[0];
        double u = U[1] / rho, v = U[2] / rho, w = 0.0;
        if constexpr (FULL) w = U[3] / rho;
        double bx = U[IBX], by = U[IBY], bz = FULL ? U[7] : 0.0;
        double E = (U[IP] - (0.5 * sq3(bx, by, bz))) / rho;
        double e = E - (0.5 * sq3(u, v, w));
        W[0] = rho;
        W[1] = u;
        W[2] = v;
        if constexpr (FULL) W[3] = w;
        W[IP] = p_of(rho, e, q);
        W[IBX] = bx;
        W[IBY] = by;
        if constexpr (FULL) W[7] = bz;
        W[IPSI] = U[IPSI];
    }
    // MHDStateVector::compute{X,Y}FluxVector (MHD/mhdstatevector.cpp:108-158, :165-215); v.B is
    // VectorAlgebra::computeDotProduct summed from 0.0 (Mathematics/vectoralgebra.cpp:38-49).
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        double rho = U[0];
        double u = U[1] / rho, v = U[2] / rho, w = 0.0;
        if constexpr (FULL) w = U[3] / rho;
        double bx = U[IBX], by = U[IBY], bz = FULL ? U[7] : 0.0, psi = U[IPSI];
        double b2 = sq3(bx, by, bz);
        double E = U[IP];
        double hydroE = (E - (0.5 * b2)) / rho;
        double e = hydroE - (0.5 * sq3(u, v, w));
        double p = p_of(rho, e, q);
        double vb = (0.0 + (u * bx)) + (v * by);
        if constexpr (FULL) vb = vb + (w * bz);
        if constexpr (AXIS == 0) {
            F[0] = rho * u;
            F[1] = (((rho * (u * u)) + p) + (0.5 * b2)) - (bx * bx);
            F[2] = (rho * (u * v)) - (bx * by);
            if constexpr (FULL) F[3] = (rho * (u * w)) - (bx * bz);
            F[IP] = (((E + p) + (0.5 * b2)) * u) - (vb * bx);
            F[IBX] = psi;
            F[IBY] = (by * u) - (bx * v);
            if constexpr (FULL) F[7] = (bz * u) - (bx * w);
            F[IPSI] = q.ch2 * bx;
        } else {
            F[0] = rho * v;
            F[1] = (rho * (v * u)) - (by * bx);
            F[2] = (((rho * (v * v)) + p) + (0.5 * b2)) - (by * by);
            if constexpr (FULL) F[3] = (rho * (v * w)) - (by * bz);
            F[IP] = (((E + p) + (0.5 * b2)) * v) - (vb * by);
            F[IBX] = (bx * v) - (by * u);
            F[IBY] = psi;
            if constexpr (FULL) F[7] = (bz * v) - (by * w);
            F[IPSI] = q.ch2 * by;
        }
    }
    // MHDWaveSpeeds::compute{X,Y}FastMagnetoAcousticSpeed (MHD/mhdwavespeeds.cpp:43-63); the Alfven speed
    // is computeNorm(B) / sqrt(rho) with the norm summed from 0.0 (:7-15).
    __device__ static double fast(const double* W, const P& q, double bn) {
        double rho = W[0], bx = W[IBX], by = W[IBY], bz = FULL ? W[7] : 0.0;
        double c = sqrt((q.g * (W[IP] + q.pinf)) / rho);
        double nb = (0.0 + (bx * bx)) + (by * by);
        if constexpr (FULL) nb = nb + (bz * bz);
        double a = sqrt(nb) / sqrt(rho);
        double c2 = c * c, a2 = a * a;
        return sqrt(0.5 * ((c2 + a2) + sqrt(((c2 + a2) * (c2 + a2)) - (4.0 * ((c2 * (bn * bn)) / rho)))));
    }
    // MHDSolvers::computeMaximumWaveSpeed{,2D} per-cell terms (Solvers/mhdsolvers.cpp:286-303, :365-388)
    __device__ static double wave(const double* W, const P& q, int dims) {
        if (dims == 1) return fabs(W[1]) + fabs(fast(W, q, W[IBX]));
        return std_max(fabs(W[1]), fabs(W[2])) + std_max(fabs(fast(W, q, W[IBX])), fabs(fast(W, q, W[IBY])));
    }
    // MHDStateVector() (MHD/mhdstatevector.cpp:3-16)
    __device__ static void default_state(double* W) {
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 1.0;
        W[IP] = 1.0;
    }
    __device__ static double density(const double* W) { return W[0]; }
    __device__ static double pressure(const double* W) { return W[IP]; }
};

// ------------------------------------------------------------------------------- Euler reduced two-material
// EulerReducedStateVector (Euler/Multiphysics/eulerreducedstatevector.cpp) with w == 0 (the host checks it; every w
// term is an exact additive zero):
// W = (alpha1, u, v, rho1, rho2, p), U = (rho, rho alpha1, rho u, rho v, alpha1 rho1, alpha2 rho2, rho E).
// Params: {gamma1, p_inf1, gamma2, p_inf2}.  Every volume fraction the model derives or uses is clamped to
// [0.001, 0.999] (:47-58, :99-108, :131-147).
struct EulerReducedF64 {
    static constexpr int NW = 6;
    static constexpr int NU = 7;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = false;
    struct P {
        double g1, pinf1, g2, pinf2, ch2;
    };
    __device__ static P params(const double* prm, double /*ch*/) { return P{prm[0], prm[1], prm[2], prm[3], 0.0}; }

    __device__ static double clamp_alpha(double a) {
        if (a < 0.001) return 0.001;
        if (a > 0.999) return 0.999;
        return a;
    }
    // EulerEquationOfState::computeSpecificInternalEnergy / computePressure / computeSoundSpeed
    // (Euler/eulerequationofstate.cpp:7-29) of material (g, pinf)
    __device__ static double e_of(double rho, double p, double g, double pinf) { return (p + (g * pinf)) / ((g - 1) * rho); }
    __device__ static double p_of(double rho, double e, double g, double pinf) { return ((e * (g - 1)) * rho) - (g * pinf); }
    __device__ static double c_of(double rho, double p, double g, double pinf) { return sqrt((g * (p + pinf)) / rho); }

    // EulerReducedStateVector::computeConservedVariableVector (:96-129)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double u = W[1], v = W[2], r1 = W[3], r2 = W[4], p = W[5];
        const double rho = (a1 * r1) + (a2 * r2);
        U[0] = rho;
        U[1] = rho * a1;
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = a1 * r1;
        U[5] = a2 * r2;
        const double v2 = (u * u) + (v * v);
        const double E1 = e_of(rho, p, q.g1, q.pinf1) + (0.5 * v2), E2 = e_of(rho, p, q.g2, q.pinf2) + (0.5 * v2);
        U[6] = rho * ((a1 * E1) + (a2 * E2));
    }
    // EulerReducedStateVector::setConservedVariableVector (:43-73)
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho;
        const double e = (U[6] / rho) - (0.5 * ((u * u) + (v * v)));
        W[0] = a1;
        W[1] = u;
        W[2] = v;
        W[3] = U[4] / a1;
        W[4] = U[5] / a2;
        W[5] = (a1 * p_of(rho, e, q.g1, q.pinf1)) + (a2 * p_of(rho, e, q.g2, q.pinf2));
    }
    // EulerReducedStateVector::compute{X,Y}FluxVector(vector, params, params) (:131-180, :187-236)
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho;
        const double r1 = U[4] / a1, r2 = U[5] / a2;
        const double E = U[6] / rho;
        const double e = E - (0.5 * ((u * u) + (v * v)));
        const double p = (a1 * p_of(rho, e, q.g1, q.pinf1)) + (a2 * p_of(rho, e, q.g2, q.pinf2));
        const double un = AXIS == 0 ? u : v;
        F[0] = rho * un;
        F[1] = rho * (un * a1);
        F[2] = rho * (un * u);
        F[3] = rho * (un * v);
        if constexpr (AXIS == 0) F[2] = F[2] + p;
        else F[3] = F[3] + p;
        F[4] = a1 * (r1 * un);
        F[5] = a2 * (r2 * un);
        F[6] = (rho * (un * E)) + (un * p);
    }
    // Solvers::computeMaximumWaveSpeed{,2D} of the reduced model (Solvers/solvers.cpp:298-316, :365-387)
    __device__ static double wave(const double* W, const P& q, int dims) {
        const double c = std_max(c_of(W[3], W[5], q.g1, q.pinf1), c_of(W[4], W[5], q.g2, q.pinf2));
        if (dims == 1) return fabs(W[1]) + c;
        return std_max(fabs(W[1]), fabs(W[2])) + c;
    }
    // EulerReducedStateVector() (:3-14)
    __device__ static void default_state(double* W) {
        W[0] = 0.999;
        W[1] = 0.0;
        W[2] = 0.0;
        W[3] = 1.0;
        W[4] = 1.0;
        W[5] = 1.0;
    }
    // the smaller material density (bad-state check: both must stay positive) and the interface pressure
    __device__ static double density(const double* W) { return W[3] < W[4] ? W[3] : W[4]; }
    __device__ static double pressure(const double* W) { return W[5]; }
};

// ------------------------------------------------------------------------- Euler multiphysics two-material
// EulerMultiphysicsStateVector (Euler/Multiphysics/eulermultiphysicsstatevector.cpp) with w == 0 (host-checked):
// W = (alpha1, u, v, rho1, p1, rho2, p2), U = (rho, rho alpha1, rho u, rho v, alpha1 rho1, alpha1 rho1 E1,
// alpha2 rho2, alpha2 rho2 E2).  Params as EulerReducedF64's; its volume fractions are clamped the same way.
struct EulerMultiphysicsF64 {
    static constexpr int NW = 7;
    static constexpr int NU = 8;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = false;
    using P = EulerReducedF64::P;
    using R2 = EulerReducedF64;
    __device__ static P params(const double* prm, double ch) { return R2::params(prm, ch); }

    // computeConservedVariableVector (:99-128) with computeMaterial{1,2}TotalEnergy (:255-260, :277-282)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = R2::clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double u = W[1], v = W[2], r1 = W[3], p1 = W[4], r2 = W[5], p2 = W[6];
        const double rho = (a1 * r1) + (a2 * r2);
        const double v2 = (u * u) + (v * v);
        U[0] = rho;
        U[1] = rho * a1;
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = a1 * r1;
        U[5] = a1 * (r1 * ((0.5 * v2) + R2::e_of(r1, p1, q.g1, q.pinf1)));
        U[6] = a2 * r2;
        U[7] = a2 * (r2 * ((0.5 * v2) + R2::e_of(r2, p2, q.g2, q.pinf2)));
    }
    // setConservedVariableVector (:46-79); its |v|^2 term w + w (meant w * w) is an exact zero here
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho;
        const double r1 = U[4] / a1;
        const double v2 = (u * u) + (v * v);
        const double e1 = (U[5] / (r1 * a1)) - (0.5 * v2);
        const double r2 = U[6] / a2;
        const double e2 = (U[7] / (r2 * a2)) - (0.5 * v2);
        W[0] = a1;
        W[1] = u;
        W[2] = v;
        W[3] = r1;
        W[4] = R2::p_of(r1, e1, q.g1, q.pinf1);
        W[5] = r2;
        W[6] = R2::p_of(r2, e2, q.g2, q.pinf2);
    }
    // compute{X,Y}FluxVector(vector, params, params) (:130-183, :190-243)
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho;
        const double r1 = U[4] / a1;
        const double v2 = (u * u) + (v * v);
        const double E1 = U[5] / (a1 * r1);
        const double p1 = R2::p_of(r1, E1 - (0.5 * v2), q.g1, q.pinf1);
        const double r2 = U[6] / a2;
        const double E2 = U[7] / (a2 * r2);
        const double p2 = R2::p_of(r2, E2 - (0.5 * v2), q.g2, q.pinf2);
        const double un = AXIS == 0 ? u : v;
        const double pm = (a1 * p1) + (a2 * p2);
        F[0] = rho * un;
        F[1] = rho * (un * a1);
        F[2] = rho * (un * u);
        F[3] = rho * (un * v);
        if constexpr (AXIS == 0) F[2] = F[2] + pm;
        else F[3] = F[3] + pm;
        F[4] = a1 * (r1 * un);
        F[5] = a1 * ((r1 * (un * E1)) + (un * p1));
        F[6] = a2 * (r2 * un);
        F[7] = a2 * ((r2 * (un * E2)) + (un * p2));
    }
    // Solvers::computeMaximumWaveSpeed{,2D} (Solvers/solvers.cpp:278-296, :345-363)
    __device__ static double wave(const double* W, const P& q, int dims) {
        const double c = std_max(R2::c_of(W[3], W[4], q.g1, q.pinf1), R2::c_of(W[5], W[6], q.g2, q.pinf2));
        if (dims == 1) return fabs(W[1]) + c;
        return std_max(fabs(W[1]), fabs(W[2])) + c;
    }
    // EulerMultiphysicsStateVector() (:3-15)
    __device__ static void default_state(double* W) {
        W[0] = 0.999;
        W[1] = 0.0;
        W[2] = 0.0;
        W[3] = 1.0;
        W[4] = 1.0;
        W[5] = 1.0;
        W[6] = 1.0;
    }
    // the smaller material density and the smaller material pressure (bad-state check)
    __device__ static double density(const double* W) { return W[3] < W[5] ? W[3] : W[5]; }
    __device__ static double pressure(const double* W) { return W[4] < W[6] ? W[4] : W[6]; }
};

// ------------------------------------------------------------------------------- MHD reduced two-material
// MHDReducedStateVector (MHD/Multiphysics/mhdreducedstatevector.cpp) with every plane carried:
// W = (alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi), U = (rho, rho alpha1, rho u, rho v, rho w, alpha1 rho1,
// alpha2 rho2, E, Bx, By, Bz, psi).  Params: {gamma1, p_inf1, gamma2, p_inf2}; c_h, the hyperbolic wave speed of both
// materials, is this step's maximum wave speed as MHDSecondOrderSolver::solve{,2D} sets it (Solvers/
// mhdsecondordersolver.cpp:454-460), with the parabolic damping c_p = sqrt(c_h * 0.18) (MHD/mhdmaterialparameters.cpp:
// 31-34).  The GLM coefficients enter as the volume-fraction mixtures of c_h^2 and c_p^2, as the reference forms them.
struct MHDReducedF64 {
    static constexpr int NW = 11;
    static constexpr int NU = 12;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = true;
    // GLM forcing at 8 resident blocks (128 registers): 7.6 % faster per 2048^2 step than at 6, same bits
    static constexpr int FORCING_MIN_BLOCKS = 8;
    struct P {
        double g1, pinf1, g2, pinf2, ch2, cp2;
    };
    __device__ static P params(const double* prm, double ch) {
        const double cp = sqrt(ch * 0.18);
        return P{prm[0], prm[1], prm[2], prm[3], ch * ch, cp * cp};
    }
    // clamp_alpha and the stiffened-gas e(rho, p) / p(rho, e) of MHDEquationOfState (MHD/mhdequationofstate.cpp:7-21),
    // which are EulerEquationOfState's
    using R2 = EulerReducedF64;

    __device__ static double b2_of(double bx, double by, double bz) { return ((bx * bx) + (by * by)) + (bz * bz); }

    // computeConservedVariableVector (:113-153)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = R2::clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double u = W[1], v = W[2], w = W[3], r1 = W[4], r2 = W[5], p = W[6], bx = W[7], by = W[8], bz = W[9];
        const double rho = (a1 * r1) + (a2 * r2);
        U[0] = rho;
        U[1] = rho * a1;
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = rho * w;
        U[5] = a1 * r1;
        U[6] = a2 * r2;
        const double v2 = ((u * u) + (v * v)) + (w * w);
        const double b2 = b2_of(bx, by, bz);
        const double h1 = rho * ((0.5 * v2) + R2::e_of(rho, p, q.g1, q.pinf1));
        const double h2 = rho * ((0.5 * v2) + R2::e_of(rho, p, q.g2, q.pinf2));
        U[7] = (a1 * (h1 + (0.5 * b2))) + (a2 * (h2 + (0.5 * b2)));
        U[8] = bx;
        U[9] = by;
        U[10] = bz;
        U[11] = W[10];
    }
    // setConservedVariableVector (:58-89)
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
        const double bx = U[8], by = U[9], bz = U[10];
        const double E = (U[7] - (0.5 * b2_of(bx, by, bz))) / rho;
        const double e = E - (0.5 * (((u * u) + (v * v)) + (w * w)));
        W[0] = a1;
        W[1] = u;
        W[2] = v;
        W[3] = w;
        W[4] = U[5] / a1;
        W[5] = U[6] / a2;
        W[6] = (a1 * R2::p_of(rho, e, q.g1, q.pinf1)) + (a2 * R2::p_of(rho, e, q.g2, q.pinf2));
        W[7] = bx;
        W[8] = by;
        W[9] = bz;
        W[10] = U[11];
    }
    // compute{X,Y}FluxVector(vector, params, params) (:155-232, :239-316); v.B summed from 0.0 as
    // VectorAlgebra::computeDotProduct (Mathematics/vectoralgebra.cpp:38-49)
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
        const double r1 = U[5] / a1, r2 = U[6] / a2;
        const double bx = U[8], by = U[9], bz = U[10], psi = U[11];
        const double v2 = ((u * u) + (v * v)) + (w * w);
        const double b2 = b2_of(bx, by, bz);
        const double E = U[7];
        const double e = ((E - (0.5 * b2)) / rho) - (0.5 * v2);
        const double p = (a1 * R2::p_of(rho, e, q.g1, q.pinf1)) + (a2 * R2::p_of(rho, e, q.g2, q.pinf2));
        const double ch2 = (a1 * q.ch2) + (a2 * q.ch2);
        const double vb = ((0.0 + (u * bx)) + (v * by)) + (w * bz);
        const double un = AXIS == 0 ? u : v, bn = AXIS == 0 ? bx : by;
        F[0] = rho * un;
        F[1] = rho * (un * a1);
        if constexpr (AXIS == 0) {
            F[2] = (((rho * (u * u)) + p) + (0.5 * b2)) - (bx * bx);
            F[3] = (rho * (u * v)) - (bx * by);
        } else {
            F[2] = (rho * (v * u)) - (by * bx);
            F[3] = (((rho * (v * v)) + p) + (0.5 * b2)) - (by * by);
        }
        F[4] = (rho * (un * w)) - (bn * bz);
        F[5] = a1 * (r1 * un);
        F[6] = a2 * (r2 * un);
        F[7] = (((E + p) + (0.5 * b2)) * un) - (vb * bn);
        if constexpr (AXIS == 0) {
            F[8] = psi;
            F[9] = (by * u) - (bx * v);
        } else {
            F[8] = (bx * v) - (by * u);
            F[9] = psi;
        }
        F[10] = (bz * un) - (bn * w);
        F[11] = ch2 * bn;
    }
    // computeSourceTermVector (:323-347): GLM damping of psi
    __device__ static void source(const double* U, const P& q, double* S) {
#pragma unroll
        for (int i = 0; i < NU; i++) S[i] = 0.0;
        const double a1 = R2::clamp_alpha(U[1] / U[0]), a2 = 1.0 - a1;
        const double ch2 = (a1 * q.ch2) + (a2 * q.ch2), cp2 = (a1 * q.cp2) + (a2 * q.cp2);
        S[11] = (-(ch2 / cp2)) * U[11];
    }
    // MHDWaveSpeeds::compute{X,Y}FastMagnetoAcousticSpeed (MHD/mhdwavespeeds.cpp:7-17, :43-63) of material (g, pinf)
    // at density rho and normal field bn; the Alfven speed is computeNorm(B) / sqrt(rho), the norm summed from 0.0
    __device__ static double fast(double rho, double p, double bx, double by, double bz, double g, double pinf,
                                  double bn) {
        const double c = sqrt((g * (p + pinf)) / rho);
        const double a = sqrt(((0.0 + (bx * bx)) + (by * by)) + (bz * bz)) / sqrt(rho);
        const double c2 = c * c, a2 = a * a;
        return sqrt(0.5 * ((c2 + a2) + sqrt(((c2 + a2) * (c2 + a2)) - (4.0 * ((c2 * (bn * bn)) / rho)))));
    }
    // MHDSolvers::computeMaximumWaveSpeed{,2D} of the reduced model (Solvers/mhdsolvers.cpp:345-363, :416-440).  Both
    // materials' speeds take material 2's density, as computeMaterial{1,2}{X,Y}FastMagnetoAcousticSpeed (:393-401,
    // :433-441) do.
    __device__ static double wave(const double* W, const P& q, int dims) {
        const double r = W[5], p = W[6], bx = W[7], by = W[8], bz = W[9];
        const double f1x = fabs(fast(r, p, bx, by, bz, q.g1, q.pinf1, bx));
        const double f2x = fabs(fast(r, p, bx, by, bz, q.g2, q.pinf2, bx));
        if (dims == 1) return fabs(W[1]) + std_max(f1x, f2x);
        const double f1y = fabs(fast(r, p, bx, by, bz, q.g1, q.pinf1, by));
        const double f2y = fabs(fast(r, p, bx, by, bz, q.g2, q.pinf2, by));
        return std_max(fabs(W[1]), fabs(W[2])) + std_max(std_max(f1x, f1y), std_max(f2x, f2y));
    }
    // MHDReducedStateVector() (:3-16)
    __device__ static void default_state(double* W) {
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 0.999;
        W[4] = 1.0;
        W[5] = 1.0;
        W[6] = 1.0;
    }
    // the smaller material density (bad-state check) and the interface pressure
    __device__ static double density(const double* W) { return W[4] < W[5] ? W[4] : W[5]; }
    __device__ static double pressure(const double* W) { return W[6]; }
};

// ------------------------------------------------------------------------ MHD intermediate two-material
// MHDIntermediateStateVector (MHD/Multiphysics/mhdintermediatestatevector.cpp), every plane carried:
// W = (alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz, psi), U = (rho, rho alpha1, rho u, rho v, rho w, alpha1 rho1,
// alpha1 E1, alpha2 rho2, alpha2 E2, Bx, By, Bz, psi), E_k the material's total energy with the shared magnetic energy.
// Params and GLM coefficients as MHDReducedF64's.
struct MHDIntermediateF64 {
    static constexpr int NW = 12;
    static constexpr int NU = 13;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = true;
    static constexpr int FORCING_MIN_BLOCKS = 8;  // 4.8 % faster per 2048^2 step than at 6, same bits
    using P = MHDReducedF64::P;
    using R2 = EulerReducedF64;
    using MR = MHDReducedF64;
    __device__ static P params(const double* prm, double ch) { return MR::params(prm, ch); }

    // computeConservedVariableVector (:131-185)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = R2::clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double u = W[1], v = W[2], w = W[3], r1 = W[4], p1 = W[5], r2 = W[6], p2 = W[7];
        const double bx = W[8], by = W[9], bz = W[10];
        U[0] = (a1 * r1) + (a2 * r2);
        U[1] = U[0] * a1;
        U[2] = U[0] * u;
        U[3] = U[0] * v;
        U[4] = U[0] * w;
        U[5] = a1 * r1;
        U[7] = a2 * r2;
        const double b2 = MR::b2_of(bx, by, bz);
        const double v2 = ((u * u) + (v * v)) + (w * w);
        const double h1 = r1 * ((0.5 * v2) + R2::e_of(r1, p1, q.g1, q.pinf1));
        const double h2 = r2 * ((0.5 * v2) + R2::e_of(r2, p2, q.g2, q.pinf2));
        U[6] = a1 * (h1 + (0.5 * b2));
        U[8] = a2 * (h2 + (0.5 * b2));
        U[9] = bx;
        U[10] = by;
        U[11] = bz;
        U[12] = W[11];
    }
    // setConservedVariableVector (:49-106)
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
        const double r1 = U[5] / a1, r2 = U[7] / a2;
        const double bx = U[9], by = U[10], bz = U[11];
        const double b2 = MR::b2_of(bx, by, bz);
        const double v2 = ((u * u) + (v * v)) + (w * w);
        const double e1 = (((U[6] / a1) - (0.5 * b2)) / r1) - (0.5 * v2);
        const double e2 = (((U[8] / a2) - (0.5 * b2)) / r2) - (0.5 * v2);
        W[0] = a1;
        W[1] = u;
        W[2] = v;
        W[3] = w;
        W[4] = r1;
        W[5] = R2::p_of(r1, e1, q.g1, q.pinf1);
        W[6] = r2;
        W[7] = R2::p_of(r2, e2, q.g2, q.pinf2);
        W[8] = bx;
        W[9] = by;
        W[10] = bz;
        W[11] = U[12];
    }
    // compute{X,Y}FluxVector(vector, params, params) (:187-279, :286-378)
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
        const double r1 = U[5] / a1, r2 = U[7] / a2;
        const double bx = U[9], by = U[10], bz = U[11], psi = U[12];
        const double v2 = ((u * u) + (v * v)) + (w * w);
        const double b2 = MR::b2_of(bx, by, bz);
        const double E1 = U[6] / a1, E2 = U[8] / a2;
        const double p1 = R2::p_of(r1, ((E1 - (0.5 * b2)) / r1) - (0.5 * v2), q.g1, q.pinf1);
        const double p2 = R2::p_of(r2, ((E2 - (0.5 * b2)) / r2) - (0.5 * v2), q.g2, q.pinf2);
        const double ch2 = (a1 * q.ch2) + (a2 * q.ch2);
        const double vb = ((0.0 + (u * bx)) + (v * by)) + (w * bz);
        const double un = AXIS == 0 ? u : v, bn = AXIS == 0 ? bx : by;
        const double pm = (a1 * p1) + (a2 * p2);
        F[0] = rho * un;
        F[1] = rho * (un * a1);
        if constexpr (AXIS == 0) {
            F[2] = (((rho * (u * u)) + pm) + (0.5 * b2)) - (bx * bx);
            F[3] = (rho * (u * v)) - (bx * by);
        } else {
            F[2] = (rho * (v * u)) - (by * bx);
            F[3] = (((rho * (v * v)) + pm) + (0.5 * b2)) - (by * by);
        }
        F[4] = (rho * (un * w)) - (bn * bz);
        F[5] = a1 * (r1 * un);
        F[6] = (a1 * (((E1 + p1) + (0.5 * b2)) * un)) - (a1 * (vb * bn));
        F[7] = a2 * (r2 * un);
        F[8] = (a2 * (((E2 + p2) + (0.5 * b2)) * un)) - (a2 * (vb * bn));
        if constexpr (AXIS == 0) {
            F[9] = psi;
            F[10] = (by * u) - (bx * v);
        } else {
            F[9] = (bx * v) - (by * u);
            F[10] = psi;
        }
        F[11] = (bz * un) - (bn * w);
        F[12] = ch2 * bn;
    }
    // computeSourceTermVector (:385-403): GLM damping of psi, as the reduced model's
    __device__ static void source(const double* U, const P& q, double* S) {
#pragma unroll
        for (int i = 0; i < NU; i++) S[i] = 0.0;
        const double a1 = R2::clamp_alpha(U[1] / U[0]), a2 = 1.0 - a1;
        const double ch2 = (a1 * q.ch2) + (a2 * q.ch2), cp2 = (a1 * q.cp2) + (a2 * q.cp2);
        S[12] = (-(ch2 / cp2)) * U[12];
    }
    // MHDSolvers::computeMaximumWaveSpeed{,2D} of the intermediate model (Solvers/mhdsolvers.cpp:325-343, :389-414);
    // each material's fast speed at its own density and pressure (:453-511)
    __device__ static double wave(const double* W, const P& q, int dims) {
        const double bx = W[8], by = W[9], bz = W[10];
        const double f1x = fabs(MR::fast(W[4], W[5], bx, by, bz, q.g1, q.pinf1, bx));
        const double f2x = fabs(MR::fast(W[6], W[7], bx, by, bz, q.g2, q.pinf2, bx));
        if (dims == 1) return fabs(W[1]) + std_max(f1x, f2x);
        const double f1y = fabs(MR::fast(W[4], W[5], bx, by, bz, q.g1, q.pinf1, by));
        const double f2y = fabs(MR::fast(W[6], W[7], bx, by, bz, q.g2, q.pinf2, by));
        return std_max(fabs(W[1]), fabs(W[2])) + std_max(std_max(f1x, f1y), std_max(f2x, f2y));
    }
    // MHDIntermediateStateVector() (:3-22)
    __device__ static void default_state(double* W) {
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 0.999;
        W[4] = 1.0;
        W[5] = 1.0;
        W[6] = 1.0;
        W[7] = 1.0;
    }
    // bad-state check: the smaller material density and the volume-fraction mixture pressure.  The trace material's
    // own pressure (alpha clamped at 0.001) goes negative in the reference's runs of this model while the mixture stays
    // physical, so it is not checked on its own.
    __device__ static double density(const double* W) { return W[4] < W[6] ? W[4] : W[6]; }
    __device__ static double pressure(const double* W) {
        const double a1 = R2::clamp_alpha(W[0]);
        return (a1 * W[5]) + ((1.0 - a1) * W[7]);
    }
};

// ------------------------------------------------------------------------ MHD multiphysics two-material
// MHDMultiphysicsStateVector (MHD/Multiphysics/mhdmultiphysicsstatevector.cpp; 1D only in the reference): each
// material carries its own density, pressure, magnetic field and GLM scalar, the velocity is shared.
// W = (alpha1, u, v, w, rho1, p1, B1 (3), psi1, rho2, p2, B2 (3), psi2) (:135-163),
// U = (rho, rho alpha1, rho u (3), then per material k at 5 + 6 k: alpha rho, alpha E, alpha^(1/2) B (3), alpha psi)
// (:165-220).  Parameters {gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2}: the reference's solve for this model sets no
// c_h (Solvers/mhdsecondordersolver.cpp:362-385), so each material keeps its own.  pow(alpha, 1/2) and the interface
// field pow(alpha1 B1^2 + alpha2 B2^2, 1/2) are CUDA's pow, which may differ from glibc's in the last place.
struct MHDMultiphysicsF64 {
    static constexpr int NW = 16;
    static constexpr int NU = 17;
    static constexpr bool HAS_Y = false;
    static constexpr bool HAS_SOURCE = false;
    struct P {
        double g[2], pinfk[2], ch2[2];  // per material (no member named pinf: the state check's floor is 0)
    };
    using R2 = EulerReducedF64;
    using MR = MHDReducedF64;
    __device__ static P params(const double* prm, double /*ch*/) {
        return P{{prm[0], prm[2]}, {prm[1], prm[3]}, {prm[4] * prm[4], prm[5] * prm[5]}};
    }
    // computeConservedVariableVector (:165-220)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = R2::clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double u = W[1], v = W[2], w = W[3];
        const double rho = (a1 * W[4]) + (a2 * W[10]);
        U[0] = rho;
        U[1] = rho * a1;
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = rho * w;
        const double v2 = ((u * u) + (v * v)) + (w * w);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const double a = k == 0 ? a1 : a2;
            const double* wk = W + 4 + 6 * k;
            double* uk = U + 5 + 6 * k;
            uk[0] = a * wk[0];
            const double b2 = MR::b2_of(wk[2], wk[3], wk[4]);
            const double h = wk[0] * ((0.5 * v2) + R2::e_of(wk[0], wk[1], q.g[k], q.pinfk[k]));
            uk[1] = a * (h + (0.5 * b2));
#pragma unroll
            for (int i = 0; i < 3; i++) uk[2 + i] = pow(a, 1.0 / 2.0) * wk[2 + i];
            uk[5] = a * wk[5];
        }
    }
    // setConservedVariableVector (:84-133)
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
        const double v2 = ((u * u) + (v * v)) + (w * w);
        W[0] = a1;
        W[1] = u;
        W[2] = v;
        W[3] = w;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const double a = k == 0 ? a1 : a2;
            double* wk = W + 4 + 6 * k;
            const double* uk = U + 5 + 6 * k;
            wk[0] = uk[0] / a;
#pragma unroll
            for (int i = 0; i < 3; i++) wk[2 + i] = uk[2 + i] / pow(a, 1.0 / 2.0);
            const double b2 = MR::b2_of(wk[2], wk[3], wk[4]);
            const double E = ((uk[1] / a) - (0.5 * b2)) / wk[0];
            wk[1] = R2::p_of(wk[0], E - (0.5 * v2), q.g[k], q.pinfk[k]);
            wk[5] = uk[5] / a;
        }
    }
    // computeXFluxVector (:222-358); the model has no Y flux
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        static_assert(AXIS == 0, "the MHD multiphysics model is 1D");
        const double rho = U[0];
        const double a1 = R2::clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
        double B[2][3];
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int i = 0; i < 3; i++) B[k][i] = U[7 + 6 * k + i] / pow(k == 0 ? a1 : a2, 1.0 / 2.0);
        double ib2[3], ib[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            ib2[i] = (a1 * (B[0][i] * B[0][i])) + (a2 * (B[1][i] * B[1][i]));
            ib[i] = pow(ib2[i], 1.0 / 2.0);
        }
        const double v2 = ((u * u) + (v * v)) + (w * w);
        double pk[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const double a = k == 0 ? a1 : a2;
            const double* uk = U + 5 + 6 * k;
            double* fk = F + 5 + 6 * k;
            const double r = uk[0] / a;
            const double Et = uk[1] / a;
            const double b2 = MR::b2_of(B[k][0], B[k][1], B[k][2]);
            const double p = R2::p_of(r, ((Et - (0.5 * b2)) / r) - (0.5 * v2), q.g[k], q.pinfk[k]);
            pk[k] = p;
            const double bv = ((0.0 + (u * B[k][0])) + (v * B[k][1])) + (w * B[k][2]);
            const double s = pow(a, 1.0 / 2.0);
            fk[0] = a * (r * u);
            fk[1] = (a * (((Et + p) + (0.5 * b2)) * u)) - (a * (bv * B[k][0]));
            fk[2] = s * (uk[5] / a);
            fk[3] = s * ((B[k][1] * u) - (B[k][0] * v));
            fk[4] = s * ((B[k][2] * u) - (B[k][0] * w));
            fk[5] = a * (q.ch2[k] * B[k][0]);
        }
        F[0] = rho * u;
        F[1] = rho * (u * a1);
        F[2] = (((rho * (u * u)) + ((a1 * pk[0]) + (a2 * pk[1]))) + (0.5 * ((ib2[0] + ib2[1]) + ib2[2]))) - ib2[0];
        F[3] = (rho * (u * v)) - (ib[0] * ib[1]);
        F[4] = (rho * (u * w)) - (ib[0] * ib[2]);
    }
    __device__ static void source(const double*, const P&, double* S) {
#pragma unroll
        for (int i = 0; i < NU; i++) S[i] = 0.0;
    }
    // MHDSolvers::computeMaximumWaveSpeed of the multiphysics model (Solvers/mhdsolvers.cpp:305-323): each material's
    // fast magneto-acoustic speed at its own density, pressure and field
    __device__ static double wave(const double* W, const P& q, int) {
        const double f1 = fabs(MR::fast(W[4], W[5], W[6], W[7], W[8], q.g[0], q.pinfk[0], W[6]));
        const double f2 = fabs(MR::fast(W[10], W[11], W[12], W[13], W[14], q.g[1], q.pinfk[1], W[12]));
        return fabs(W[1]) + std_max(f1, f2);
    }
    // MHDMultiphysicsStateVector() (:3-27)
    __device__ static void default_state(double* W) {
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 0.999;
        W[4] = 1.0;
        W[5] = 1.0;
        W[10] = 1.0;
        W[11] = 1.0;
    }
    // bad-state check: finite values and positive material densities.  The trace material's pressure, and with it the
    // volume-fraction mixture, goes below zero in the reference's own runs of this model (its Dumbser multimaterial
    // layout at t = 0.05: mixture -2.9e-3), so no pressure is required positive.
    __device__ static double density(const double* W) { return W[4] < W[10] ? W[4] : W[10]; }
    __device__ static double pressure(const double* W) {
        const double a1 = R2::clamp_alpha(W[0]);
        return (a1 * W[5]) + ((1.0 - a1) * W[11]);
    }
    __device__ static bool positive_pressure(const P&) { return false; }
};

}  // namespace vg
