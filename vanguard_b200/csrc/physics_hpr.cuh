// Exact-FP64 device restatement of the HPR / GPR model: the StiffenedGas, ShockMieGruneisen and GodunovRomenski
// branches of HPRMieGruneisen and the elastic and plastic strain relaxation of HPRSourceTerms.
//
// Compiled with -fmad=false and IEEE division / square root; every expression keeps the reference's
// association order (matrix products summed from 0.0 in index order, Mathematics/matrixalgebra.cpp:62-81),
// so the sweeps and the CFL reproduce the reference bit for bit.  The relaxation source uses pow(det A, 5/3)
// (HPR/hprsourceterms.cpp:21-26), and the ShockMieGruneisen and GodunovRomenski branches pow of the density
// ratio; CUDA's pow and glibc's may differ in the last place, so runs with the source switched on or a solid
// equation of state agree with the reference to ~1e-15 relative rather than bitwise.
//
// computeGruneisenCoefficientDerivative (HPR/hprmiegruneisen.cpp:104-119) has no GodunovRomenski return, and
// compiled with -O2 a call to it does not return; the Grueneisen coefficient of that branch is the constant
// gamma (:23-26), so its derivative is 0 here.
//
// W = (rho, p, A00..A22, u, v, w, Jx, Jy, Jz)   (HPR/hprstatevector.cpp:50-73)
// U = (rho, rho E, A00..A22, rho u, rho v, rho w, rho Jx, rho Jy, rho Jz)   (HPR/hprstatevector.cpp:134-162)
// params = {gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, is_thermal,
//           eos (0 StiffenedGas, 1 ShockMieGruneisen, 2 GodunovRomenski), Gamma0, c0, s, alpha_eos, is_plastic,
//           sigma0, n}
#pragma once

#include "vg_common.cuh"

namespace vg {

// SOLID = false: the StiffenedGas gas with elastic strain relaxation only (the thermal-gas configurations);
// SOLID = true: every equation-of-state branch (params[12]) and the plastic relaxation (params[17]).  The gas
// instantiation compiles the StiffenedGas formulas alone, so it carries no branch or register cost for solids.
template <bool SOLID>
struct HPRModel {
    static constexpr int NW = 17;
    static constexpr int NU = 17;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = true;
    static constexpr int J_PLANE = 14;  // first heat-flux plane (kept by setConservedVariableVector when cold)
    struct P {
        double g, pinf, cv, rho0, T0, cs, alpha, tau1, tau2, Tref;
        int thermal;
        double ch2;
        int eos, plastic;
        double pref_mat, G0, c0, s, aeos, sigma0, npl;
    };
    __device__ static P params(const double* prm, double /*ch*/) {
        return P{prm[0], prm[1], prm[2], prm[3], prm[4], prm[5], prm[6], prm[7], prm[8], prm[9], prm[11] != 0.0, 0.0,
                 (int)prm[12], prm[17] != 0.0, prm[10], prm[13], prm[14], prm[15], prm[16], prm[18], prm[19]};
    }
    // gases need a positive pressure; the solid equations of state admit zero and tension
    __device__ static bool positive_pressure(const P& q) { return !SOLID || q.eos == 0; }

    // ---- 3x3 algebra in the reference's order
    struct M3 {
        double m[3][3];
    };
    __device__ static M3 load(const double* a9) {
        M3 r;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) r.m[i][j] = a9[3 * i + j];
        return r;
    }
    __device__ static M3 mul(const M3& a, const M3& b) {
        M3 r;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) r.m[i][j] = ((0.0 + (a.m[i][0] * b.m[0][j])) + (a.m[i][1] * b.m[1][j])) + (a.m[i][2] * b.m[2][j]);
        return r;
    }
    __device__ static M3 tmul(const M3& a, const M3& b) {  // a^T b
        M3 r;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) r.m[i][j] = ((0.0 + (a.m[0][i] * b.m[0][j])) + (a.m[1][i] * b.m[1][j])) + (a.m[2][i] * b.m[2][j]);
        return r;
    }
    // TensorAlgebra::computeDeviator (Mathematics/tensoralgebra.cpp:27-30)
    __device__ static M3 dev(const M3& g) {
        double c = (((0.0 + g.m[0][0]) + g.m[1][1]) + g.m[2][2]) / 3.0;
        M3 r;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) r.m[i][j] = g.m[i][j] + (-1.0 * (c * (i == j ? 1.0 : 0.0)));
        return r;
    }
    __device__ static double det(const M3& a) {  // Mathematics/matrixalgebra.cpp:131-135
        return ((a.m[0][0] * ((a.m[1][1] * a.m[2][2]) - (a.m[2][1] * a.m[1][2]))) -
                (a.m[0][1] * ((a.m[1][0] * a.m[2][2]) - (a.m[1][2] * a.m[2][0])))) +
               (a.m[0][2] * ((a.m[1][0] * a.m[2][1]) - (a.m[1][1] * a.m[2][0])));
    }

    // ---- HPRMieGruneisen (HPR/hprmiegruneisen.cpp), branch q.eos
    __device__ static double mg_G(double rho, const P& q) {  // computeGruneisenCoefficient (:7-28)
        if constexpr (!SOLID) return q.g - 1.0;
        if (q.eos == 1) return q.G0 * (q.rho0 / rho);
        if (q.eos == 2) return q.g;
        return q.g - 1.0;
    }
    __device__ static double gr_coef(double rho, const P& q) { return pow((rho / q.rho0), q.aeos); }
    __device__ static double mg_pref(double rho, const P& q) {  // computeReferencePressure (:30-66)
        if constexpr (!SOLID) return -q.pinf;
        if (q.eos == 1) {
            double c0sq = q.c0 * q.c0;
            if (rho > q.rho0)
                return c0sq * (((1.0 / q.rho0) - (1.0 / rho)) / pow(((1.0 / q.rho0) - (q.s * ((1.0 / q.rho0) - (1.0 / rho)))), 2.0));
            return c0sq * (rho - q.rho0);
        }
        if (q.eos == 2) {
            double c = gr_coef(rho, q);
            return (((q.c0 * q.c0) * (rho / q.aeos)) * (c - 1.0)) * c;
        }
        return -q.pinf;
    }
    __device__ static double mg_eref(double rho, const P& q) {  // computeReferenceInternalEnergy (:68-102)
        if constexpr (!SOLID) return q.pinf / rho;
        if (q.eos == 1) return rho > q.rho0 ? (0.5 * q.pref_mat) * ((1.0 / q.rho0) - (1.0 / rho)) : 0.0;
        if (q.eos == 2) {
            double c = gr_coef(rho, q);
            return ((q.c0 * q.c0) / (2.0 * (q.aeos * q.aeos))) * ((c - 1.0) * (c - 1.0));
        }
        return q.pinf / rho;
    }
    __device__ static double mg_dG(double rho, const P& q) {  // computeGruneisenCoefficientDerivative (:104-119)
        return (SOLID && q.eos == 1) ? (-q.G0) * (q.rho0 / (rho * rho)) : 0.0;
    }
    __device__ static double mg_dpref(double rho, const P& q) {  // computeReferencePressureDerivative (:121-155)
        if constexpr (!SOLID) return 0.0;
        if (q.eos == 1) {
            double c0sq = q.c0 * q.c0;
            if (rho > q.rho0)
                return (c0sq * (q.rho0 * q.rho0)) * (((q.s * (q.rho0 - rho)) - rho) / pow((q.s * (rho - q.rho0)) - rho, 3.0));
            return c0sq;
        }
        if (q.eos == 2) {
            double c = gr_coef(rho, q);
            return (((q.c0 * q.c0) / q.aeos) * c) * (((1.0 + q.aeos) * (c - 1.0)) + (q.aeos * c));
        }
        return 0.0;
    }
    __device__ static double mg_deref(double rho, const P& q) {  // computeReferenceInternalEnergyDerivative (:157-192)
        if constexpr (!SOLID) return -(q.pinf / (rho * rho));
        if (q.eos == 1) {
            if (rho > q.rho0) return (-(((rho - q.rho0) * q.rho0) * (q.c0 * q.c0))) / pow(((q.s * (rho - q.rho0)) - rho), 3.0);
            return 0.0;
        }
        if (q.eos == 2) {
            double c = gr_coef(rho, q);
            return (((q.c0 * q.c0) / (rho * q.aeos)) * (c - 1.0)) * c;
        }
        return -(q.pinf / (rho * rho));
    }
    // computeInternalEnergy / computePressure / computeTemperature (:194-221)
    __device__ static double mg_energy(double rho, double p, const P& q) {
        return mg_eref(rho, q) + ((p - mg_pref(rho, q)) / (rho * mg_G(rho, q)));
    }
    __device__ static double mg_pressure(double rho, double e, const P& q) {
        return (((e - mg_eref(rho, q)) * rho) * mg_G(rho, q)) + mg_pref(rho, q);
    }
    __device__ static double mg_temperature(double rho, double p, const P& q) {
        return q.Tref + ((p - mg_pref(rho, q)) / ((rho * mg_G(rho, q)) * q.cv));
    }
    // computeInternalEnergyDerivativeDensity / Pressure, computeTemperatureDerivativeDensity / Pressure (:223-262)
    __device__ static double mg_dedrho(double rho, double p, const P& q) {
        double G = mg_G(rho, q), dG = mg_dG(rho, q), pr = mg_pref(rho, q), dpr = mg_dpref(rho, q), der = mg_deref(rho, q);
        return der - ((((dpr * rho) * G) + ((G + (rho * dG)) * (p - pr))) / ((rho * G) * (rho * G)));
    }
    __device__ static double mg_dedp(double rho, const P& q) { return 1.0 / (rho * mg_G(rho, q)); }
    __device__ static double mg_dTdrho(double rho, double p, const P& q) {
        double G = mg_G(rho, q), dG = mg_dG(rho, q), pr = mg_pref(rho, q), dpr = mg_dpref(rho, q);
        return (-(((dpr * rho) * G) + ((G + (rho * dG)) * (p - pr)))) / (((rho * G) * (rho * G)) / q.cv);
    }
    __device__ static double mg_dTdp(double rho, const P& q) { return mg_dedp(rho, q) / q.cv; }

    // ---- HPREquationOfState (HPR/hprequationofstate.cpp:7-81)
    __device__ static double meso_distortion(const M3& A, const P& q) {
        M3 D = dev(tmul(A, A));
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++) sum += ((0.0 + (D.m[i][0] * D.m[i][0])) + (D.m[i][1] * D.m[i][1])) + (D.m[i][2] * D.m[i][2]);
        return (0.25 * (q.cs * q.cs)) * sum;
    }
    __device__ static double meso_thermal(double jx, double jy, double jz, const P& q) {
        return (0.5 * (q.alpha * q.alpha)) * (((jx * jx) + (jy * jy)) + (jz * jz));
    }
    __device__ static double macro(double u, double v, double w) { return 0.5 * (((u * u) + (v * v)) + (w * w)); }
    __device__ static double total_energy(double rho, double p, double u, double v, double w, const M3& A, double jx, double jy,
                                          double jz, const P& q) {
        double E = (mg_energy(rho, p, q) + meso_distortion(A, q)) + macro(u, v, w);
        if (q.thermal) E += meso_thermal(jx, jy, jz, q);
        return E;
    }
    __device__ static double pressure_of(double rho, double E, double u, double v, double w, const M3& A, double jx, double jy,
                                         double jz, const P& q) {
        double e = E - (macro(u, v, w) + meso_distortion(A, q));
        if (q.thermal) e -= meso_thermal(jx, jy, jz, q);
        return mg_pressure(rho, e, q);
    }
    // c_s^2 A dev(A^T A)   (HPR/hprderivatives.cpp:17-25)
    __device__ static M3 dEdA(const M3& A, const P& q) {
        M3 AD = mul(A, dev(tmul(A, A)));
        double cs2 = q.cs * q.cs;
        M3 r;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) r.m[i][j] = cs2 * AD.m[i][j];
        return r;
    }

    // HPRStateVector::computeConservedVariableVector (HPR/hprstatevector.cpp:134-162)
    __device__ static void cons(const double* W, const P& q, double* U) {
        M3 A = load(W + 2);
        double rho = W[0];
        U[0] = rho;
        U[1] = rho * total_energy(rho, W[1], W[11], W[12], W[13], A, W[14], W[15], W[16], q);
#pragma unroll
        for (int i = 0; i < 9; i++) U[2 + i] = W[2 + i];
        U[11] = rho * W[11];
        U[12] = rho * W[12];
        U[13] = rho * W[13];
        U[14] = q.thermal ? rho * W[14] : 0.0;
        U[15] = q.thermal ? rho * W[15] : 0.0;
        U[16] = q.thermal ? rho * W[16] : 0.0;
    }
    // HPRStateVector::setConservedVariableVector (HPR/hprstatevector.cpp:78-103); J kept when not thermal
    __device__ static void setcons(const double* U, const P& q, double* W) {
        double rho = U[0];
        W[0] = rho;
#pragma unroll
        for (int i = 0; i < 9; i++) W[2 + i] = U[2 + i];
        W[11] = U[11] / rho;
        W[12] = U[12] / rho;
        W[13] = U[13] / rho;
        if (q.thermal) {
            W[14] = U[14] / rho;
            W[15] = U[15] / rho;
            W[16] = U[16] / rho;
        }
        M3 A = load(W + 2);
        W[1] = pressure_of(rho, U[1] / rho, W[11], W[12], W[13], A, W[14], W[15], W[16], q);
    }
    // HPRStateVector::compute{X,Y}FluxVector (HPR/hprstatevector.cpp:164-298)
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        double rho = U[0];
        M3 A = load(U + 2);
        M3 d = dEdA(A, q);
        M3 Pm = tmul(A, d);
        double sig[3];
#pragma unroll
        for (int i = 0; i < 3; i++) sig[i] = (-rho) * Pm.m[AXIS][i];
        double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
        double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
        double E = U[1] / rho;
        double p = pressure_of(rho, E, u, v, w, A, jx, jy, jz, q);
        double un = AXIS == 0 ? u : v;
#pragma unroll
        for (int i = 0; i < 17; i++) F[i] = 0.0;
        F[0] = rho * un;
        F[1] = (rho * (un * E)) + (p * un);
        if (AXIS == 0) {
            F[11] = (rho * (u * u)) + p;
            F[12] = rho * (u * v);
            F[13] = rho * (u * w);
        } else {
            F[11] = rho * (v * u);
            F[12] = (rho * (v * v)) + p;
            F[13] = rho * (v * w);
        }
        F[1] -= ((0.0 + (sig[0] * u)) + (sig[1] * v)) + (sig[2] * w);
#pragma unroll
        for (int i = 0; i < 3; i++) F[11 + i] -= sig[i];
#pragma unroll
        for (int i = 0; i < 3; i++) F[2 + (i * 3) + AXIS] = ((0.0 + (A.m[i][0] * u)) + (A.m[i][1] * v)) + (A.m[i][2] * w);
        if (q.thermal) {
            double T = mg_temperature(rho, p, q);
            double a2 = q.alpha * q.alpha;
            F[1] += T * (a2 * (AXIS == 0 ? jx : jy));
            if (AXIS == 0) {
                F[14] = (rho * (u * jx)) + T;
                F[15] = rho * (u * jy);
                F[16] = rho * (u * jz);
            } else {
                F[14] = rho * (v * jx);
                F[15] = (rho * (v * jy)) + T;
                F[16] = rho * (v * jz);
            }
        }
    }
    // HPRSourceTerms::computeTheta1Reciprocal (HPR/hprsourceterms.cpp:7-27) given d = dE/dA; the plastic branch
    // scales it by (min(|sigma|, 1e8) / sigma0)^n, |sigma| = TensorAlgebra::computeSigmaNorm
    // (Mathematics/tensoralgebra.cpp:276-283) of sigma = -rho A^T dE/dA, with std::min's tie rule
    __device__ static double theta1(double rho, const M3& A, const M3& d, const P& q) {
        const double cs2 = q.cs * q.cs;
        const double th = 3.0 * (pow(det(A), (5.0 / 3.0)) / (cs2 * q.tau1));
        if (!SOLID || !q.plastic) return th;
        M3 Pm = tmul(A, d);
        double t[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) t[i][j] = (-rho) * Pm.m[i][j];
        double c1 = (((t[0][0] - t[1][1]) * (t[0][0] - t[1][1])) + ((t[1][1] - t[2][2]) * (t[1][1] - t[2][2]))) +
                    ((t[2][2] - t[0][0]) * (t[2][2] - t[0][0]));
        double c2 = ((t[0][1] * t[0][1]) + (t[1][2] * t[1][2])) + (t[2][0] * t[2][0]);
        double nrm = sqrt((0.5 * c1) + (3.0 * c2));
        const double cap = 1.0e8;  // pow(10.0, 8.0), exact
        nrm = cap < nrm ? cap : nrm;
        return th * pow(nrm / q.sigma0, q.npl);
    }
    // HPRStateVector::computeSourceTermVector (HPR/hprstatevector.cpp:312-366), HPRSourceTerms (HPR/hprsourceterms.cpp:7-39)
    __device__ static void source(const double* U, const P& q, double* S) {
        double rho = U[0];
        M3 A = load(U + 2);
        M3 d = dEdA(A, q);
        double th1 = theta1(rho, A, d, q);
#pragma unroll
        for (int i = 0; i < 17; i++) S[i] = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) S[2 + (i * 3) + j] = -d.m[i][j] * th1;
        if (q.thermal) {
            double E = U[1] / rho;
            double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
            double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
            double p = pressure_of(rho, E, u, v, w, A, jx, jy, jz, q);
            double T = mg_temperature(rho, p, q);
            double a2 = q.alpha * q.alpha;
            double th2 = 1.0 / ((a2 * q.tau2) * ((rho / q.rho0) * (q.T0 / T)));
            S[14] = ((-rho) * th2) * (a2 * jx);
            S[15] = ((-rho) * th2) * (a2 * jy);
            S[16] = ((-rho) * th2) * (a2 * jz);
        }
    }

    // HPRAcousticTensor::computeMaximumWaveSpeed (HPR/hpracoustictensor.cpp:7-97) with the 10-step power iteration of
    // MatrixAlgebra::computeLargestEigenvalue (Mathematics/matrixalgebra.cpp:182-199).  Only the entries
    // d sigma / d A [d][i][j][d] of HPREquationOfState::computeShearStressTensorDerivativeDistortionTensor
    // (HPR/hprequationofstate.cpp:83-113) enter; the i == d entries receive its += update twice.
    // diag: the first block reads dsigma/dA[d][i][i][d] for every column j, as the HPR multiphysics model's material-2
    // tensor does (HPR/Multiphysics/hprmultiphysicsacoustictensor.cpp:61)
    __device__ static double acoustic_speed(const double* W, int d, const P& q, bool diag = false) {
        double rho = W[0], p = W[1];
        M3 A = load(W + 2);
        M3 G = tmul(A, A), D = dev(G), AD = mul(A, D);
        double cs2 = q.cs * q.cs;
        double c1[4][5], c2[5][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 5; j++) c1[i][j] = 0.0;
#pragma unroll
        for (int i = 0; i < 5; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) c2[i][j] = 0.0;
        double ir = 1.0 / rho;
        c1[0][1] = ir;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j0 = 0; j0 < 3; j0++) {
                const int j = diag ? i : j0;
                double s1 = 0.0 + (G.m[d][i] * A.m[j][d]);
                double s2 = 0.0 + (G.m[d][d] * A.m[j][i]);
                double pp = 0.0 + (G.m[d][i] * A.m[j][d]);
                double t = (s1 + s2) + (-1.0 * ((2.0 / 3.0) * pp));
                t += AD.m[j][i];
                if (i == d) t += AD.m[j][d];
                c1[i][2 + j0] = -ir * ((-(rho * cs2)) * t);
            }
        M3 dd = dEdA(A, q);
        M3 Pm = tmul(A, dd);
#pragma unroll
        for (int i = 0; i < 3; i++) c1[i][0] = -ir * (-1.0 * Pm.m[d][i]);
        if (q.thermal) {
            c1[3][0] = mg_dTdrho(rho, p, q) / rho;
            c1[3][1] = mg_dTdp(rho, q) / rho;
        }
        double cad = sqrt(((p / (rho * rho)) - mg_dedrho(rho, p, q)) / mg_dedp(rho, q));
        c2[0][0] = rho;
        c2[1][d] = rho * (cad * cad);
#pragma unroll
        for (int i = 0; i < 3; i++) c2[1][i] += ((-rho) * Pm.m[d][i]) - (rho * (-1.0 * Pm.m[d][i]));
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) c2[2 + i][j] = A.m[i][j];
        if (q.thermal) {
            double T = mg_temperature(rho, p, q);
            double dTdp = mg_dTdp(rho, q);
            double ch = (sqrt((q.alpha * q.alpha) * (T / q.cv))) / rho;
            c2[1][3] = rho * ((ch * ch) / dTdp);
        }
        double om[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < 5; k++) s += c1[i][k] * c2[k][j];
                om[i][j] = s;
            }
        double x[4] = {1.0, 1.0, 1.0, 1.0}, y[4];
        for (int it = 0; it < 10; it++) {
#pragma unroll
            for (int i = 0; i < 4; i++) y[i] = (((0.0 + (om[i][0] * x[0])) + (om[i][1] * x[1])) + (om[i][2] * x[2])) + (om[i][3] * x[3]);
            double n2 = (((0.0 + (y[0] * y[0])) + (y[1] * y[1])) + (y[2] * y[2])) + (y[3] * y[3]);
            double inv = 1.0 / sqrt(n2);
#pragma unroll
            for (int i = 0; i < 4; i++) x[i] = inv * y[i];
        }
#pragma unroll
        for (int i = 0; i < 4; i++) y[i] = (((0.0 + (om[i][0] * x[0])) + (om[i][1] * x[1])) + (om[i][2] * x[2])) + (om[i][3] * x[3]);
        double n2 = (((0.0 + (y[0] * y[0])) + (y[1] * y[1])) + (y[2] * y[2])) + (y[3] * y[3]);
        return sqrt(sqrt(n2));
    }
    // HPRSolvers::computeMaximumWaveSpeed{,2D} per-cell terms (Solvers/hprsolvers.cpp:286-303, :362-385)
    __device__ static double wave(const double* W, const P& q, int dims) {
        if (dims == 1) return fabs(W[11]) + acoustic_speed(W, 0, q);
        return std_max(fabs(W[11]), fabs(W[12])) + std_max(acoustic_speed(W, 0, q), acoustic_speed(W, 1, q));
    }
    // HPRStateVector() (HPR/hprstatevector.cpp:3-16): rho 1, p 1/1.4, A = 1^(1/3) I = I
    __device__ static void default_state(double* W) {
#pragma unroll
        for (int i = 0; i < 17; i++) W[i] = 0.0;
        W[0] = 1.0;
        W[1] = 1.0 / 1.4;
        W[2] = 1.0;
        W[6] = 1.0;
        W[10] = 1.0;
    }
    __device__ static double density(const double* W) { return W[0]; }
    __device__ static double pressure(const double* W) { return W[1]; }
};

using HPRF64 = HPRModel<false>;
using HPRSolidF64 = HPRModel<true>;

// ---------------------------------------------------------------------------- HPR reduced two-material
// HPRReducedStateVector (HPR/Multiphysics/hprreducedstatevector.cpp), every plane carried: W = (alpha1, p, A (9,
// row-major), u, v, w, Jx, Jy, Jz, rho1, rho2), U = (rho, rho alpha1, rho E, A, rho u (3), rho J (3), alpha1 rho1,
// alpha2 rho2).  Each material's single-material formulas enter with that material's parameters: its pressure and
// total energy at the mixture density in the conversions and fluxes, at its own density in the source; its acoustic
// speed at its own density.  The materials take every HPRMieGruneisen branch and the plastic relaxation
// (HPRModel<true>), as the reference's scenarios of the two-material models run GodunovRomenski solids
// (HPR/Multiphysics/hprreducedtests.cpp); with a StiffenedGas material those branches compute the gas formulas.
// Parameters: the single-material 20-value block of each material, material k at params[20 k].  J is carried when
// either material is thermal (:104-109); otherwise the cell keeps its own.
struct HPRReducedF64 {
    static constexpr int NW = 19;
    static constexpr int NU = 20;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = true;
    static constexpr int J_PLANE = 14;
    using H = HPRModel<true>;
    using M3 = H::M3;
    struct P {
        H::P m1, m2;
        int thermal;   // either material thermal
        double pinf;   // the smaller stiffening pressure: the state check's pressure floor is -pinf
        double ch2;
    };
    __device__ static H::P material(const double* prm, int k) { return H::params(prm + 20 * k, 0.0); }
    __device__ static P params(const double* prm, double /*ch*/) {
        P q;
        q.m1 = material(prm, 0);
        q.m2 = material(prm, 1);
        q.thermal = q.m1.thermal || q.m2.thermal;
        q.pinf = q.m1.pinf < q.m2.pinf ? q.m1.pinf : q.m2.pinf;
        q.ch2 = 0.0;
        return q;
    }
    __device__ static double clamp_alpha(double a) { return a < 0.001 ? 0.001 : (a > 0.999 ? 0.999 : a); }

    // computeConservedVariableVector (:187-231)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double p = W[1], u = W[11], v = W[12], w = W[13], jx = W[14], jy = W[15], jz = W[16];
        const double r1 = W[17], r2 = W[18];
        const M3 A = H::load(W + 2);
        const double rho = (a1 * r1) + (a2 * r2);
        U[0] = rho;
        U[1] = rho * a1;
        const double E1 = H::total_energy(rho, p, u, v, w, A, jx, jy, jz, q.m1);
        const double E2 = H::total_energy(rho, p, u, v, w, A, jx, jy, jz, q.m2);
        U[2] = rho * ((a1 * E1) + (a2 * E2));
#pragma unroll
        for (int i = 0; i < 9; i++) U[3 + i] = W[2 + i];
        U[12] = rho * u;
        U[13] = rho * v;
        U[14] = rho * w;
        U[15] = q.thermal ? rho * jx : 0.0;
        U[16] = q.thermal ? rho * jy : 0.0;
        U[17] = q.thermal ? rho * jz : 0.0;
        U[18] = a1 * r1;
        U[19] = a2 * r2;
    }
    // setConservedVariableVector (:111-152); J kept when no material is thermal
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
#pragma unroll
        for (int i = 0; i < 9; i++) W[2 + i] = U[3 + i];
        W[11] = U[12] / rho;
        W[12] = U[13] / rho;
        W[13] = U[14] / rho;
        if (q.thermal) {
            W[14] = U[15] / rho;
            W[15] = U[16] / rho;
            W[16] = U[17] / rho;
        }
        W[17] = U[18] / a1;
        W[18] = U[19] / a2;
        const M3 A = H::load(W + 2);
        const double E = U[2] / rho;
        const double p1 = H::pressure_of(rho, E, W[11], W[12], W[13], A, W[14], W[15], W[16], q.m1);
        const double p2 = H::pressure_of(rho, E, W[11], W[12], W[13], A, W[14], W[15], W[16], q.m2);
        W[0] = a1;
        W[1] = (a1 * p1) + (a2 * p2);
    }
    // compute{X,Y}FluxVector (:233-330, :337-432), with the reference's X-flux mixture temperature alpha1 T1 + alpha1
    // T2 (:315; alpha1 T1 + alpha2 T2 in Y) and its Y-flux volume-fraction component (rho v) alpha1 (:414)
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const M3 A = H::load(U + 3);
        const double u = U[12] / rho, v = U[13] / rho, w = U[14] / rho;
        const double jx = U[15] / rho, jy = U[16] / rho, jz = U[17] / rho;
        const double r1 = U[18] / a1, r2 = U[19] / a2;
        const double E = U[2] / rho;
        const double p1 = H::pressure_of(rho, E, u, v, w, A, jx, jy, jz, q.m1);
        const double p2 = H::pressure_of(rho, E, u, v, w, A, jx, jy, jz, q.m2);
        const double p = (a1 * p1) + (a2 * p2);
        // HPREquationOfState::computeShearStressTensor (HPR/hprequationofstate.cpp:76-81) of each material at the
        // mixture density, mixed by volume fraction; only row AXIS enters
        const M3 P1 = H::tmul(A, H::dEdA(A, q.m1)), P2 = H::tmul(A, H::dEdA(A, q.m2));
        double sig[3];
#pragma unroll
        for (int i = 0; i < 3; i++) sig[i] = (a1 * ((-rho) * P1.m[AXIS][i])) + (a2 * ((-rho) * P2.m[AXIS][i]));
        const double un = AXIS == 0 ? u : v;
#pragma unroll
        for (int i = 0; i < NU; i++) F[i] = 0.0;
        F[0] = rho * un;
        F[1] = AXIS == 0 ? rho * (u * a1) : (rho * v) * a1;
        F[2] = (rho * (un * E)) + (p * un);
        if constexpr (AXIS == 0) {
            F[12] = (rho * (u * u)) + p;
            F[13] = rho * (u * v);
            F[14] = rho * (u * w);
        } else {
            F[12] = rho * (v * u);
            F[13] = (rho * (v * v)) + p;
            F[14] = rho * (v * w);
        }
        F[2] -= ((0.0 + (sig[0] * u)) + (sig[1] * v)) + (sig[2] * w);
#pragma unroll
        for (int i = 0; i < 3; i++) F[12 + i] -= sig[i];
#pragma unroll
        for (int i = 0; i < 3; i++) F[3 + (i * 3) + AXIS] = ((0.0 + (A.m[i][0] * u)) + (A.m[i][1] * v)) + (A.m[i][2] * w);
        if (q.thermal) {
            const double T1 = H::mg_temperature(r1, p, q.m1), T2 = H::mg_temperature(r2, p, q.m2);
            const double a21 = q.m1.alpha * q.m1.alpha, a22 = q.m2.alpha * q.m2.alpha;
            const double jn = AXIS == 0 ? jx : jy;
            F[2] += (a1 * (T1 * (a21 * jn))) + (a2 * (T2 * (a22 * jn)));
            const double T = AXIS == 0 ? (a1 * T1) + (a1 * T2) : (a1 * T1) + (a2 * T2);
            if constexpr (AXIS == 0) {
                F[15] = (rho * (u * jx)) + T;
                F[16] = rho * (u * jy);
                F[17] = rho * (u * jz);
            } else {
                F[15] = rho * (v * jx);
                F[16] = (rho * (v * jy)) + T;
                F[17] = rho * (v * jz);
            }
        }
        F[18] = a1 * (r1 * un);
        F[19] = a2 * (r2 * un);
    }
    // computeSourceTermVector (:439-520)
    __device__ static void source(const double* U, const P& q, double* S) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const M3 A = H::load(U + 3);
        const double r1 = U[18] / a1, r2 = U[19] / a2;
        const M3 d1 = H::dEdA(A, q.m1), d2 = H::dEdA(A, q.m2);
        const double th1 = (a1 * H::theta1(r1, A, d1, q.m1)) + (a2 * H::theta1(r2, A, d2, q.m2));
#pragma unroll
        for (int i = 0; i < NU; i++) S[i] = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) S[3 + (i * 3) + j] = -((a1 * d1.m[i][j]) + (a2 * d2.m[i][j])) * th1;
        if (q.thermal) {
            const double E = U[2] / rho;
            const double u = U[12] / rho, v = U[13] / rho, w = U[14] / rho;
            const double jx = U[15] / rho, jy = U[16] / rho, jz = U[17] / rho;
            const double p1 = H::pressure_of(r1, E, u, v, w, A, jx, jy, jz, q.m1);
            const double p2 = H::pressure_of(r2, E, u, v, w, A, jx, jy, jz, q.m2);
            const double p = (a1 * p1) + (a2 * p2);
            const double T = (a1 * H::mg_temperature(r1, p, q.m1)) + (a2 * H::mg_temperature(r2, p, q.m2));
            const double a21 = q.m1.alpha * q.m1.alpha, a22 = q.m2.alpha * q.m2.alpha;
            // HPRSourceTerms::computeTheta2Reciprocal (HPR/hprsourceterms.cpp:29-39) of each material
            const double t21 = 1.0 / ((a21 * q.m1.tau2) * ((r1 / q.m1.rho0) * (q.m1.T0 / T)));
            const double t22 = 1.0 / ((a22 * q.m2.tau2) * ((r2 / q.m2.rho0) * (q.m2.T0 / T)));
            const double th2 = (a1 * t21) + (a2 * t22);
            const double j3[3] = {jx, jy, jz};
#pragma unroll
            for (int i = 0; i < 3; i++) S[15 + i] = ((-rho) * th2) * ((a1 * (a21 * j3[i])) + (a2 * (a22 * j3[i])));
        }
    }
    // HPRReducedAcousticTensor::computeMaximumWaveSpeed (HPR/Multiphysics/hprreducedacoustictensor.cpp:169-183): each
    // material's single-material acoustic speed at its own density with the interface pressure and distortion
    __device__ static double speed(const double* W, int d, const H::P& qk, double rho_k) {
        double Wk[17];
        Wk[0] = rho_k;
#pragma unroll
        for (int i = 1; i < 17; i++) Wk[i] = W[i];
        return H::acoustic_speed(Wk, d, qk);
    }
    // HPRSolvers::computeMaximumWaveSpeed{,2D} of the reduced model (Solvers/hprsolvers.cpp:343-360, :412-436)
    __device__ static double wave(const double* W, const P& q, int dims) {
        const double sx = std_max(speed(W, 0, q.m1, W[17]), speed(W, 0, q.m2, W[18]));
        if (dims == 1) return fabs(W[11]) + sx;
        const double sy = std_max(speed(W, 1, q.m1, W[17]), speed(W, 1, q.m2, W[18]));
        return std_max(fabs(W[11]), fabs(W[12])) + std_max(sx, sy);
    }
    // HPRReducedStateVector() (:3-19)
    __device__ static void default_state(double* W) {
#pragma unroll
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 0.999;
        W[1] = 1.0 / 1.4;
        W[2] = 1.0;
        W[6] = 1.0;
        W[10] = 1.0;
        W[17] = 1.0;
        W[18] = 1.0;
    }
    // the smaller material density (bad-state check) and the interface pressure
    __device__ static double density(const double* W) { return W[17] < W[18] ? W[17] : W[18]; }
    __device__ static double pressure(const double* W) { return W[1]; }
    // The interface pressure of this model goes below zero within steps of runs the reference completes (a stiffened
    // material, the volume-fraction mixing of both materials' pressures at the mixture density), so the bad-state
    // check asks for finite values and positive densities only.
    __device__ static bool positive_pressure(const P&) { return false; }
};

// ---------------------------------------------------------------------------- HPR multiphysics two-material
// HPRMultiphysicsStateVector (HPR/Multiphysics/hprmultiphysicsstatevector.cpp; 1D only in the reference) for two
// StiffenedGas materials: each material carries its own density, pressure, distortion and heat flux, the velocity is
// shared.  W = (alpha1, u, v, w, rho1, p1, A1 (9), J1 (3), rho2, p2, A2 (9), J2 (3)) (:204-249),
// U = (rho, rho alpha1, rho u (3), then per material k at 5 + 14 k: alpha rho, alpha rho E, alpha^(1/3) A (9),
// alpha rho J (3)) (:251-317).  A material's J is carried when that material is thermal.  pow(alpha, 1/3) scales the
// distortion: CUDA's pow and glibc's may differ in the last place, so results agree with the reference to round-off
// rather than bitwise.  Parameters as for HPRReducedF64.
struct HPRMultiphysicsF64 {
    static constexpr int NW = 32;
    static constexpr int NU = 33;
    static constexpr bool HAS_Y = false;
    static constexpr bool HAS_SOURCE = false;
    using H = HPRReducedF64::H;
    using M3 = H::M3;
    using P = HPRReducedF64::P;
    __device__ static P params(const double* prm, double ch) { return HPRReducedF64::params(prm, ch); }
    __device__ static double clamp_alpha(double a) { return HPRReducedF64::clamp_alpha(a); }
    __device__ static const H::P& mat(const P& q, int k) { return k == 0 ? q.m1 : q.m2; }

    // computeConservedVariableVector (:251-317)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double u = W[1], v = W[2], w = W[3];
        const double rho = (a1 * W[4]) + (a2 * W[18]);
#pragma unroll
        for (int i = 0; i < NU; i++) U[i] = 0.0;
        U[0] = rho;
        U[1] = rho * a1;
        U[2] = rho * u;
        U[3] = rho * v;
        U[4] = rho * w;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const H::P& m = mat(q, k);
            const double a = k == 0 ? a1 : a2;
            const double* wk = W + 4 + 14 * k;  // rho, p, A (9), J (3)
            double* uk = U + 5 + 14 * k;        // a rho, a rho E, a^(1/3) A (9), a rho J (3)
            uk[0] = a * wk[0];
#pragma unroll
            for (int i = 0; i < 9; i++) uk[2 + i] = pow(a, (1.0 / 3.0)) * wk[2 + i];
            if (m.thermal)
#pragma unroll
                for (int i = 0; i < 3; i++) uk[11 + i] = a * (wk[0] * wk[11 + i]);
            const M3 A = H::load(wk + 2);
            uk[1] = a * (wk[0] * H::total_energy(wk[0], wk[1], u, v, w, A, wk[11], wk[12], wk[13], m));
        }
    }
    // setConservedVariableVector (:141-202); material k's J kept when it is not thermal
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        W[1] = U[2] / rho;
        W[2] = U[3] / rho;
        W[3] = U[4] / rho;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const H::P& m = mat(q, k);
            const double a = k == 0 ? a1 : a2;
            double* wk = W + 4 + 14 * k;
            const double* uk = U + 5 + 14 * k;
            wk[0] = uk[0] / a;
#pragma unroll
            for (int i = 0; i < 9; i++) wk[2 + i] = uk[2 + i] / pow(a, (1.0 / 3.0));
            if (m.thermal)
#pragma unroll
                for (int i = 0; i < 3; i++) wk[11 + i] = uk[11 + i] / (a * wk[0]);
            const double E = uk[1] / (a * wk[0]);
            const M3 A = H::load(wk + 2);
            wk[1] = H::pressure_of(wk[0], E, W[1], W[2], W[3], A, wk[11], wk[12], wk[13], m);
        }
        W[0] = a1;
    }
    // computeXFluxVector (:319-463); the model has no Y flux
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        static_assert(AXIS == 0, "the HPR multiphysics model is 1D");
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
#pragma unroll
        for (int i = 0; i < NU; i++) F[i] = 0.0;
        double pk[2], sig0[2][3];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const H::P& m = mat(q, k);
            const double a = k == 0 ? a1 : a2;
            const double* uk = U + 5 + 14 * k;
            const double r = uk[0] / a;
            M3 A;
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) A.m[i][j] = uk[2 + (i * 3) + j] / pow(a, (1.0 / 3.0));
            const double jx = uk[11] / (a * r), jy = uk[12] / (a * r), jz = uk[13] / (a * r);
            const double E = uk[1] / (a * r);
            const double p = H::pressure_of(r, E, u, v, w, A, jx, jy, jz, m);
            pk[k] = p;
            // HPREquationOfState::computeShearStressTensor (HPR/hprequationofstate.cpp:76-81), row 0
            const M3 Pm = H::tmul(A, H::dEdA(A, m));
#pragma unroll
            for (int i = 0; i < 3; i++) sig0[k][i] = (-r) * Pm.m[0][i];
            double* fk = F + 5 + 14 * k;
            fk[0] = a * (r * u);
            fk[1] = a * ((r * (u * E)) + (p * u));
            fk[1] -= a * (((0.0 + (sig0[k][0] * u)) + (sig0[k][1] * v)) + (sig0[k][2] * w));
#pragma unroll
            for (int i = 0; i < 3; i++)
                fk[2 + (i * 3)] = pow(a, (1.0 / 3.0)) * (((0.0 + (A.m[i][0] * u)) + (A.m[i][1] * v)) + (A.m[i][2] * w));
            if (m.thermal) {
                const double T = H::mg_temperature(r, p, m);
                fk[1] += a * (T * ((m.alpha * m.alpha) * jx));
                fk[11] = a * ((r * (u * jx)) + T);
                fk[12] = a * (r * (u * jy));
                fk[13] = a * (r * (u * jz));
            }
        }
        F[0] = rho * u;
        F[1] = rho * (u * a1);
        F[2] = (rho * (u * u)) + ((a1 * pk[0]) + (a2 * pk[1]));
        F[3] = rho * (u * v);
        F[4] = rho * (u * w);
#pragma unroll
        for (int i = 0; i < 3; i++) F[2 + i] -= (a1 * sig0[0][i]) + (a2 * sig0[1][i]);
    }
    __device__ static void source(const double*, const P&, double* S) {
#pragma unroll
        for (int i = 0; i < NU; i++) S[i] = 0.0;
    }
    // HPRMultiphysicsAcousticTensor::computeMaximumWaveSpeed (HPR/Multiphysics/hprmultiphysicsacoustictensor.cpp:
    // 177-184): each material's acoustic speed at its own state; material 2's with the diagonal quirk (:61)
    __device__ static double speed(const double* W, int d, const H::P& qk, int k) {
        double Wk[17];
        const double* wk = W + 4 + 14 * k;
        Wk[0] = wk[0];
        Wk[1] = wk[1];
#pragma unroll
        for (int i = 0; i < 9; i++) Wk[2 + i] = wk[2 + i];
        Wk[11] = W[1];
        Wk[12] = W[2];
        Wk[13] = W[3];
#pragma unroll
        for (int i = 0; i < 3; i++) Wk[14 + i] = wk[11 + i];
        return H::acoustic_speed(Wk, d, qk, k == 1);
    }
    // HPRSolvers::computeMaximumWaveSpeed of the multiphysics model (Solvers/hprsolvers.cpp:305-322)
    __device__ static double wave(const double* W, const P& q, int) {
        return fabs(W[1]) + std_max(speed(W, 0, q.m1, 0), speed(W, 0, q.m2, 1));
    }
    // HPRMultiphysicsStateVector() (:3-26)
    __device__ static void default_state(double* W) {
#pragma unroll
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 0.999;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            W[4 + 14 * k] = 1.0;
            W[5 + 14 * k] = 1.0 / 1.4;
            W[6 + 14 * k] = 1.0;
            W[10 + 14 * k] = 1.0;
            W[14 + 14 * k] = 1.0;
        }
    }
    // setConservedVariableVector leaves a cold material's J alone (:167-172, :191-196)
    __device__ static void keep_cold(const SweepArgs& a, long idx, const P& q, double* W) {
        if (!q.m1.thermal)
            for (int v = 15; v < 18; v++) W[v] = a.in[v * a.plane + idx];
        if (!q.m2.thermal)
            for (int v = 29; v < 32; v++) W[v] = a.in[v * a.plane + idx];
    }
    // the smaller material density (bad-state check); the mixture pressure, which as in the other HPR two-material
    // models is not required positive
    __device__ static double density(const double* W) { return W[4] < W[18] ? W[4] : W[18]; }
    __device__ static double pressure(const double* W) { return (clamp_alpha(W[0]) * W[5]) + ((1.0 - clamp_alpha(W[0])) * W[19]); }
    __device__ static bool positive_pressure(const P&) { return false; }
};

// ---------------------------------------------------------------------------- HPR intermediate two-material
// HPRIntermediateStateVector (HPR/Multiphysics/hprintermediatestatevector.cpp) for two StiffenedGas materials: a
// density, pressure and total energy per material, with a shared distortion, velocity and heat flux.
// W = (alpha1, A (9, row-major), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2) (:161-193),
// U = (rho, rho alpha1, A, rho u (3), rho J (3), alpha1 rho1, alpha1 rho1 E1, alpha2 rho2, alpha2 rho2 E2) (:195-247).
// Each material's EOS terms take that material's own density and pressure.  Parameters as for HPRReducedF64.
struct HPRIntermediateF64 {
    static constexpr int NW = 20;
    static constexpr int NU = 21;
    static constexpr bool HAS_Y = true;
    static constexpr bool HAS_SOURCE = true;
    static constexpr int J_PLANE = 13;  // first heat-flux plane (kept by setConservedVariableVector when cold)
    using H = HPRReducedF64::H;
    using M3 = H::M3;
    using P = HPRReducedF64::P;
    __device__ static P params(const double* prm, double ch) { return HPRReducedF64::params(prm, ch); }
    __device__ static double clamp_alpha(double a) { return HPRReducedF64::clamp_alpha(a); }

    // computeConservedVariableVector (:195-247)
    __device__ static void cons(const double* W, const P& q, double* U) {
        const double a1 = clamp_alpha(W[0]), a2 = 1.0 - a1;
        const double u = W[10], v = W[11], w = W[12], jx = W[13], jy = W[14], jz = W[15];
        const double r1 = W[16], p1 = W[17], r2 = W[18], p2 = W[19];
        const M3 A = H::load(W + 1);
        const double rho = (a1 * r1) + (a2 * r2);
        U[0] = rho;
        U[1] = rho * a1;
#pragma unroll
        for (int i = 0; i < 9; i++) U[2 + i] = W[1 + i];
        U[11] = rho * u;
        U[12] = rho * v;
        U[13] = rho * w;
        U[14] = q.thermal ? rho * jx : 0.0;
        U[15] = q.thermal ? rho * jy : 0.0;
        U[16] = q.thermal ? rho * jz : 0.0;
        U[17] = a1 * r1;
        U[18] = a1 * (r1 * H::total_energy(r1, p1, u, v, w, A, jx, jy, jz, q.m1));
        U[19] = a2 * r2;
        U[20] = a2 * (r2 * H::total_energy(r2, p2, u, v, w, A, jx, jy, jz, q.m2));
    }
    // setConservedVariableVector (:112-159); J kept when neither material is thermal
    __device__ static void setcons(const double* U, const P& q, double* W) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
#pragma unroll
        for (int i = 0; i < 9; i++) W[1 + i] = U[2 + i];
        W[10] = U[11] / rho;
        W[11] = U[12] / rho;
        W[12] = U[13] / rho;
        if (q.thermal) {
            W[13] = U[14] / rho;
            W[14] = U[15] / rho;
            W[15] = U[16] / rho;
        }
        W[16] = U[17] / a1;
        W[18] = U[19] / a2;
        const M3 A = H::load(W + 1);
        const double E1 = U[18] / (a1 * W[16]);
        W[17] = H::pressure_of(W[16], E1, W[10], W[11], W[12], A, W[13], W[14], W[15], q.m1);
        const double E2 = U[20] / (a2 * W[18]);
        W[19] = H::pressure_of(W[18], E2, W[10], W[11], W[12], A, W[13], W[14], W[15], q.m2);
        W[0] = a1;
    }
    // compute{X,Y}FluxVector (:249-367, :374-492): each material's energy flux with its own stress and heat flux; the
    // momentum takes the mixture pressure and the volume-fraction mean of both stresses
    template <int AXIS>
    __device__ static void flux(const double* U, const P& q, double* F) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const M3 A = H::load(U + 2);
        const double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
        const double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
        const double r1 = U[17] / a1, r2 = U[19] / a2;
        const double E1 = U[18] / (a1 * r1);
        const double p1 = H::pressure_of(r1, E1, u, v, w, A, jx, jy, jz, q.m1);
        const double E2 = U[20] / (a2 * r2);
        const double p2 = H::pressure_of(r2, E2, u, v, w, A, jx, jy, jz, q.m2);
        const double p = (a1 * p1) + (a2 * p2);
        // HPREquationOfState::computeShearStressTensor (HPR/hprequationofstate.cpp:76-81) of each material at its own
        // density; only row AXIS enters
        const M3 P1 = H::tmul(A, H::dEdA(A, q.m1)), P2 = H::tmul(A, H::dEdA(A, q.m2));
        double s1[3], s2[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            s1[i] = (-r1) * P1.m[AXIS][i];
            s2[i] = (-r2) * P2.m[AXIS][i];
        }
        const double un = AXIS == 0 ? u : v;
#pragma unroll
        for (int i = 0; i < NU; i++) F[i] = 0.0;
        F[0] = rho * un;
        F[1] = rho * (un * a1);
        F[18] = a1 * ((r1 * (un * E1)) + (p1 * un));
        F[20] = a2 * ((r2 * (un * E2)) + (p2 * un));
        if constexpr (AXIS == 0) {
            F[11] = (rho * (u * u)) + p;
            F[12] = rho * (u * v);
            F[13] = rho * (u * w);
        } else {
            F[11] = rho * (v * u);
            F[12] = (rho * (v * v)) + p;
            F[13] = rho * (v * w);
        }
        F[18] -= a1 * (((0.0 + (s1[0] * u)) + (s1[1] * v)) + (s1[2] * w));
        F[20] -= a2 * (((0.0 + (s2[0] * u)) + (s2[1] * v)) + (s2[2] * w));
#pragma unroll
        for (int i = 0; i < 3; i++) F[11 + i] -= (a1 * s1[i]) + (a2 * s2[i]);
#pragma unroll
        for (int i = 0; i < 3; i++) F[2 + (i * 3) + AXIS] = ((0.0 + (A.m[i][0] * u)) + (A.m[i][1] * v)) + (A.m[i][2] * w);
        if (q.thermal) {
            const double T1 = H::mg_temperature(r1, p1, q.m1), T2 = H::mg_temperature(r2, p2, q.m2);
            const double a21 = q.m1.alpha * q.m1.alpha, a22 = q.m2.alpha * q.m2.alpha;
            const double jn = AXIS == 0 ? jx : jy;
            const double T = (a1 * T1) + (a2 * T2);
            F[18] += a1 * (T1 * (a21 * jn));
            F[20] += a2 * (T2 * (a22 * jn));
            if constexpr (AXIS == 0) {
                F[14] = (rho * (u * jx)) + T;
                F[15] = rho * (u * jy);
                F[16] = rho * (u * jz);
            } else {
                F[14] = rho * (v * jx);
                F[15] = (rho * (v * jy)) + T;
                F[16] = rho * (v * jz);
            }
        }
        F[17] = a1 * (r1 * un);
        F[19] = a2 * (r2 * un);
    }
    // computeSourceTermVector (:499-592); the heat-flux rows are 0.0 - (rho theta2) dE/dJ, as the reference's -= on a
    // zeroed vector forms them
    __device__ static void source(const double* U, const P& q, double* S) {
        const double rho = U[0];
        const double a1 = clamp_alpha(U[1] / rho), a2 = 1.0 - a1;
        const M3 A = H::load(U + 2);
        const double r1 = U[17] / a1, r2 = U[19] / a2;
        const M3 d1 = H::dEdA(A, q.m1), d2 = H::dEdA(A, q.m2);
        const double th1 = (a1 * H::theta1(r1, A, d1, q.m1)) + (a2 * H::theta1(r2, A, d2, q.m2));
#pragma unroll
        for (int i = 0; i < NU; i++) S[i] = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) S[2 + (i * 3) + j] = -((a1 * d1.m[i][j]) + (a2 * d2.m[i][j])) * th1;
        if (q.thermal) {
            const double E1 = U[18] / (a1 * r1), E2 = U[20] / (a2 * r2);
            const double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
            const double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
            const double p1 = H::pressure_of(r1, E1, u, v, w, A, jx, jy, jz, q.m1);
            const double p2 = H::pressure_of(r2, E2, u, v, w, A, jx, jy, jz, q.m2);
            const double T1 = H::mg_temperature(r1, p1, q.m1), T2 = H::mg_temperature(r2, p2, q.m2);
            const double a21 = q.m1.alpha * q.m1.alpha, a22 = q.m2.alpha * q.m2.alpha;
            // HPRSourceTerms::computeTheta2Reciprocal (HPR/hprsourceterms.cpp:29-39) of each material
            const double t21 = 1.0 / ((a21 * q.m1.tau2) * ((r1 / q.m1.rho0) * (q.m1.T0 / T1)));
            const double t22 = 1.0 / ((a22 * q.m2.tau2) * ((r2 / q.m2.rho0) * (q.m2.T0 / T2)));
            const double th2 = (a1 * t21) + (a2 * t22);
            const double j3[3] = {jx, jy, jz};
#pragma unroll
            for (int i = 0; i < 3; i++) S[14 + i] = 0.0 - ((rho * th2) * ((a1 * (a21 * j3[i])) + (a2 * (a22 * j3[i]))));
        }
    }
    // HPRIntermediateAcousticTensor::computeMaximumWaveSpeed (HPR/Multiphysics/hprintermediateacoustictensor.cpp:
    // 177-184): each material's single-material acoustic speed at its own density and pressure
    __device__ static double speed(const double* W, int d, const H::P& qk, int k) {
        double Wk[17];
        Wk[0] = W[16 + 2 * k];
        Wk[1] = W[17 + 2 * k];
#pragma unroll
        for (int i = 0; i < 15; i++) Wk[2 + i] = W[1 + i];
        return H::acoustic_speed(Wk, d, qk);
    }
    // HPRSolvers::computeMaximumWaveSpeed{,2D} of the intermediate model (Solvers/hprsolvers.cpp:324-341, :387-410)
    __device__ static double wave(const double* W, const P& q, int dims) {
        const double sx = std_max(speed(W, 0, q.m1, 0), speed(W, 0, q.m2, 1));
        if (dims == 1) return fabs(W[10]) + sx;
        const double sy = std_max(speed(W, 1, q.m1, 0), speed(W, 1, q.m2, 1));
        return std_max(fabs(W[10]), fabs(W[11])) + std_max(sx, sy);
    }
    // HPRIntermediateStateVector() (:3-21)
    __device__ static void default_state(double* W) {
#pragma unroll
        for (int i = 0; i < NW; i++) W[i] = 0.0;
        W[0] = 0.999;
        W[1] = 1.0;
        W[5] = 1.0;
        W[9] = 1.0;
        W[16] = 1.0;
        W[17] = 1.0 / 1.4;
        W[18] = 1.0;
        W[19] = 1.0 / 1.4;
    }
    // the smaller material density (bad-state check); the mixture pressure
    __device__ static double density(const double* W) { return W[16] < W[18] ? W[16] : W[18]; }
    __device__ static double pressure(const double* W) { return (clamp_alpha(W[0]) * W[17]) + ((1.0 - clamp_alpha(W[0])) * W[19]); }
    // as for the reduced model: finite values and positive densities only
    __device__ static bool positive_pressure(const P&) { return false; }
};

}  // namespace vg
