/* CPU restatement of Vanguard's SLIC/FORCE path -- TEST INFRASTRUCTURE, never the product.
 *
 * Each function restates one reference function with the reference's floating-point operation
 * order (left-to-right sums, a - b written as a + (-1 * b) where the reference does so, which is
 * bit-identical to a - b).  Built with -ffp-contract=off so no FMA is formed, like the reference's
 * x86-64 build.  Pinned bit-for-bit against the compiled reference (oracle/_ref/libvgref.so) by
 * tests/test_oracle_pin.py and against tests/golden/ fixtures.
 *
 * Citations are path:line inside the Vanguard source tree.
 */
#include "slic_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXV 33

/* std::min / std::max semantics: min(a,b) = (b < a) ? b : a; max(a,b) = (a < b) ? b : a. */
static double smin(double a, double b) { return (b < a) ? b : a; }
static double smax(double a, double b) { return (a < b) ? b : a; }

/* ------------------------------------------------------------------------------ slope limiters */

/* SlopeLimiters::computeRCoefficient, Solvers/slopelimiters.cpp:7-10 */
static double r_coefficient(double r, double w) { return 2.0 / ((1.0 - w) + ((1.0 + w) * r)); }

/* Solvers/slopelimiters.cpp:12-74 (superbee :12-30, van Leer :32-42, minbee :44-58, dispatch :60-74) */
double vo_slope_limiter(double r, double w, int id) {
    if (id == 0) {
        if (r < 0.0) return 0.0;
        if (r < 0.5) return 2.0 * r;
        if (r < 1.0) return 1.0;
        return smin(smin(r, r_coefficient(r, w)), 2.0);
    } else if (id == 1) {
        if (r < 0.0) return 0.0;
        return smin((2.0 * r) / (1.0 + r), r_coefficient(r, w));
    } else {
        if (r < 0.0) return 0.0;
        if (r < 1.0) return r;
        return smin(1.0, r_coefficient(r, w));
    }
}

/* SlopeLimiters::computeSlopeVector(vector,vector,vector,...), Solvers/slopelimiters.cpp:217-246.
 * The 1e-5 floor is pow(10.0, -5.0) in the reference and replaces |x| < 1e-5 by +1e-5 (sign lost). */
static void slope_vector(int nv, const double* uL, const double* u, const double* uR, double w, int lim,
                         double* slope) {
    const double floor5 = pow(10.0, -5.0);
    const double cm = 0.5 * (1.0 + w), cp = 0.5 * (1.0 - w);
    for (int i = 0; i < nv; i++) {
        double dm = u[i] + (-1.0 * uL[i]);
        double dp = uR[i] + (-1.0 * u[i]);
        slope[i] = (cm * dm) + (cp * dp);
        double num = dm, den = dp;
        if (fabs(num) < floor5) num = floor5;
        if (fabs(den) < floor5) den = floor5;
        slope[i] *= vo_slope_limiter(num / den, w, lim);
    }
}

/* -------------------------------------------------------------------------------------- models */

typedef struct model model;
struct model {
    int nv;
    void (*cons)(const double* W, const double* prm, double* U);
    /* setConservedVariableVector: W is the state's previous primitives (read for HPR fields the
     * reference leaves untouched), overwritten with the new ones. */
    void (*setcons)(const double* U, const double* prm, double* W);
    void (*flux)(const double* U, int axis, const double* prm, double* F);
    double (*wave1d)(const double* W, const double* prm);
    double (*wave2d)(const double* W, const double* prm);
    void (*default_state)(const double* prm, double* W);
    /* computeSourceTermVector of the conserved vector (null: the model has no source) */
    void (*source)(const double* U, const double* prm, double* S);
};

/* ---- Euler: Euler/eulerstatevector.cpp, Euler/eulerequationofstate.cpp
 * prm = {gamma, p_inf, c_v, E0, T_ign, rate}.  W = rho,u,v,w,p,lambda. */

/* EulerEquationOfState::computeSpecificInternalEnergy, Euler/eulerequationofstate.cpp:7-13 */
static double euler_e(double rho, double p, const double* prm) {
    return (p + (prm[0] * prm[1])) / ((prm[0] - 1) * rho);
}
/* EulerEquationOfState::computePressure, Euler/eulerequationofstate.cpp:15-21 */
static double euler_p(double rho, double e, const double* prm) {
    return ((e * (prm[0] - 1)) * rho) - (prm[0] * prm[1]);
}
/* EulerStateVector::computeConservedVariableVector + computeTotalEnergy,
 * Euler/eulerstatevector.cpp:78-91, :192-198 */
static void euler_cons(const double* W, const double* prm, double* U) {
    double rho = W[0], u = W[1], v = W[2], w = W[3], p = W[4], lam = W[5];
    double v2 = ((u * u) + (v * v)) + (w * w);
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = rho * w;
    U[4] = rho * (((0.5 * v2) + euler_e(rho, p, prm)) + (prm[3] * (lam - 1.0)));
    U[5] = rho * lam;
}
/* EulerStateVector::setConservedVariableVector, Euler/eulerstatevector.cpp:47-61 */
static void euler_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho, lam = U[5] / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e = ((U[4] / rho) - (0.5 * v2)) - (prm[3] * (lam - 1.0));
    W[0] = rho; W[1] = u; W[2] = v; W[3] = w; W[4] = euler_p(rho, e, prm); W[5] = lam;
}
/* EulerStateVector::compute{X,Y}FluxVector(vector, params), Euler/eulerstatevector.cpp:93-120, :127-154 */
static void euler_flux(const double* U, int axis, const double* prm, double* F) {
    double rho = U[0];
    double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho, lam = U[5] / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double E = U[4] / rho;
    double e = (E - (0.5 * v2)) - (prm[3] * (lam - 1.0));
    double p = euler_p(rho, e, prm);
    if (axis == 0) {
        F[0] = rho * u;
        F[1] = (rho * (u * u)) + p;
        F[2] = rho * (u * v);
        F[3] = rho * (u * w);
        F[4] = (rho * (u * E)) + (u * p);
        F[5] = rho * (u * lam);
    } else {
        F[0] = rho * v;
        F[1] = rho * (v * u);
        F[2] = (rho * (v * v)) + p;
        F[3] = rho * (v * w);
        F[4] = (rho * (v * E)) + (v * p);
        F[5] = rho * (v * lam);
    }
}
/* EulerEquationOfState::computeSoundSpeed, Euler/eulerequationofstate.cpp:23-29 */
static double euler_c(const double* W, const double* prm) {
    return sqrt((prm[0] * (W[4] + prm[1])) / W[0]);
}
/* Solvers::computeMaximumWaveSpeed per-cell term, Solvers/solvers.cpp:259-276 */
static double euler_wave1d(const double* W, const double* prm) { return fabs(W[1]) + euler_c(W, prm); }
/* Solvers::computeMaximumWaveSpeed2D per-cell term, Solvers/solvers.cpp:318-339 */
static double euler_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[1]), fabs(W[2])) + euler_c(W, prm);
}
/* EulerStateVector(), Euler/eulerstatevector.cpp:3-12 */
static void euler_default(const double* prm, double* W) {
    (void)prm;
    W[0] = 1.0; W[1] = 0.0; W[2] = 0.0; W[3] = 0.0; W[4] = 1.0; W[5] = 1.0;
}

/* ---- ideal MHD with GLM: MHD/mhdstatevector.cpp, MHD/mhdequationofstate.cpp, MHD/mhdwavespeeds.cpp
 * prm = {gamma, p_inf, c_h}.  W = rho,u,v,w,p,Bx,By,Bz,psi. */

static double mhd_e(double rho, double p, const double* prm) {          /* mhdequationofstate.cpp:7-13 */
    return (p + (prm[0] * prm[1])) / ((prm[0] - 1) * rho);
}
static double mhd_p(double rho, double e, const double* prm) {          /* mhdequationofstate.cpp:15-21 */
    return ((e * (prm[0] - 1)) * rho) - (prm[0] * prm[1]);
}
/* MHDStateVector::computeConservedVariableVector + computeTotalEnergy, MHD/mhdstatevector.cpp:89-106, :236-245 */
static void mhd_cons(const double* W, const double* prm, double* U) {
    double rho = W[0], u = W[1], v = W[2], w = W[3], p = W[4], bx = W[5], by = W[6], bz = W[7];
    double v2 = ((u * u) + (v * v)) + (w * w);
    double hydro = rho * ((0.5 * v2) + mhd_e(rho, p, prm));
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    U[0] = rho; U[1] = rho * u; U[2] = rho * v; U[3] = rho * w;
    U[4] = hydro + (0.5 * b2);
    U[5] = bx; U[6] = by; U[7] = bz; U[8] = W[8];
}
/* MHDStateVector::setConservedVariableVector, MHD/mhdstatevector.cpp:49-68 */
static void mhd_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho;
    double bx = U[5], by = U[6], bz = U[7];
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double E = (U[4] - (0.5 * b2)) / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e = E - (0.5 * v2);
    W[0] = rho; W[1] = u; W[2] = v; W[3] = w; W[4] = mhd_p(rho, e, prm);
    W[5] = bx; W[6] = by; W[7] = bz; W[8] = U[8];
}
/* MHDStateVector::computeSourceTermVector (MHD/mhdstatevector.cpp:222-234): GLM damping of psi with
 * c_h = prm[2] and the parabolic damping of MHDMaterialParameters::configureParabolicDamping,
 * c_p = sqrt(c_h * 0.18) (MHD/mhdmaterialparameters.cpp:21-36). */
static void mhd_source(const double* U, const double* prm, double* S) {
    double ch2 = prm[2] * prm[2];
    double cp = sqrt(prm[2] * 0.18);
    double cp2 = cp * cp;
    for (int i = 0; i < 9; i++) S[i] = 0.0;
    S[8] = (-(ch2 / cp2)) * U[8];
}
/* MHDStateVector::compute{X,Y}FluxVector(vector, params), MHD/mhdstatevector.cpp:108-158, :165-215.
 * v.B is VectorAlgebra::computeDotProduct (Mathematics/vectoralgebra.cpp:38-49), summed from 0.0. */
static void mhd_flux(const double* U, int axis, const double* prm, double* F) {
    double rho = U[0];
    double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho;
    double bx = U[5], by = U[6], bz = U[7], psi = U[8];
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double E = U[4];
    double hydroE = (E - (0.5 * b2)) / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e = hydroE - (0.5 * v2);
    double p = mhd_p(rho, e, prm);
    double ch2 = prm[2] * prm[2];
    double vb = ((0.0 + (u * bx)) + (v * by)) + (w * bz);
    if (axis == 0) {
        F[0] = rho * u;
        F[1] = (((rho * (u * u)) + p) + (0.5 * b2)) - (bx * bx);
        F[2] = (rho * (u * v)) - (bx * by);
        F[3] = (rho * (u * w)) - (bx * bz);
        F[4] = (((E + p) + (0.5 * b2)) * u) - (vb * bx);
        F[5] = psi;
        F[6] = (by * u) - (bx * v);
        F[7] = (bz * u) - (bx * w);
        F[8] = ch2 * bx;
    } else {
        F[0] = rho * v;
        F[1] = (rho * (v * u)) - (by * bx);
        F[2] = (((rho * (v * v)) + p) + (0.5 * b2)) - (by * by);
        F[3] = (rho * (v * w)) - (by * bz);
        F[4] = (((E + p) + (0.5 * b2)) * v) - (vb * by);
        F[5] = (bx * v) - (by * u);
        F[6] = psi;
        F[7] = (bz * v) - (by * w);
        F[8] = ch2 * by;
    }
}
/* MHDWaveSpeeds::compute{X,Y}FastMagnetoAcousticSpeed, MHD/mhdwavespeeds.cpp:7-17, :43-63 */
static double mhd_fast(const double* W, const double* prm, double bn) {
    double rho = W[0], bx = W[5], by = W[6], bz = W[7];
    double c = sqrt((prm[0] * (W[4] + prm[1])) / rho);
    double a = sqrt(((0.0 + (bx * bx)) + (by * by)) + (bz * bz)) / sqrt(rho);
    double c2 = c * c, a2 = a * a;
    return sqrt(0.5 * ((c2 + a2) + sqrt(((c2 + a2) * (c2 + a2)) - (4.0 * ((c2 * (bn * bn)) / rho)))));
}
/* MHDSolvers::computeMaximumWaveSpeed{,2D} per-cell terms, Solvers/mhdsolvers.cpp:286-303, :365-388 */
static double mhd_wave1d(const double* W, const double* prm) {
    return fabs(W[1]) + fabs(mhd_fast(W, prm, W[5]));
}
static double mhd_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[1]), fabs(W[2])) + smax(fabs(mhd_fast(W, prm, W[5])), fabs(mhd_fast(W, prm, W[6])));
}
/* MHDStateVector(), MHD/mhdstatevector.cpp:3-16 */
static void mhd_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 9; i++) W[i] = 0.0;
    W[0] = 1.0; W[4] = 1.0;
}


/* ---- HPR / GPR.
 * prm = {gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, is_thermal,
 *        eos, Gamma0, c0, s, alpha_eos, is_plastic, sigma0, n}.
 * W = rho, p, A(9 row-major), u, v, w, Jx, Jy, Jz;  U = rho, rho E, A(9), rho v(3), rho J(3).
 * Matrix products sum from 0.0 in index order (MatrixAlgebra::multiplyMatrices,
 * Mathematics/matrixalgebra.cpp:62-81). */

typedef struct { double m[3][3]; } mat3;

/* MatrixAlgebra::multiplyMatrices of two 3x3 matrices */
static mat3 mm3(const mat3* a, const mat3* b) {
    mat3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0.0;
            for (int k = 0; k < 3; k++) s += a->m[i][k] * b->m[k][j];
            r.m[i][j] = s;
        }
    return r;
}
static mat3 tr3(const mat3* a) {
    mat3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[j][i] = a->m[i][j];
    return r;
}
static mat3 load_A(const double* a9) {
    mat3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = a9[3 * i + j];
    return r;
}
/* TensorAlgebra::computeDeviator (Mathematics/tensoralgebra.cpp:27-30): G + (-1 * ((tr/3) * I)) */
static mat3 deviator3(const mat3* g) {
    double tr = ((0.0 + g->m[0][0]) + g->m[1][1]) + g->m[2][2];
    double c = tr / 3.0;
    mat3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = g->m[i][j] + (-1.0 * (c * (i == j ? 1.0 : 0.0)));
    return r;
}
/* MatrixAlgebra::computeDeterminant (Mathematics/matrixalgebra.cpp:131-135) */
static double det3(const mat3* a) {
    const double(*m)[3] = a->m;
    return ((m[0][0] * ((m[1][1] * m[2][2]) - (m[2][1] * m[1][2]))) - (m[0][1] * ((m[1][0] * m[2][2]) - (m[1][2] * m[2][0])))) +
           (m[0][2] * ((m[1][0] * m[2][1]) - (m[1][1] * m[2][0])));
}
/* ---- HPRMieGruneisen (HPR/hprmiegruneisen.cpp) for the three equations of state, selected by prm[12]:
 * 0 StiffenedGas, 1 ShockMieGruneisen, 2 GodunovRomenski.  prm[13] Gamma0, prm[14] c0, prm[15] Hugoniot slope s,
 * prm[16] GodunovRomenski alpha, prm[10] the reference pressure of the shock branch's reference energy.
 * computeGruneisenCoefficientDerivative (:104-119) has no GodunovRomenski return; the Grueneisen coefficient
 * of that branch is the constant gamma (:23-26), so its derivative is taken as 0 here. */
static int hpr_eos(const double* prm) { return (int)prm[12]; }
/* computeGruneisenCoefficient (:7-28) */
static double mg_G(double rho, const double* prm) {
    switch (hpr_eos(prm)) {
        case 1: return prm[13] * (prm[3] / rho);
        case 2: return prm[0];
        default: return prm[0] - 1.0;
    }
}
/* the GodunovRomenski coefficient (rho / rho0)^alpha (:57-58, :94-95, :150-151, :187-188) */
static double gr_coef(double rho, const double* prm) { return pow((rho / prm[3]), prm[16]); }
/* computeReferencePressure (:30-66) */
static double mg_pref(double rho, const double* prm) {
    switch (hpr_eos(prm)) {
        case 1: {
            double c0sq = prm[14] * prm[14], rho0 = prm[3], s = prm[15];
            if (rho > rho0)
                return c0sq * (((1.0 / rho0) - (1.0 / rho)) / pow(((1.0 / rho0) - (s * ((1.0 / rho0) - (1.0 / rho)))), 2.0));
            return c0sq * (rho - rho0);
        }
        case 2: {
            double c = gr_coef(rho, prm);
            return (((prm[14] * prm[14]) * (rho / prm[16])) * (c - 1.0)) * c;
        }
        default: return -prm[1];
    }
}
/* computeReferenceInternalEnergy (:68-102) */
static double mg_eref(double rho, const double* prm) {
    switch (hpr_eos(prm)) {
        case 1:
            if (rho > prm[3]) return 0.5 * prm[10] * ((1.0 / prm[3]) - (1.0 / rho));
            return 0.0;
        case 2: {
            double c = gr_coef(rho, prm);
            return ((prm[14] * prm[14]) / (2.0 * (prm[16] * prm[16]))) * ((c - 1.0) * (c - 1.0));
        }
        default: return prm[1] / rho;
    }
}
/* computeGruneisenCoefficientDerivative (:104-119); 0 for GodunovRomenski, see above */
static double mg_dG(double rho, const double* prm) {
    if (hpr_eos(prm) == 1) return -prm[13] * (prm[3] / (rho * rho));
    return 0.0;
}
/* computeReferencePressureDerivative (:121-155) */
static double mg_dpref(double rho, const double* prm) {
    switch (hpr_eos(prm)) {
        case 1: {
            double c0sq = prm[14] * prm[14], rho0 = prm[3], s = prm[15];
            if (rho > rho0)
                return c0sq * (rho0 * rho0) * (((s * (rho0 - rho)) - rho) / pow((s * (rho - rho0)) - rho, 3.0));
            return c0sq;
        }
        case 2: {
            double c = gr_coef(rho, prm), a = prm[16];
            return ((prm[14] * prm[14]) / a) * c * (((1.0 + a) * (c - 1.0)) + (a * c));
        }
        default: return 0.0;
    }
}
/* computeReferenceInternalEnergyDerivative (:157-192) */
static double mg_deref(double rho, const double* prm) {
    switch (hpr_eos(prm)) {
        case 1: {
            double c0sq = prm[14] * prm[14], rho0 = prm[3], s = prm[15];
            if (rho > rho0) return -((rho - rho0) * rho0 * c0sq) / pow(((s * (rho - rho0)) - rho), 3.0);
            return 0.0;
        }
        case 2: {
            double c = gr_coef(rho, prm);
            return ((prm[14] * prm[14]) / (rho * prm[16])) * (c - 1.0) * c;
        }
        default: return -(prm[1] / (rho * rho));
    }
}
/* computeInternalEnergy / computePressure / computeTemperature (:194-221) */
static double mg_energy(double rho, double p, const double* prm) {
    return mg_eref(rho, prm) + ((p - mg_pref(rho, prm)) / (rho * mg_G(rho, prm)));
}
static double mg_pressure(double rho, double e, const double* prm) {
    return (((e - mg_eref(rho, prm)) * rho) * mg_G(rho, prm)) + mg_pref(rho, prm);
}
static double mg_temperature(double rho, double p, const double* prm) {
    return prm[9] + ((p - mg_pref(rho, prm)) / ((rho * mg_G(rho, prm)) * prm[2]));
}
/* computeInternalEnergyDerivativeDensity (:223-234) */
static double mg_dedrho(double rho, double p, const double* prm) {
    double G = mg_G(rho, prm), dG = mg_dG(rho, prm), pr = mg_pref(rho, prm), dpr = mg_dpref(rho, prm);
    double der = mg_deref(rho, prm);
    return der - ((((dpr * rho) * G) + ((G + (rho * dG)) * (p - pr))) / ((rho * G) * (rho * G)));
}
static double mg_dedp(double rho, const double* prm) { return 1.0 / (rho * mg_G(rho, prm)); } /* :236-241 */
static double mg_dTdrho(double rho, double p, const double* prm) {                            /* :243-255 */
    double G = mg_G(rho, prm), dG = mg_dG(rho, prm), pr = mg_pref(rho, prm), dpr = mg_dpref(rho, prm);
    return (-(((dpr * rho) * G) + ((G + (rho * dG)) * (p - pr)))) / (((rho * G) * (rho * G)) / prm[2]);
}
static double mg_dTdp(double rho, const double* prm) { return mg_dedp(rho, prm) / prm[2]; } /* :257-262 */

/* HPREquationOfState::computeMesoscaleDistortionEnergy (HPR/hprequationofstate.cpp:12-19) */
static double meso_distortion(const mat3* A, const double* prm) {
    mat3 At = tr3(A), G = mm3(&At, A), D = deviator3(&G);
    double sum = 0.0;
    for (int i = 0; i < 3; i++) {
        double row = 0.0;
        for (int j = 0; j < 3; j++) row += D.m[i][j] * D.m[i][j];
        sum += row;
    }
    return (0.25 * (prm[5] * prm[5])) * sum;
}
static double meso_thermal(double jx, double jy, double jz, const double* prm) {   /* :21-27 */
    return (0.5 * (prm[6] * prm[6])) * (((jx * jx) + (jy * jy)) + (jz * jz));
}
static double macro_energy(double u, double v, double w) { return 0.5 * (((u * u) + (v * v)) + (w * w)); } /* :29-34 */
static int hpr_thermal(const double* prm) { return prm[11] != 0.0; }
/* HPREquationOfState::computeTotalEnergy / computePressure (:36-62) */
static double hpr_total_energy(double rho, double p, double u, double v, double w, const mat3* A, double jx, double jy,
                               double jz, const double* prm) {
    double E = (mg_energy(rho, p, prm) + meso_distortion(A, prm)) + macro_energy(u, v, w);
    if (hpr_thermal(prm)) E += meso_thermal(jx, jy, jz, prm);
    return E;
}
static double hpr_pressure(double rho, double E, double u, double v, double w, const mat3* A, double jx, double jy, double jz,
                           const double* prm) {
    double e = E - (macro_energy(u, v, w) + meso_distortion(A, prm));
    if (hpr_thermal(prm)) e -= meso_thermal(jx, jy, jz, prm);
    return mg_pressure(rho, e, prm);
}
/* HPRDerivatives::computeTotalEnergyDerivativeDistortionTensor (HPR/hprderivatives.cpp:17-25): c_s^2 (A dev(A^T A)) */
static mat3 dE_dA(const mat3* A, const double* prm) {
    mat3 At = tr3(A), G = mm3(&At, A), D = deviator3(&G), AD = mm3(A, &D), r;
    double cs2 = prm[5] * prm[5];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = cs2 * AD.m[i][j];
    return r;
}
/* HPREquationOfState::computeShearStressTensor (:76-81): -rho A^T dE/dA */
static mat3 shear_stress(double rho, const mat3* A, const double* prm) {
    mat3 d = dE_dA(A, prm), At = tr3(A), P = mm3(&At, &d), r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = (-rho) * P.m[i][j];
    return r;
}

/* TensorAlgebra::computeSigmaNorm (Mathematics/tensoralgebra.cpp:276-283) */
static double sigma_norm(const mat3* s) {
    const double(*t)[3] = s->m;
    double c1 = (((t[0][0] - t[1][1]) * (t[0][0] - t[1][1])) + ((t[1][1] - t[2][2]) * (t[1][1] - t[2][2]))) +
                ((t[2][2] - t[0][0]) * (t[2][2] - t[0][0]));
    double c2 = ((t[0][1] * t[0][1]) + (t[1][2] * t[1][2])) + (t[2][0] * t[2][0]);
    return sqrt((0.5 * c1) + (3.0 * c2));
}
/* HPRSourceTerms::computeTheta1Reciprocal (HPR/hprsourceterms.cpp:7-27); prm[17] selects the plastic branch,
 * prm[18] its transition stress sigma0, prm[19] its power-law index; the stress norm is capped at 1e8 with
 * std::min's tie rule */
static double hpr_theta1(double rho, const mat3* A, const double* prm) {
    double cs2 = prm[5] * prm[5];
    if (prm[17] != 0.0) {
        mat3 sig = shear_stress(rho, A, prm);
        double nrm = sigma_norm(&sig), cap = pow(10.0, 8.0);
        nrm = cap < nrm ? cap : nrm;
        return 3.0 * (pow(det3(A), (5.0 / 3.0)) / (cs2 * prm[7])) * pow(nrm / prm[18], prm[19]);
    }
    return 3.0 * (pow(det3(A), (5.0 / 3.0)) / (cs2 * prm[7]));
}

/* HPRStateVector::computeConservedVariableVector (HPR/hprstatevector.cpp:134-162) */
static void hpr_cons(const double* W, const double* prm, double* U) {
    mat3 A = load_A(W + 2);
    double rho = W[0];
    for (int i = 0; i < 17; i++) U[i] = 0.0;
    U[0] = rho;
    U[1] = rho * hpr_total_energy(rho, W[1], W[11], W[12], W[13], &A, W[14], W[15], W[16], prm);
    for (int i = 0; i < 9; i++) U[2 + i] = W[2 + i];
    U[11] = rho * W[11];
    U[12] = rho * W[12];
    U[13] = rho * W[13];
    if (hpr_thermal(prm)) {
        U[14] = rho * W[14];
        U[15] = rho * W[15];
        U[16] = rho * W[16];
    }
}
/* HPRStateVector::setConservedVariableVector (HPR/hprstatevector.cpp:78-103); J kept when not thermal */
static void hpr_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    W[0] = rho;
    for (int i = 0; i < 9; i++) W[2 + i] = U[2 + i];
    W[11] = U[11] / rho;
    W[12] = U[12] / rho;
    W[13] = U[13] / rho;
    if (hpr_thermal(prm)) {
        W[14] = U[14] / rho;
        W[15] = U[15] / rho;
        W[16] = U[16] / rho;
    }
    mat3 A = load_A(W + 2);
    W[1] = hpr_pressure(rho, U[1] / rho, W[11], W[12], W[13], &A, W[14], W[15], W[16], prm);
}
/* HPRStateVector::compute{X,Y}FluxVector (HPR/hprstatevector.cpp:164-228, :235-298) */
static void hpr_flux(const double* U, int axis, const double* prm, double* F) {
    double rho = U[0];
    mat3 A = load_A(U + 2);
    mat3 sig = shear_stress(rho, &A, prm);
    double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
    double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
    double E = U[1] / rho;
    double p = hpr_pressure(rho, E, u, v, w, &A, jx, jy, jz, prm);
    double vel[3] = {u, v, w};
    double un = axis == 0 ? u : v;
    for (int i = 0; i < 17; i++) F[i] = 0.0;
    F[0] = rho * un;
    F[1] = (rho * (un * E)) + (p * un);
    if (axis == 0) {
        F[11] = (rho * (u * u)) + p;
        F[12] = rho * (u * v);
        F[13] = rho * (u * w);
    } else {
        F[11] = rho * (v * u);
        F[12] = (rho * (v * v)) + p;
        F[13] = rho * (v * w);
    }
    /* MatrixAlgebra::multiplyMatrixByVector (Mathematics/matrixalgebra.cpp:97-106): sums from 0.0 */
    double Av[3];
    for (int i = 0; i < 3; i++) Av[i] = ((0.0 + (A.m[i][0] * u)) + (A.m[i][1] * v)) + (A.m[i][2] * w);
    F[1] -= ((0.0 + (sig.m[axis][0] * vel[0])) + (sig.m[axis][1] * vel[1])) + (sig.m[axis][2] * vel[2]);
    for (int i = 0; i < 3; i++) F[11 + i] -= sig.m[axis][i];
    for (int i = 0; i < 3; i++) F[2 + (i * 3) + axis] = Av[i];
    if (hpr_thermal(prm)) {
        double T = mg_temperature(rho, p, prm);
        double a2 = prm[6] * prm[6];
        double q[3] = {T * (a2 * jx), T * (a2 * jy), T * (a2 * jz)};
        F[1] += q[axis];
        if (axis == 0) {
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
/* HPRStateVector::computeSourceTermVector (HPR/hprstatevector.cpp:312-366) with HPRSourceTerms
 * (HPR/hprsourceterms.cpp:7-39) */
static void hpr_source(const double* U, const double* prm, double* S) {
    double rho = U[0];
    mat3 A = load_A(U + 2);
    mat3 d = dE_dA(&A, prm);
    double th1 = hpr_theta1(rho, &A, prm);
    for (int i = 0; i < 17; i++) S[i] = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) S[2 + (i * 3) + j] = -d.m[i][j] * th1;
    if (hpr_thermal(prm)) {
        double E = U[1] / rho;
        double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
        double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
        double p = hpr_pressure(rho, E, u, v, w, &A, jx, jy, jz, prm);
        double T = mg_temperature(rho, p, prm);
        double a2 = prm[6] * prm[6];
        double dj[3] = {a2 * jx, a2 * jy, a2 * jz};
        double th2 = 1.0 / ((a2 * prm[8]) * ((rho / prm[3]) * (prm[4] / T)));
        for (int i = 0; i < 3; i++) S[14 + i] = ((-rho) * th2) * dj[i];
    }
}

/* ---- Stiff relaxation of the HPR source over a time h, cell by cell.  No counterpart in the reference, whose
 * only source integrator is the explicit RK4 forcing solver (stable for sub-steps up to ~2.8 tau).
 * Distortion: S_A = -c A dev(A^T A), c = 3 det(A)^(5/3) / tau1 (the non-plastic source above with dE/dA =
 * c_s^2 A dev(A^T A)).  det A is conserved (dev is traceless), so c is constant; G = A^T A keeps its eigenvectors
 * and its eigenvalues obey d(ln l_i)/dt = -2 c (l_i - mean(l)).  That system is integrated by implicit Euler
 * (L-stable; Newton on three unknowns), then A <- A V diag(sqrt(l_i' / l_i)) V^T.
 * Heat flux: d(rho J)/dt = -(rho0 T / (tau2 T0 rho)) rho J with rho, v, E and the relaxed A fixed.  Every equation
 * of state here has T = T_ref + (e - e_ref(rho)) / c_v, and e = e_J0 - alpha^2 |J|^2 / 2, so T = T_J0 - beta s with
 * s = |J|^2, beta = alpha^2 / (2 c_v): s obeys the Bernoulli equation ds/dt = -2 kappa (T_J0 - beta s) s
 * (kappa = rho0 / (tau2 T0 rho)), solved exactly over h: J scales by sqrt(E / ((1 - r) + r E)),
 * E = exp(-2 kappa T_J0 h), r = beta s0 / T_J0.  J is left alone where T <= 0.  rho, rho v and rho E do not change. */

/* cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix: g = V diag(l) V^T (published method) */
static void sym_eig3(const mat3* g, double l[3], double V[3][3]) {
    double a[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            a[i][j] = g->m[i][j];
            V[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 16; sweep++) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-32 * dia) break;
        for (int pq = 0; pq < 3; pq++) {
            int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            if (a[p][q] == 0.0) continue;
            double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
            double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
            double apq = a[p][q];
            a[p][p] -= t * apq;
            a[q][q] += t * apq;
            a[p][q] = a[q][p] = 0.0;
            for (int r = 0; r < 3; r++) {
                if (r != p && r != q) {
                    double arp = a[r][p], arq = a[r][q];
                    a[r][p] = a[p][r] = c * arp - s * arq;
                    a[r][q] = a[q][r] = s * arp + c * arq;
                }
                double vrp = V[r][p], vrq = V[r][q];
                V[r][p] = c * vrp - s * vrq;
                V[r][q] = s * vrp + c * vrq;
            }
        }
    }
    for (int i = 0; i < 3; i++) l[i] = a[i][i];
}

/* n implicit-Euler steps of d(mu_i)/dt = -2 c (exp(mu_i) - mean(exp(mu))) with k = 2 c h / n per step.  Newton
 * starts from the linear extrapolation of the last two step values and stops once a correction below 1e-8 has been
 * applied (quadratic convergence: the next correction would be below the double resolution of mu). */
static void relax_log_eigs(double mu[3], double k, int n) {
    double prev[3] = {mu[0], mu[1], mu[2]};
    for (int s = 0; s < n; s++) {
        double m0[3] = {mu[0], mu[1], mu[2]}, x[3];
        for (int i = 0; i < 3; i++) x[i] = m0[i] + (m0[i] - prev[i]);
        for (int i = 0; i < 3; i++) prev[i] = m0[i];
        for (int it = 0; it < 100; it++) {
            double e[3] = {exp(x[0]), exp(x[1]), exp(x[2])};
            double mean = (e[0] + e[1] + e[2]) / 3.0;
            /* J dx = -F with J = diag(1 + k e_i) - (k / 3) 1 e^T, by the Sherman-Morrison formula:
             * dx = y + k z (e . y) / sum(z), z_i = 1 / (1 + k e_i), y_i = -F_i z_i
             * (1 - (k / 3) e . z = sum(z) / 3 exactly, so the denominator takes no cancellation) */
            double z[3], y[3];
            for (int i = 0; i < 3; i++) {
                double F = (x[i] - m0[i]) + k * (e[i] - mean);
                z[i] = 1.0 / (1.0 + k * e[i]);
                y[i] = -F * z[i];
            }
            double g = k * (((e[0] * y[0]) + (e[1] * y[1]) + (e[2] * y[2])) / ((z[0] + z[1]) + z[2]));
            double dx[3], big = 0.0;
            for (int c = 0; c < 3; c++) {
                dx[c] = y[c] + z[c] * g;
                if (fabs(dx[c]) > big) big = fabs(dx[c]);
            }
            double damp = big > 0.5 ? 0.5 / big : 1.0;
            for (int i = 0; i < 3; i++) x[i] += damp * dx[i];
            if (big < 1e-8) break;
        }
        for (int i = 0; i < 3; i++) mu[i] = x[i];
    }
}

static int clampi(double v, int lo, int hi) {
    if (!(v > lo)) return lo;
    if (v > hi) return hi;
    return (int)ceil(v);
}

static void hpr_relax_cell(double* U, double h, const double* prm) {
    double rho = U[0];
    mat3 A = load_A(U + 2);
    double d = det3(&A);
    if (!(d > 0.0) || !(h > 0.0)) return;
    mat3 At = tr3(&A), G = mm3(&At, &A);
    double l[3], V[3][3], mu[3];
    sym_eig3(&G, l, V);
    if (!(l[0] > 0.0 && l[1] > 0.0 && l[2] > 0.0)) return;
    double c = 3.0 * (pow(d, 5.0 / 3.0) / prm[7]);
    double lmax = fmax(l[0], fmax(l[1], l[2]));
    int nA = clampi((2.0 * c * lmax * h) / 0.25, 1, 256);
    for (int i = 0; i < 3; i++) mu[i] = log(l[i]);
    relax_log_eigs(mu, 2.0 * c * (h / nA), nA);
    /* A' = A V diag(sqrt(l'/l)) V^T */
    double f[3], M[3][3];
    for (int i = 0; i < 3; i++) f[i] = exp(0.5 * (mu[i] - log(l[i])));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double sum = 0.0;
            for (int k = 0; k < 3; k++) sum += V[i][k] * f[k] * V[j][k];
            M[i][j] = sum;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double sum = 0.0;
            for (int k = 0; k < 3; k++) sum += A.m[i][k] * M[k][j];
            U[2 + 3 * i + j] = sum;
        }
    if (!hpr_thermal(prm)) return;
    mat3 An = load_A(U + 2);
    double E = U[1] / rho, u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
    double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
    double s0 = ((jx * jx) + (jy * jy)) + (jz * jz);
    double T = mg_temperature(rho, hpr_pressure(rho, E, u, v, w, &An, jx, jy, jz, prm), prm);
    if (!(s0 > 0.0) || !(T > 0.0)) return;
    double beta = (0.5 * (prm[6] * prm[6])) / prm[2];
    double TJ0 = T + (beta * s0); /* the temperature at J = 0 */
    double kappa = prm[3] / (prm[8] * prm[4] * rho);
    double Eh = exp(-2.0 * (kappa * (TJ0 * h)));
    double r = (beta * s0) / TJ0;
    double fac = sqrt(Eh / ((1.0 - r) + (r * Eh)));
    for (int i = 14; i < 17; i++) U[i] *= fac;
}

/* HPRAcousticTensor::computeMaximumWaveSpeed (HPR/hpracoustictensor.cpp:7-97) with the 10-step power
 * iteration of MatrixAlgebra::computeLargestEigenvalue (Mathematics/matrixalgebra.cpp:182-199).
 * Only the entries dsigma/dA[d][i][j][d] of HPREquationOfState::computeShearStressTensorDerivativeDistortionTensor
 * (HPR/hprequationofstate.cpp:83-113) enter; they are rebuilt here with the same sums and the same order of
 * the two += updates (the i == d entries receive the update twice, in the same loop iteration). */
static double hpr_acoustic_speed_q(const double* W, int d, const double* prm, int diag);
static double hpr_acoustic_speed(const double* W, int d, const double* prm) { return hpr_acoustic_speed_q(W, d, prm, 0); }
/* diag != 0: the second tensor block reads dsigma/dA[d][i][i][d] for every column j, as the HPR multiphysics model's
 * material-2 tensor does (HPR/Multiphysics/hprmultiphysicsacoustictensor.cpp:61) */
static double hpr_acoustic_speed_q(const double* W, int d, const double* prm, int diag) {
    double rho = W[0], p = W[1];
    mat3 A = load_A(W + 2);
    mat3 At = tr3(&A), G = mm3(&At, &A), D = deviator3(&G);
    mat3 AD = mm3(&A, &D), M = tr3(&AD);
    double cs2 = prm[5] * prm[5];
    double dsdA[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            /* P[a][b][c][e] = 0 + G[a][b] A[c][e]; T[a][b][c][e] = (P[e][b][c][a] + P[a][e][c][b]) + (-1 ((2/3) P[a][b][c][e]))
             * at a = d, b = i, c = j, e = d */
            double s1 = 0.0 + (G.m[d][i] * A.m[j][d]);
            double s2 = 0.0 + (G.m[d][d] * A.m[j][i]);
            double pp = 0.0 + (G.m[d][i] * A.m[j][d]);
            double t = (s1 + s2) + (-1.0 * ((2.0 / 3.0) * pp));
            t += M.m[i][j];
            if (i == d) t += M.m[d][j];
            dsdA[i][j] = (-(rho * cs2)) * t;
        }
    mat3 dEdA = dE_dA(&A, prm), Pd = mm3(&At, &dEdA), dsdrho, sig;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            dsdrho.m[i][j] = -1.0 * Pd.m[i][j];
            sig.m[i][j] = (-rho) * Pd.m[i][j];
        }
    double c1[4][5], c2[5][4];
    memset(c1, 0, sizeof(c1));
    memset(c2, 0, sizeof(c2));
    c1[0][1] = 1.0 / rho;
    for (int i = 0; i < 3; i++) c1[i][0] = -(1.0 / rho) * dsdrho.m[d][i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c1[i][2 + j] = -(1.0 / rho) * dsdA[i][diag ? i : j];
    if (hpr_thermal(prm)) {
        c1[3][0] = mg_dTdrho(rho, p, prm) / rho;
        c1[3][1] = mg_dTdp(rho, prm) / rho;
    }
    /* HPRWaveSpeeds::computeAdiabaticSoundSpeed (HPR/hprwavespeeds.cpp:7-13) */
    double cad = sqrt(((p / (rho * rho)) - mg_dedrho(rho, p, prm)) / mg_dedp(rho, prm));
    c2[0][0] = rho;
    c2[1][d] = rho * (cad * cad);
    for (int i = 0; i < 3; i++) c2[1][i] += sig.m[d][i] - (rho * dsdrho.m[d][i]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c2[2 + i][j] = A.m[i][j];
    if (hpr_thermal(prm)) {
        double T = mg_temperature(rho, p, prm);
        double dTdp = mg_dTdp(rho, prm);
        double ch = (sqrt((prm[6] * prm[6]) * (T / prm[2]))) / rho;  /* HPR/hprwavespeeds.cpp:15-21 */
        c2[1][3] = rho * ((ch * ch) / dTdp);
    }
    double om[4][4];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double s = 0.0;
            for (int k = 0; k < 5; k++) s += c1[i][k] * c2[k][j];
            om[i][j] = s;
        }
    double x[4] = {1.0, 1.0, 1.0, 1.0}, y[4];
    for (int it = 0; it < 10; it++) {
        for (int i = 0; i < 4; i++) {
            double s = 0.0;
            for (int k = 0; k < 4; k++) s += om[i][k] * x[k];
            y[i] = s;
        }
        double n2 = 0.0;
        for (int i = 0; i < 4; i++) n2 += y[i] * y[i];
        double inv = 1.0 / sqrt(n2);
        for (int i = 0; i < 4; i++) x[i] = inv * y[i];
    }
    for (int i = 0; i < 4; i++) {
        double s = 0.0;
        for (int k = 0; k < 4; k++) s += om[i][k] * x[k];
        y[i] = s;
    }
    double n2 = 0.0;
    for (int i = 0; i < 4; i++) n2 += y[i] * y[i];
    return sqrt(sqrt(n2));
}
/* HPRSolvers::computeMaximumWaveSpeed{,2D} per-cell terms (Solvers/hprsolvers.cpp:286-303, :362-385) */
static double hpr_wave1d(const double* W, const double* prm) { return fabs(W[11]) + hpr_acoustic_speed(W, 0, prm); }
static double hpr_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[11]), fabs(W[12])) + smax(hpr_acoustic_speed(W, 0, prm), hpr_acoustic_speed(W, 1, prm));
}
/* HPRStateVector() (HPR/hprstatevector.cpp:3-16): rho 1, p 1/1.4, A = 1^(1/3) I */
static void hpr_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 17; i++) W[i] = 0.0;
    double c = pow(1.0, (1.0 / 3.0));
    W[0] = 1.0;
    W[1] = 1.0 / 1.4;
    W[2] = c * 1.0;
    W[3] = c * 0.0;
    W[4] = c * 0.0;
    W[5] = c * 0.0;
    W[6] = c * 1.0;
    W[7] = c * 0.0;
    W[8] = c * 0.0;
    W[9] = c * 0.0;
    W[10] = c * 1.0;
}

/* ---- Euler reduced two-material model: Euler/Multiphysics/eulerreducedstatevector.cpp, prm = {gamma1, p_inf1,
 * gamma2, p_inf2}.  W = alpha1, u, v, w, rho1, rho2, p (the reference's primitive order) and an unused eighth plane;
 * U = rho, rho alpha1, rho u, rho v, rho w, alpha1 rho1, alpha2 rho2, rho E.  Every volume fraction the model derives
 * or uses is clamped to [0.001, 0.999] (:47-58, :99-108, :131-147). */
static double red_clamp(double a) {
    if (a < 0.001) return 0.001;
    if (a > 0.999) return 0.999;
    return a;
}
/* EulerReducedStateVector::computeConservedVariableVector (:96-129) */
static void red_cons(const double* W, const double* prm, double* U) {
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    double u = W[1], v = W[2], w = W[3], r1 = W[4], r2 = W[5], p = W[6];
    double rho = (a1 * r1) + (a2 * r2);
    U[0] = rho;
    U[1] = rho * a1;
    U[2] = rho * u;
    U[3] = rho * v;
    U[4] = rho * w;
    U[5] = a1 * r1;
    U[6] = a2 * r2;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e1 = euler_e(rho, p, prm) + (0.5 * v2), e2 = euler_e(rho, p, prm + 2) + (0.5 * v2);
    U[7] = rho * ((a1 * e1) + (a2 * e2));
}
/* EulerReducedStateVector::setConservedVariableVector (:43-73) */
static void red_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e = (U[7] / rho) - (0.5 * v2);
    W[0] = a1; W[1] = u; W[2] = v; W[3] = w;
    W[4] = U[5] / a1;
    W[5] = U[6] / a2;
    W[6] = (a1 * euler_p(rho, e, prm)) + (a2 * euler_p(rho, e, prm + 2));
    W[7] = 0.0;
}
/* EulerReducedStateVector::compute{X,Y}FluxVector(vector, params, params) (:131-180, :187-236) */
static void red_flux(const double* U, int axis, const double* prm, double* F) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double r1 = U[5] / a1, r2 = U[6] / a2;
    double E = U[7] / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e = E - (0.5 * v2);
    double p = (a1 * euler_p(rho, e, prm)) + (a2 * euler_p(rho, e, prm + 2));
    double un = axis == 0 ? u : v;
    F[0] = rho * un;
    F[1] = rho * (un * a1);
    F[2] = rho * (un * u);
    F[3] = rho * (un * v);
    F[4] = rho * (un * w);
    F[axis == 0 ? 2 : 3] += p;
    F[5] = a1 * (r1 * un);
    F[6] = a2 * (r2 * un);
    F[7] = (rho * (un * E)) + (un * p);
}
/* EulerEquationOfState::computeSoundSpeed (Euler/eulerequationofstate.cpp:23-29) of material k */
static double red_c(double rho_k, double p, const double* mk) { return sqrt((mk[0] * (p + mk[1])) / rho_k); }
/* Solvers::computeMaximumWaveSpeed{,2D} for the reduced model (Solvers/solvers.cpp:298-316, :365-387) */
static double red_wave1d(const double* W, const double* prm) {
    return fabs(W[1]) + smax(red_c(W[4], W[6], prm), red_c(W[5], W[6], prm + 2));
}
static double red_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[1]), fabs(W[2])) + smax(red_c(W[4], W[6], prm), red_c(W[5], W[6], prm + 2));
}
/* EulerReducedStateVector() (:3-14) */
static void red_default(const double* prm, double* W) {
    (void)prm;
    W[0] = 0.999; W[1] = 0.0; W[2] = 0.0; W[3] = 0.0; W[4] = 1.0; W[5] = 1.0; W[6] = 1.0; W[7] = 0.0;
}

/* ---- Euler multiphysics two-material model: Euler/Multiphysics/eulermultiphysicsstatevector.cpp, prm as the reduced
 * model's.  W = alpha1, u, v, w, rho1, p1, rho2, p2 (the reference's primitive order) and an unused ninth plane;
 * U = rho, rho alpha1, rho u, rho v, rho w, alpha1 rho1, alpha1 rho1 E1, alpha2 rho2, alpha2 rho2 E2. */
/* computeConservedVariableVector (:99-128) with computeMaterial{1,2}TotalEnergy (:255-260, :277-282) */
static void mph_cons(const double* W, const double* prm, double* U) {
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    double u = W[1], v = W[2], w = W[3], r1 = W[4], p1 = W[5], r2 = W[6], p2 = W[7];
    double rho = (a1 * r1) + (a2 * r2);
    double v2 = ((u * u) + (v * v)) + (w * w);
    U[0] = rho;
    U[1] = rho * a1;
    U[2] = rho * u;
    U[3] = rho * v;
    U[4] = rho * w;
    U[5] = a1 * r1;
    U[6] = a1 * (r1 * ((0.5 * v2) + euler_e(r1, p1, prm)));
    U[7] = a2 * r2;
    U[8] = a2 * (r2 * ((0.5 * v2) + euler_e(r2, p2, prm + 2)));
}
/* setConservedVariableVector (:46-79); its |v|^2 adds w + w where w * w is meant, as the reference does */
static void mph_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double r1 = U[5] / a1;
    double v2 = ((u * u) + (v * v)) + (w + w);
    double e1 = (U[6] / (r1 * a1)) - (0.5 * v2);
    double r2 = U[7] / a2;
    double e2 = (U[8] / (r2 * a2)) - (0.5 * v2);
    W[0] = a1; W[1] = u; W[2] = v; W[3] = w;
    W[4] = r1; W[5] = euler_p(r1, e1, prm);
    W[6] = r2; W[7] = euler_p(r2, e2, prm + 2);
    W[8] = 0.0;
}
/* compute{X,Y}FluxVector(vector, params, params) (:130-183, :190-243) */
static void mph_flux(const double* U, int axis, const double* prm, double* F) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double r1 = U[5] / a1;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double E1 = U[6] / (a1 * r1);
    double p1 = euler_p(r1, E1 - (0.5 * v2), prm);
    double r2 = U[7] / a2;
    double E2 = U[8] / (a2 * r2);
    double p2 = euler_p(r2, E2 - (0.5 * v2), prm + 2);
    double un = axis == 0 ? u : v;
    double pm = (a1 * p1) + (a2 * p2);
    F[0] = rho * un;
    F[1] = rho * (un * a1);
    F[2] = rho * (un * u);
    F[3] = rho * (un * v);
    F[4] = rho * (un * w);
    F[axis == 0 ? 2 : 3] += pm;
    F[5] = a1 * (r1 * un);
    F[6] = a1 * ((r1 * (un * E1)) + (un * p1));
    F[7] = a2 * (r2 * un);
    F[8] = a2 * ((r2 * (un * E2)) + (un * p2));
}
/* Solvers::computeMaximumWaveSpeed{,2D} (Solvers/solvers.cpp:278-296, :345-363) */
static double mph_wave1d(const double* W, const double* prm) {
    return fabs(W[1]) + smax(red_c(W[4], W[5], prm), red_c(W[6], W[7], prm + 2));
}
static double mph_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[1]), fabs(W[2])) + smax(red_c(W[4], W[5], prm), red_c(W[6], W[7], prm + 2));
}
/* EulerMultiphysicsStateVector() (:3-15) */
static void mph_default(const double* prm, double* W) {
    (void)prm;
    W[0] = 0.999; W[1] = 0.0; W[2] = 0.0; W[3] = 0.0; W[4] = 1.0; W[5] = 1.0; W[6] = 1.0; W[7] = 1.0; W[8] = 0.0;
}

/* ---- MHD reduced two-material model: MHD/Multiphysics/mhdreducedstatevector.cpp, prm = {gamma1, p_inf1, gamma2, p_inf2,
 * c_h}; c_h is both materials' hyperbolic wave speed (MHDMaterialParameters::setHyperbolicWaveSpeed, which solve{,2D}
 * sets to the padded grid's maximum wave speed every step).  W = alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi (the
 * reference's primitive order) and an unused twelfth plane; U = rho, rho alpha1, rho u, rho v, rho w, alpha1 rho1,
 * alpha2 rho2, E, Bx, By, Bz, psi.  Volume fractions are clamped to [0.001, 0.999] as in the Euler reduced model. */
/* the mixture c_h^2 (computeHyperbolicWaveSpeedSquared of both materials weighted by the volume fractions) */
static double mred_ch2(double a1, double a2, const double* prm) {
    double ch2 = prm[4] * prm[4];
    return (a1 * ch2) + (a2 * ch2);
}
/* computeConservedVariableVector (:113-153) */
static void mred_cons(const double* W, const double* prm, double* U) {
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    double u = W[1], v = W[2], w = W[3], r1 = W[4], r2 = W[5], p = W[6], bx = W[7], by = W[8], bz = W[9];
    double rho = (a1 * r1) + (a2 * r2);
    U[0] = rho;
    U[1] = rho * a1;
    U[2] = rho * u;
    U[3] = rho * v;
    U[4] = rho * w;
    U[5] = a1 * r1;
    U[6] = a2 * r2;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double h1 = rho * ((0.5 * v2) + mhd_e(rho, p, prm)), h2 = rho * ((0.5 * v2) + mhd_e(rho, p, prm + 2));
    U[7] = (a1 * (h1 + (0.5 * b2))) + (a2 * (h2 + (0.5 * b2)));
    U[8] = bx;
    U[9] = by;
    U[10] = bz;
    U[11] = W[10];
}
/* setConservedVariableVector (:58-89) */
static void mred_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double bx = U[8], by = U[9], bz = U[10];
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double E = (U[7] - (0.5 * b2)) / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e = E - (0.5 * v2);
    W[0] = a1; W[1] = u; W[2] = v; W[3] = w;
    W[4] = U[5] / a1;
    W[5] = U[6] / a2;
    W[6] = (a1 * mhd_p(rho, e, prm)) + (a2 * mhd_p(rho, e, prm + 2));
    W[7] = bx; W[8] = by; W[9] = bz; W[10] = U[11];
    W[11] = 0.0;
}
/* compute{X,Y}FluxVector(vector, params, params) (:155-232, :239-316); v.B summed from 0.0 as computeDotProduct */
static void mred_flux(const double* U, int axis, const double* prm, double* F) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double r1 = U[5] / a1, r2 = U[6] / a2;
    double bx = U[8], by = U[9], bz = U[10], psi = U[11];
    double v2 = ((u * u) + (v * v)) + (w * w);
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double E = U[7];
    double e = ((E - (0.5 * b2)) / rho) - (0.5 * v2);
    double p = (a1 * mhd_p(rho, e, prm)) + (a2 * mhd_p(rho, e, prm + 2));
    double ch2 = mred_ch2(a1, a2, prm);
    double vb = ((0.0 + (u * bx)) + (v * by)) + (w * bz);
    double un = axis == 0 ? u : v, bn = axis == 0 ? bx : by;
    F[0] = rho * un;
    F[1] = rho * (un * a1);
    F[2] = (rho * (un * u)) - (bn * bx);
    F[3] = (rho * (un * v)) - (bn * by);
    F[4] = (rho * (un * w)) - (bn * bz);
    if (axis == 0) F[2] = (((rho * (u * u)) + p) + (0.5 * b2)) - (bx * bx);
    else F[3] = (((rho * (v * v)) + p) + (0.5 * b2)) - (by * by);
    F[5] = a1 * (r1 * un);
    F[6] = a2 * (r2 * un);
    F[7] = (((E + p) + (0.5 * b2)) * un) - (vb * bn);
    if (axis == 0) {
        F[8] = psi;
        F[9] = (by * u) - (bx * v);
    } else {
        F[8] = (bx * v) - (by * u);
        F[9] = psi;
    }
    F[10] = (bz * un) - (bn * w);
    F[11] = ch2 * bn;
}
/* computeSourceTermVector (:323-347): GLM damping of psi with the mixtures of c_h^2 and of the parabolic damping
 * c_p^2, c_p = sqrt(c_h * 0.18) (MHDMaterialParameters::configureParabolicDamping, MHD/mhdmaterialparameters.cpp:31-34) */
static void mred_source(const double* U, const double* prm, double* S) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double cp = sqrt(prm[4] * 0.18);
    double cp2 = cp * cp;
    double ch2 = mred_ch2(a1, a2, prm);
    double cpm = (a1 * cp2) + (a2 * cp2);
    for (int i = 0; i < 12; i++) S[i] = 0.0;
    S[11] = (-(ch2 / cpm)) * U[11];
}
/* MHDWaveSpeeds::compute{X,Y}FastMagnetoAcousticSpeed (MHD/mhdwavespeeds.cpp:7-17, :43-63) of material k; the
 * reference's computeMaterial{1,2}{X,Y}FastMagnetoAcousticSpeed (:393-401, :433-441) both pass material 2's density */
static double mred_fast(const double* W, const double* mk, double bn) {
    double V[9] = {W[5], 0.0, 0.0, 0.0, W[6], W[7], W[8], W[9], 0.0};
    return mhd_fast(V, mk, bn);
}
/* MHDSolvers::computeMaximumWaveSpeed{,2D} of the reduced model (Solvers/mhdsolvers.cpp:345-363, :416-440) */
static double mred_wave1d(const double* W, const double* prm) {
    return fabs(W[1]) + smax(fabs(mred_fast(W, prm, W[7])), fabs(mred_fast(W, prm + 2, W[7])));
}
static double mred_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[1]), fabs(W[2])) +
           smax(smax(fabs(mred_fast(W, prm, W[7])), fabs(mred_fast(W, prm, W[8]))),
                smax(fabs(mred_fast(W, prm + 2, W[7])), fabs(mred_fast(W, prm + 2, W[8]))));
}
/* MHDReducedStateVector() (:3-16) */
static void mred_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 12; i++) W[i] = 0.0;
    W[0] = 0.999; W[4] = 1.0; W[5] = 1.0; W[6] = 1.0;
}

/* ---- MHD intermediate two-material model: MHD/Multiphysics/mhdintermediatestatevector.cpp, prm as the MHD reduced
 * model's.  W = alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz, psi (the reference's primitive order) and an unused
 * thirteenth plane; U = rho, rho alpha1, rho u, rho v, rho w, alpha1 rho1, alpha1 E1, alpha2 rho2, alpha2 E2, Bx, By,
 * Bz, psi, E_k the material's total energy with the shared magnetic energy. */
/* computeConservedVariableVector (:131-185) */
static void mint_cons(const double* W, const double* prm, double* U) {
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    double u = W[1], v = W[2], w = W[3], r1 = W[4], p1 = W[5], r2 = W[6], p2 = W[7], bx = W[8], by = W[9], bz = W[10];
    double rho = (a1 * r1) + (a2 * r2);
    U[0] = rho;
    U[1] = rho * a1;
    U[2] = rho * u;
    U[3] = rho * v;
    U[4] = rho * w;
    U[5] = a1 * r1;
    U[7] = a2 * r2;
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double v2 = ((u * u) + (v * v)) + (w * w);
    double h1 = r1 * ((0.5 * v2) + mhd_e(r1, p1, prm)), h2 = r2 * ((0.5 * v2) + mhd_e(r2, p2, prm + 2));
    U[6] = a1 * (h1 + (0.5 * b2));
    U[8] = a2 * (h2 + (0.5 * b2));
    U[9] = bx;
    U[10] = by;
    U[11] = bz;
    U[12] = W[11];
}
/* setConservedVariableVector (:49-106) */
static void mint_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double r1 = U[5] / a1, r2 = U[7] / a2;
    double bx = U[9], by = U[10], bz = U[11];
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double v2 = ((u * u) + (v * v)) + (w * w);
    double e1 = ((((U[6] / a1) - (0.5 * b2)) / r1)) - (0.5 * v2);
    double e2 = ((((U[8] / a2) - (0.5 * b2)) / r2)) - (0.5 * v2);
    W[0] = a1; W[1] = u; W[2] = v; W[3] = w;
    W[4] = r1; W[5] = mhd_p(r1, e1, prm);
    W[6] = r2; W[7] = mhd_p(r2, e2, prm + 2);
    W[8] = bx; W[9] = by; W[10] = bz; W[11] = U[12];
    W[12] = 0.0;
}
/* compute{X,Y}FluxVector(vector, params, params) (:187-279, :286-378) */
static void mint_flux(const double* U, int axis, const double* prm, double* F) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double r1 = U[5] / a1, r2 = U[7] / a2;
    double bx = U[9], by = U[10], bz = U[11], psi = U[12];
    double v2 = ((u * u) + (v * v)) + (w * w);
    double b2 = ((bx * bx) + (by * by)) + (bz * bz);
    double E1 = U[6] / a1, E2 = U[8] / a2;
    double p1 = mhd_p(r1, ((E1 - (0.5 * b2)) / r1) - (0.5 * v2), prm);
    double p2 = mhd_p(r2, ((E2 - (0.5 * b2)) / r2) - (0.5 * v2), prm + 2);
    double ch2 = mred_ch2(a1, a2, prm);
    double vb = ((0.0 + (u * bx)) + (v * by)) + (w * bz);
    double un = axis == 0 ? u : v, bn = axis == 0 ? bx : by;
    double pm = (a1 * p1) + (a2 * p2);
    F[0] = rho * un;
    F[1] = rho * (un * a1);
    F[2] = (rho * (un * u)) - (bn * bx);
    F[3] = (rho * (un * v)) - (bn * by);
    F[4] = (rho * (un * w)) - (bn * bz);
    if (axis == 0) F[2] = (((rho * (u * u)) + pm) + (0.5 * b2)) - (bx * bx);
    else F[3] = (((rho * (v * v)) + pm) + (0.5 * b2)) - (by * by);
    F[5] = a1 * (r1 * un);
    F[7] = a2 * (r2 * un);
    F[6] = (a1 * (((E1 + p1) + (0.5 * b2)) * un)) - (a1 * (vb * bn));
    F[8] = (a2 * (((E2 + p2) + (0.5 * b2)) * un)) - (a2 * (vb * bn));
    if (axis == 0) {
        F[9] = psi;
        F[10] = (by * u) - (bx * v);
    } else {
        F[9] = (bx * v) - (by * u);
        F[10] = psi;
    }
    F[11] = (bz * un) - (bn * w);
    F[12] = ch2 * bn;
}
/* computeSourceTermVector (:385-403): GLM damping of psi, as the reduced model's */
static void mint_source(const double* U, const double* prm, double* S) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double cp = sqrt(prm[4] * 0.18);
    double cp2 = cp * cp;
    double ch2 = mred_ch2(a1, a2, prm);
    double cpm = (a1 * cp2) + (a2 * cp2);
    for (int i = 0; i < 13; i++) S[i] = 0.0;
    S[12] = (-(ch2 / cpm)) * U[12];
}
/* compute{X,Y}FastMagnetoAcousticSpeed of material k at its own density and pressure (:453-511) */
static double mint_fast(const double* W, int k, const double* prm, double bn) {
    double V[9] = {W[4 + 2 * k], 0.0, 0.0, 0.0, W[5 + 2 * k], W[8], W[9], W[10], 0.0};
    return mhd_fast(V, prm + 2 * k, bn);
}
/* MHDSolvers::computeMaximumWaveSpeed{,2D} of the intermediate model (Solvers/mhdsolvers.cpp:325-343, :390-414) */
static double mint_wave1d(const double* W, const double* prm) {
    return fabs(W[1]) + smax(fabs(mint_fast(W, 0, prm, W[8])), fabs(mint_fast(W, 1, prm, W[8])));
}
static double mint_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[1]), fabs(W[2])) +
           smax(smax(fabs(mint_fast(W, 0, prm, W[8])), fabs(mint_fast(W, 0, prm, W[9]))),
                smax(fabs(mint_fast(W, 1, prm, W[8])), fabs(mint_fast(W, 1, prm, W[9]))));
}
/* MHDIntermediateStateVector() (:3-22) */
static void mint_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 13; i++) W[i] = 0.0;
    W[0] = 0.999; W[4] = 1.0; W[5] = 1.0; W[6] = 1.0; W[7] = 1.0;
}

/* ---- HPR reduced two-material model: HPR/Multiphysics/hprreducedstatevector.cpp.  prm holds the two materials'
 * HPRMaterialParameters as the single-material 20-value block each, material k at prm[20 k] ({gamma, p_inf, c_v, rho0,
 * T0, c_s, alpha, tau1, tau2, T_ref, p_ref, is_thermal, eos, Gamma0, c0, s, alpha_eos, is_plastic, sigma0, n}): any
 * equation of state of HPRMieGruneisen, elastic or plastic, as the reference's scenarios of these models use
 * (GodunovRomenski solids, HPR/Multiphysics/hprreducedtests.cpp).
 * W = alpha1, p, A (9, row-major), u, v, w, Jx, Jy, Jz, rho1, rho2 (the reference's primitive order, :154-185) and an
 * unused twentieth plane; U = rho, rho alpha1, rho E, A, rho u (3), rho J (3), alpha1 rho1, alpha2 rho2 (:187-231).
 * J is carried when either material is thermal (:104-109).  Every volume fraction is clamped to [0.001, 0.999]. */
static void hred_mat(const double* prm, int k, double* b) {
    for (int i = 0; i < 24; i++) b[i] = 0.0;
    for (int i = 0; i < 20; i++) b[i] = prm[20 * k + i];
}
static int hred_thermal(const double* prm) { return prm[11] != 0.0 || prm[31] != 0.0; }
/* computeConservedVariableVector (:187-231): the state's volume fraction is clamped first; the total energy is the
 * volume-fraction mean of each material's HPREquationOfState::computeTotalEnergy at the mixture density */
static void hred_cons(const double* W, const double* prm, double* U) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    double p = W[1], u = W[11], v = W[12], w = W[13], jx = W[14], jy = W[15], jz = W[16], r1 = W[17], r2 = W[18];
    mat3 A = load_A(W + 2);
    double rho = (a1 * r1) + (a2 * r2);
    for (int i = 0; i < 20; i++) U[i] = 0.0;
    U[0] = rho;
    U[1] = rho * a1;
    double E1 = hpr_total_energy(rho, p, u, v, w, &A, jx, jy, jz, b1);
    double E2 = hpr_total_energy(rho, p, u, v, w, &A, jx, jy, jz, b2);
    U[2] = rho * ((a1 * E1) + (a2 * E2));
    for (int i = 0; i < 9; i++) U[3 + i] = W[2 + i];
    U[12] = rho * u;
    U[13] = rho * v;
    U[14] = rho * w;
    if (hred_thermal(prm)) {
        U[15] = rho * jx;
        U[16] = rho * jy;
        U[17] = rho * jz;
    }
    U[18] = a1 * r1;
    U[19] = a2 * r2;
}
/* setConservedVariableVector (:111-152): each material's pressure from the mixture density and total energy */
static void hred_setcons(const double* U, const double* prm, double* W) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    for (int i = 0; i < 9; i++) W[2 + i] = U[3 + i];
    W[11] = U[12] / rho;
    W[12] = U[13] / rho;
    W[13] = U[14] / rho;
    if (hred_thermal(prm)) {
        W[14] = U[15] / rho;
        W[15] = U[16] / rho;
        W[16] = U[17] / rho;
    }
    W[17] = U[18] / a1;
    W[18] = U[19] / a2;
    mat3 A = load_A(W + 2);
    double E = U[2] / rho;
    double p1 = hpr_pressure(rho, E, W[11], W[12], W[13], &A, W[14], W[15], W[16], b1);
    double p2 = hpr_pressure(rho, E, W[11], W[12], W[13], &A, W[14], W[15], W[16], b2);
    W[0] = a1;
    W[1] = (a1 * p1) + (a2 * p2);
}
/* compute{X,Y}FluxVector (:233-330, :337-432).  Kept as the reference has them: the X flux's mixture temperature
 * alpha1 T1 + alpha1 T2 (:315; the Y flux's is alpha1 T1 + alpha2 T2), and the Y flux's volume-fraction component
 * (rho v) alpha1 against the X flux's rho (u alpha1) (:310, :414). */
static void hred_flux(const double* U, int axis, const double* prm, double* F) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    mat3 A = load_A(U + 3);
    double u = U[12] / rho, v = U[13] / rho, w = U[14] / rho;
    double jx = U[15] / rho, jy = U[16] / rho, jz = U[17] / rho;
    double r1 = U[18] / a1, r2 = U[19] / a2;
    double E = U[2] / rho;
    double p1 = hpr_pressure(rho, E, u, v, w, &A, jx, jy, jz, b1);
    double p2 = hpr_pressure(rho, E, u, v, w, &A, jx, jy, jz, b2);
    double p = (a1 * p1) + (a2 * p2);
    mat3 s1 = shear_stress(rho, &A, b1), s2 = shear_stress(rho, &A, b2), sig;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) sig.m[i][j] = (a1 * s1.m[i][j]) + (a2 * s2.m[i][j]);
    double vel[3] = {u, v, w};
    double un = axis == 0 ? u : v;
    for (int i = 0; i < 20; i++) F[i] = 0.0;
    F[0] = rho * un;
    F[1] = axis == 0 ? rho * (u * a1) : (rho * v) * a1;
    F[2] = (rho * (un * E)) + (p * un);
    if (axis == 0) {
        F[12] = (rho * (u * u)) + p;
        F[13] = rho * (u * v);
        F[14] = rho * (u * w);
    } else {
        F[12] = rho * (v * u);
        F[13] = (rho * (v * v)) + p;
        F[14] = rho * (v * w);
    }
    double Av[3];
    for (int i = 0; i < 3; i++) Av[i] = ((0.0 + (A.m[i][0] * u)) + (A.m[i][1] * v)) + (A.m[i][2] * w);
    F[2] -= ((0.0 + (sig.m[axis][0] * vel[0])) + (sig.m[axis][1] * vel[1])) + (sig.m[axis][2] * vel[2]);
    for (int i = 0; i < 3; i++) F[12 + i] -= sig.m[axis][i];
    for (int i = 0; i < 3; i++) F[3 + (i * 3) + axis] = Av[i];
    if (hred_thermal(prm)) {
        double T1 = mg_temperature(r1, p, b1), T2 = mg_temperature(r2, p, b2);
        double a21 = b1[6] * b1[6], a22 = b2[6] * b2[6];
        double j3[3] = {jx, jy, jz}, q[3];
        for (int i = 0; i < 3; i++) q[i] = (a1 * (T1 * (a21 * j3[i]))) + (a2 * (T2 * (a22 * j3[i])));
        double T = axis == 0 ? (a1 * T1) + (a1 * T2) : (a1 * T1) + (a2 * T2);
        F[2] += q[axis];
        if (axis == 0) {
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
/* computeSourceTermVector (:439-520): the mixture of both materials' distortion relaxation at each material's
 * density and, when either is thermal, of their heat-flux relaxation at the mixture temperature, with each material's
 * pressure from its own density */
static void hred_source(const double* U, const double* prm, double* S) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    mat3 A = load_A(U + 3);
    double r1 = U[18] / a1, r2 = U[19] / a2;
    mat3 d1 = dE_dA(&A, b1), d2 = dE_dA(&A, b2);
    double th1 = (a1 * hpr_theta1(r1, &A, b1)) + (a2 * hpr_theta1(r2, &A, b2));
    for (int i = 0; i < 20; i++) S[i] = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) S[3 + (i * 3) + j] = -((a1 * d1.m[i][j]) + (a2 * d2.m[i][j])) * th1;
    if (hred_thermal(prm)) {
        double E = U[2] / rho;
        double u = U[12] / rho, v = U[13] / rho, w = U[14] / rho;
        double jx = U[15] / rho, jy = U[16] / rho, jz = U[17] / rho;
        double p1 = hpr_pressure(r1, E, u, v, w, &A, jx, jy, jz, b1);
        double p2 = hpr_pressure(r2, E, u, v, w, &A, jx, jy, jz, b2);
        double p = (a1 * p1) + (a2 * p2);
        double T = (a1 * mg_temperature(r1, p, b1)) + (a2 * mg_temperature(r2, p, b2));
        double a21 = b1[6] * b1[6], a22 = b2[6] * b2[6];
        /* HPRSourceTerms::computeTheta2Reciprocal (HPR/hprsourceterms.cpp:29-39) of each material */
        double t21 = 1.0 / ((a21 * b1[8]) * ((r1 / b1[3]) * (b1[4] / T)));
        double t22 = 1.0 / ((a22 * b2[8]) * ((r2 / b2[3]) * (b2[4] / T)));
        double th2 = (a1 * t21) + (a2 * t22);
        double j3[3] = {jx, jy, jz};
        for (int i = 0; i < 3; i++) S[15 + i] = ((-rho) * th2) * ((a1 * (a21 * j3[i])) + (a2 * (a22 * j3[i])));
    }
}
/* HPRReducedAcousticTensor::computeMaximumWaveSpeed (HPR/Multiphysics/hprreducedacoustictensor.cpp:169-183): the
 * larger of the two materials' acoustic speeds, each the single-material tensor (HPR/hpracoustictensor.cpp) at that
 * material's density, the interface pressure and distortion, with that material's parameters */
static double hred_speed(const double* W, int d, const double* prm, int k) {
    double b[24], Wk[17];
    hred_mat(prm, k, b);
    Wk[0] = W[17 + k];
    for (int i = 1; i < 17; i++) Wk[i] = W[i];
    return hpr_acoustic_speed(Wk, d, b);
}
/* HPRSolvers::computeMaximumWaveSpeed{,2D} for the reduced model (Solvers/hprsolvers.cpp:343-360, :412-436) */
static double hred_wave1d(const double* W, const double* prm) {
    return fabs(W[11]) + smax(hred_speed(W, 0, prm, 0), hred_speed(W, 0, prm, 1));
}
static double hred_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[11]), fabs(W[12])) +
           smax(smax(hred_speed(W, 0, prm, 0), hred_speed(W, 0, prm, 1)), smax(hred_speed(W, 1, prm, 0), hred_speed(W, 1, prm, 1)));
}
/* HPRReducedStateVector::setPrimitiveVariableVector (:78-104) takes J only when either material is thermal; otherwise
 * the cells keep the default J = 0, which nothing reads.  HPRIntermediateStateVector's (hprintermediatestatevector.cpp:
 * 82-110) does the same with its J planes 13-15. */
static void hred_drop_cold_heat_flux(int id, double* planes, long n, const double* prm) {
    if (id == VO_HPR_REDUCED && !hred_thermal(prm))
        for (long i = 14 * n; i < 17 * n; i++) planes[i] = 0.0;
    if (id == VO_HPR_INTERMEDIATE && !hred_thermal(prm))
        for (long i = 13 * n; i < 16 * n; i++) planes[i] = 0.0;
}

/* ---- HPR intermediate two-material model: HPR/Multiphysics/hprintermediatestatevector.cpp.  Each material carries
 * its own density, pressure and total energy; the distortion, velocity and heat flux are shared.  prm as for the
 * reduced model (the 20-value block of each material).
 * W = alpha1, A (9, row-major), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2 (:161-193) and an unused twenty-first plane;
 * U = rho, rho alpha1, A, rho u (3), rho J (3), alpha1 rho1, alpha1 rho1 E1, alpha2 rho2, alpha2 rho2 E2 (:195-247).
 * Each material's EOS terms take that material's own density and pressure. */
/* computeConservedVariableVector (:195-247) */
static void hint_cons(const double* W, const double* prm, double* U) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    mat3 A = load_A(W + 1);
    double u = W[10], v = W[11], w = W[12], jx = W[13], jy = W[14], jz = W[15];
    double r1 = W[16], p1 = W[17], r2 = W[18], p2 = W[19];
    double rho = (a1 * r1) + (a2 * r2);
    for (int i = 0; i < 21; i++) U[i] = 0.0;
    U[0] = rho;
    U[1] = rho * a1;
    for (int i = 0; i < 9; i++) U[2 + i] = W[1 + i];
    U[11] = rho * u;
    U[12] = rho * v;
    U[13] = rho * w;
    if (hred_thermal(prm)) {
        U[14] = rho * jx;
        U[15] = rho * jy;
        U[16] = rho * jz;
    }
    U[17] = a1 * r1;
    U[19] = a2 * r2;
    double E1 = hpr_total_energy(r1, p1, u, v, w, &A, jx, jy, jz, b1);
    U[18] = a1 * (r1 * E1);
    double E2 = hpr_total_energy(r2, p2, u, v, w, &A, jx, jy, jz, b2);
    U[20] = a2 * (r2 * E2);
}
/* setConservedVariableVector (:112-159): each material's pressure from its own density and total energy; J kept when
 * neither material is thermal */
static void hint_setcons(const double* U, const double* prm, double* W) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    for (int i = 0; i < 9; i++) W[1 + i] = U[2 + i];
    W[10] = U[11] / rho;
    W[11] = U[12] / rho;
    W[12] = U[13] / rho;
    if (hred_thermal(prm)) {
        W[13] = U[14] / rho;
        W[14] = U[15] / rho;
        W[15] = U[16] / rho;
    }
    W[16] = U[17] / a1;
    W[18] = U[19] / a2;
    mat3 A = load_A(W + 1);
    double E1 = U[18] / (a1 * W[16]);
    W[17] = hpr_pressure(W[16], E1, W[10], W[11], W[12], &A, W[13], W[14], W[15], b1);
    double E2 = U[20] / (a2 * W[18]);
    W[19] = hpr_pressure(W[18], E2, W[10], W[11], W[12], &A, W[13], W[14], W[15], b2);
    W[0] = a1;
}
/* compute{X,Y}FluxVector (:249-367, :374-492): per-material energy fluxes with that material's own stress and heat
 * flux; the momentum takes the volume-fraction mean of the two stresses and the mixture pressure */
static void hint_flux(const double* U, int axis, const double* prm, double* F) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    mat3 A = load_A(U + 2);
    double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
    double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
    double r1 = U[17] / a1, r2 = U[19] / a2;
    double E1 = U[18] / (a1 * r1);
    double p1 = hpr_pressure(r1, E1, u, v, w, &A, jx, jy, jz, b1);
    double E2 = U[20] / (a2 * r2);
    double p2 = hpr_pressure(r2, E2, u, v, w, &A, jx, jy, jz, b2);
    double p = (a1 * p1) + (a2 * p2);
    mat3 s1 = shear_stress(r1, &A, b1), s2 = shear_stress(r2, &A, b2), sig;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) sig.m[i][j] = (a1 * s1.m[i][j]) + (a2 * s2.m[i][j]);
    double vel[3] = {u, v, w};
    double un = axis == 0 ? u : v;
    for (int i = 0; i < 21; i++) F[i] = 0.0;
    F[0] = rho * un;
    F[1] = rho * (un * a1);
    F[18] = a1 * ((r1 * (un * E1)) + (p1 * un));
    F[20] = a2 * ((r2 * (un * E2)) + (p2 * un));
    if (axis == 0) {
        F[11] = (rho * (u * u)) + p;
        F[12] = rho * (u * v);
        F[13] = rho * (u * w);
    } else {
        F[11] = rho * (v * u);
        F[12] = (rho * (v * v)) + p;
        F[13] = rho * (v * w);
    }
    double Av[3];
    for (int i = 0; i < 3; i++) Av[i] = ((0.0 + (A.m[i][0] * u)) + (A.m[i][1] * v)) + (A.m[i][2] * w);
    F[18] -= a1 * (((0.0 + (s1.m[axis][0] * vel[0])) + (s1.m[axis][1] * vel[1])) + (s1.m[axis][2] * vel[2]));
    F[20] -= a2 * (((0.0 + (s2.m[axis][0] * vel[0])) + (s2.m[axis][1] * vel[1])) + (s2.m[axis][2] * vel[2]));
    for (int i = 0; i < 3; i++) F[11 + i] -= sig.m[axis][i];
    for (int i = 0; i < 3; i++) F[2 + (i * 3) + axis] = Av[i];
    if (hred_thermal(prm)) {
        double T1 = mg_temperature(r1, p1, b1), T2 = mg_temperature(r2, p2, b2);
        double a21 = b1[6] * b1[6], a22 = b2[6] * b2[6];
        double j3[3] = {jx, jy, jz};
        double T = (a1 * T1) + (a2 * T2);
        F[18] += a1 * (T1 * (a21 * j3[axis]));
        F[20] += a2 * (T2 * (a22 * j3[axis]));
        if (axis == 0) {
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
/* computeSourceTermVector (:499-592): distortion relaxation with the volume-fraction means of both materials'
 * dE/dA and theta1 (each at its own density); heat-flux relaxation, when either material is thermal, with each
 * material's theta2 at its own temperature.  The heat-flux rows are 0.0 - (rho theta2) dE/dJ, as the reference's
 * -= on a zeroed vector forms them. */
static void hint_source(const double* U, const double* prm, double* S) {
    double b1[24], b2[24];
    hred_mat(prm, 0, b1);
    hred_mat(prm, 1, b2);
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    mat3 A = load_A(U + 2);
    double r1 = U[17] / a1, r2 = U[19] / a2;
    mat3 d1 = dE_dA(&A, b1), d2 = dE_dA(&A, b2);
    double th1 = (a1 * hpr_theta1(r1, &A, b1)) + (a2 * hpr_theta1(r2, &A, b2));
    for (int i = 0; i < 21; i++) S[i] = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) S[2 + (i * 3) + j] = (-((a1 * d1.m[i][j]) + (a2 * d2.m[i][j]))) * th1;
    if (hred_thermal(prm)) {
        double E1 = U[18] / (a1 * r1), E2 = U[20] / (a2 * r2);
        double u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
        double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
        double p1 = hpr_pressure(r1, E1, u, v, w, &A, jx, jy, jz, b1);
        double p2 = hpr_pressure(r2, E2, u, v, w, &A, jx, jy, jz, b2);
        double T1 = mg_temperature(r1, p1, b1), T2 = mg_temperature(r2, p2, b2);
        double a21 = b1[6] * b1[6], a22 = b2[6] * b2[6];
        double j3[3] = {jx, jy, jz};
        /* HPRSourceTerms::computeTheta2Reciprocal (HPR/hprsourceterms.cpp:29-39) of each material */
        double t21 = 1.0 / ((a21 * b1[8]) * ((r1 / b1[3]) * (b1[4] / T1)));
        double t22 = 1.0 / ((a22 * b2[8]) * ((r2 / b2[3]) * (b2[4] / T2)));
        double th2 = (a1 * t21) + (a2 * t22);
        for (int i = 0; i < 3; i++) S[14 + i] = 0.0 - ((rho * th2) * ((a1 * (a21 * j3[i])) + (a2 * (a22 * j3[i]))));
    }
}
/* HPRIntermediateAcousticTensor::computeMaximumWaveSpeed (HPR/Multiphysics/hprintermediateacoustictensor.cpp:
 * 177-184): the larger of the two materials' single-material acoustic speeds, each at that material's own density
 * and pressure with the shared distortion */
static double hint_speed(const double* W, int d, const double* prm, int k) {
    double b[24], Wk[17];
    hred_mat(prm, k, b);
    Wk[0] = W[16 + 2 * k];
    Wk[1] = W[17 + 2 * k];
    for (int i = 0; i < 15; i++) Wk[2 + i] = W[1 + i];
    return hpr_acoustic_speed(Wk, d, b);
}
/* HPRSolvers::computeMaximumWaveSpeed{,2D} for the intermediate model (Solvers/hprsolvers.cpp:324-341, :387-410) */
static double hint_wave1d(const double* W, const double* prm) {
    return fabs(W[10]) + smax(hint_speed(W, 0, prm, 0), hint_speed(W, 0, prm, 1));
}
static double hint_wave2d(const double* W, const double* prm) {
    return smax(fabs(W[10]), fabs(W[11])) +
           smax(smax(hint_speed(W, 0, prm, 0), hint_speed(W, 0, prm, 1)), smax(hint_speed(W, 1, prm, 0), hint_speed(W, 1, prm, 1)));
}
/* HPRIntermediateStateVector() (:3-21) */
static void hint_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 21; i++) W[i] = 0.0;
    W[0] = 0.999;
    W[1] = 1.0;
    W[5] = 1.0;
    W[9] = 1.0;
    W[16] = 1.0;
    W[17] = 1.0 / 1.4;
    W[18] = 1.0;
    W[19] = 1.0 / 1.4;
}
/* ---- HPR multiphysics two-material model: HPR/Multiphysics/hprmultiphysicsstatevector.cpp (1D only in the
 * reference).  Each material carries its own density, pressure, distortion tensor and heat flux; the velocity is
 * shared.  prm as for the reduced model (the 20-value block of each material); each material's J is carried when that
 * material is thermal.  The distortion enters the conserved vector as pow(alpha_k, 1/3) A_k.
 * W = alpha1, u, v, w, rho1, p1, A1 (9), J1 (3), rho2, p2, A2 (9), J2 (3) (:204-249) and an unused plane;
 * U = rho, rho alpha1, rho u (3), alpha1 rho1, alpha1 rho1 E1, alpha1^(1/3) A1, alpha1 rho1 J1, then the same five
 * groups of material 2 from 19 (:251-317). */
static int hmph_thermal(const double* prm, int k) { return prm[20 * k + 11] != 0.0; }
/* computeConservedVariableVector (:251-317) */
static void hmph_cons(const double* W, const double* prm, double* U) {
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    double rho = (a1 * W[4]) + (a2 * W[18]);
    for (int i = 0; i < 33; i++) U[i] = 0.0;
    U[0] = rho;
    U[1] = rho * a1;
    U[2] = rho * W[1];
    U[3] = rho * W[2];
    U[4] = rho * W[3];
    for (int k = 0; k < 2; k++) {
        double b[24];
        hred_mat(prm, k, b);
        double a = k == 0 ? a1 : a2;
        const double* w = W + 4 + 14 * k; /* rho_k, p_k, A_k (9), J_k (3) */
        double* u = U + 5 + 14 * k;       /* a rho_k, a rho_k E_k, a^(1/3) A_k (9), a rho_k J_k (3) */
        u[0] = a * w[0];
        for (int i = 0; i < 9; i++) u[2 + i] = pow(a, (1.0 / 3.0)) * w[2 + i];
        if (hmph_thermal(prm, k))
            for (int i = 0; i < 3; i++) u[11 + i] = a * (w[0] * w[11 + i]);
        mat3 A = load_A(w + 2);
        double E = hpr_total_energy(w[0], w[1], W[1], W[2], W[3], &A, w[11], w[12], w[13], b);
        u[1] = a * (w[0] * E);
    }
}
/* setConservedVariableVector (:141-202): J_k kept when material k is not thermal */
static void hmph_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    W[1] = U[2] / rho;
    W[2] = U[3] / rho;
    W[3] = U[4] / rho;
    for (int k = 0; k < 2; k++) {
        double b[24];
        hred_mat(prm, k, b);
        double a = k == 0 ? a1 : a2;
        double* w = W + 4 + 14 * k;
        const double* u = U + 5 + 14 * k;
        w[0] = u[0] / a;
        for (int i = 0; i < 9; i++) w[2 + i] = u[2 + i] / pow(a, (1.0 / 3.0));
        if (hmph_thermal(prm, k))
            for (int i = 0; i < 3; i++) w[11 + i] = u[11 + i] / (a * w[0]);
        double E = u[1] / (a * w[0]);
        mat3 A = load_A(w + 2);
        w[1] = hpr_pressure(w[0], E, W[1], W[2], W[3], &A, w[11], w[12], w[13], b);
    }
    W[0] = a1;
}
/* computeXFluxVector (:319-463); the reference has no Y flux for this model */
static void hmph_flux(const double* U, int axis, const double* prm, double* F) {
    (void)axis;
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double vel[3] = {u, v, w};
    double r[2], p[2], E[2], J[2][3];
    mat3 A[2], sg[2];
    for (int k = 0; k < 2; k++) {
        double b[24];
        hred_mat(prm, k, b);
        double a = k == 0 ? a1 : a2;
        const double* c = U + 5 + 14 * k;
        r[k] = c[0] / a;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) A[k].m[i][j] = c[2 + (i * 3) + j] / pow(a, (1.0 / 3.0));
        for (int i = 0; i < 3; i++) J[k][i] = c[11 + i] / (a * r[k]);
        E[k] = c[1] / (a * r[k]);
        p[k] = hpr_pressure(r[k], E[k], u, v, w, &A[k], J[k][0], J[k][1], J[k][2], b);
        sg[k] = shear_stress(r[k], &A[k], b);
    }
    double pi = (a1 * p[0]) + (a2 * p[1]);
    for (int i = 0; i < 33; i++) F[i] = 0.0;
    F[0] = rho * u;
    F[1] = rho * (u * a1);
    F[2] = (rho * (u * u)) + pi;
    F[3] = rho * (u * v);
    F[4] = rho * (u * w);
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2;
        F[5 + 14 * k] = a * (r[k] * u);
        F[6 + 14 * k] = a * ((r[k] * (u * E[k])) + (p[k] * u));
    }
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2;
        F[6 + 14 * k] -= a * (((0.0 + (sg[k].m[0][0] * vel[0])) + (sg[k].m[0][1] * vel[1])) + (sg[k].m[0][2] * vel[2]));
    }
    for (int i = 0; i < 3; i++) F[2 + i] -= (a1 * sg[0].m[0][i]) + (a2 * sg[1].m[0][i]);
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2;
        for (int i = 0; i < 3; i++) {
            double Av = ((0.0 + (A[k].m[i][0] * u)) + (A[k].m[i][1] * v)) + (A[k].m[i][2] * w);
            F[7 + 14 * k + (i * 3)] = pow(a, (1.0 / 3.0)) * Av;
        }
    }
    for (int k = 0; k < 2; k++) {
        if (!hmph_thermal(prm, k)) continue;
        double b[24];
        hred_mat(prm, k, b);
        double a = k == 0 ? a1 : a2;
        double T = mg_temperature(r[k], p[k], b);
        F[6 + 14 * k] += a * (T * ((b[6] * b[6]) * J[k][0]));
        F[16 + 14 * k] = a * ((r[k] * (u * J[k][0])) + T);
        F[17 + 14 * k] = a * (r[k] * (u * J[k][1]));
        F[18 + 14 * k] = a * (r[k] * (u * J[k][2]));
    }
}
/* HPRMultiphysicsAcousticTensor::computeMaximumWaveSpeed (HPR/Multiphysics/hprmultiphysicsacoustictensor.cpp:177-184):
 * each material's single-material acoustic speed at its own density, pressure and distortion; material 2's reads the
 * diagonal dsigma/dA entries in its second block (:61) */
static double hmph_speed(const double* W, int d, const double* prm, int k) {
    double b[24], Wk[17];
    hred_mat(prm, k, b);
    const double* w = W + 4 + 14 * k;
    Wk[0] = w[0];
    Wk[1] = w[1];
    for (int i = 0; i < 9; i++) Wk[2 + i] = w[2 + i];
    Wk[11] = W[1];
    Wk[12] = W[2];
    Wk[13] = W[3];
    for (int i = 0; i < 3; i++) Wk[14 + i] = w[11 + i];
    return hpr_acoustic_speed_q(Wk, d, b, k == 1);
}
/* HPRSolvers::computeMaximumWaveSpeed for the multiphysics model (Solvers/hprsolvers.cpp:305-322) */
static double hmph_wave1d(const double* W, const double* prm) {
    return fabs(W[1]) + smax(hmph_speed(W, 0, prm, 0), hmph_speed(W, 0, prm, 1));
}
static double hmph_wave2d(const double* W, const double* prm) { (void)W; (void)prm; return NAN; }
/* HPRMultiphysicsStateVector() (:3-26) */
static void hmph_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 33; i++) W[i] = 0.0;
    W[0] = 0.999;
    for (int k = 0; k < 2; k++) {
        double* w = W + 4 + 14 * k;
        w[0] = 1.0;
        w[1] = 1.0 / 1.4;
        w[2] = 1.0;
        w[6] = 1.0;
        w[10] = 1.0;
    }
}
/* setPrimitiveVariableVector (:98-139) takes material k's J only when that material is thermal; otherwise the cells
 * keep the default J_k = 0, which nothing reads */
static void hmph_drop_cold_heat_flux(int id, double* planes, long n, const double* prm) {
    if (id != VO_HPR_MULTIPHYSICS) return;
    for (int k = 0; k < 2; k++)
        if (!hmph_thermal(prm, k))
            for (long i = (15 + 14 * k) * n; i < (18 + 14 * k) * n; i++) planes[i] = 0.0;
}
/* MultiphysicsSolvers::reinitialiseVolumeFraction for the HPR multiphysics model (Solvers/multiphysicssolvers.cpp:
 * 807-839; 1D): the last cell i >= 1 with alpha_i < 0.5 <= alpha_{i-1}, or 0, and the window i-2 .. i+1, whose cells
 * relax the density, pressure, distortion (pow(alpha_k, 1/3)-weighted) and heat flux components of both materials to
 * their mixtures (:614-704) with the cell's own alpha, then take 0.999 | 0.001.  Window cells outside the grid, which
 * the reference writes out of bounds, are skipped. */
static void hmph_reinit(double* planes, int nx) {
    long plane = nx;
    int loc = 0;
    for (int i = 1; i < nx; i++)
        if (planes[i] < 0.5 && planes[i - 1] >= 0.5) loc = i;
    for (int i = loc - 2; i < loc + 2; i++) {
        if (i < 0 || i >= nx) continue;
        double a1 = planes[i], a2 = 1.0 - a1;
#define HM(v) planes[(long)(v) * plane + i]
        double rho = (a1 * HM(4)) + (a2 * HM(18));
        HM(4) = rho;
        HM(18) = rho;
        double p = (a1 * HM(5)) + (a2 * HM(19));
        HM(5) = p;
        HM(19) = p;
        for (int e = 0; e < 9; e++) {
            double A = (pow(a1, (1.0 / 3.0)) * HM(6 + e)) + (pow(a2, (1.0 / 3.0)) * HM(20 + e));
            HM(6 + e) = A;
            HM(20 + e) = A;
        }
        for (int e = 0; e < 3; e++) {
            double J = (a1 * HM(15 + e)) + (a2 * HM(29 + e));
            HM(15 + e) = J;
            HM(29 + e) = J;
        }
#undef HM
        planes[i] = i < loc ? 0.999 : 0.001;
    }
}
/* ---- MHD multiphysics two-material model: MHD/Multiphysics/mhdmultiphysicsstatevector.cpp (1D only in the
 * reference).  Each material carries its own density, pressure, magnetic field and GLM scalar; the velocity is shared.
 * prm = {gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2}: the materials' hyperbolic wave speeds stay as given, since the
 * reference's solve sets none (Solvers/mhdsecondordersolver.cpp:362-385).
 * W = alpha1, u, v, w, rho1, p1, B1 (3), psi1, rho2, p2, B2 (3), psi2 (:135-163) and an unused plane;
 * U = rho, rho alpha1, rho u (3), then per material k at 5 + 6 k: alpha rho, alpha E, alpha^(1/2) B (3), alpha psi
 * (:165-220). */
/* computeConservedVariableVector (:165-220) */
static void mmph_cons(const double* W, const double* prm, double* U) {
    double a1 = red_clamp(W[0]), a2 = 1.0 - a1;
    double u = W[1], v = W[2], w = W[3];
    double rho = (a1 * W[4]) + (a2 * W[10]);
    for (int i = 0; i < 17; i++) U[i] = 0.0;
    U[0] = rho;
    U[1] = rho * a1;
    U[2] = rho * u;
    U[3] = rho * v;
    U[4] = rho * w;
    double v2 = ((u * u) + (v * v)) + (w * w);
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2;
        const double* wk = W + 4 + 6 * k; /* rho, p, B (3), psi */
        double* uk = U + 5 + 6 * k;
        uk[0] = a * wk[0];
        double b2 = ((wk[2] * wk[2]) + (wk[3] * wk[3])) + (wk[4] * wk[4]);
        double h = wk[0] * ((0.5 * v2) + mhd_e(wk[0], wk[1], prm + 2 * k));
        uk[1] = a * (h + (0.5 * b2));
        for (int i = 0; i < 3; i++) uk[2 + i] = pow(a, 1.0 / 2.0) * wk[2 + i];
        uk[5] = a * wk[5];
    }
}
/* setConservedVariableVector (:84-133) */
static void mmph_setcons(const double* U, const double* prm, double* W) {
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double v2 = ((u * u) + (v * v)) + (w * w);
    W[1] = u;
    W[2] = v;
    W[3] = w;
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2;
        double* wk = W + 4 + 6 * k;
        const double* uk = U + 5 + 6 * k;
        wk[0] = uk[0] / a;
        for (int i = 0; i < 3; i++) wk[2 + i] = uk[2 + i] / pow(a, 1.0 / 2.0);
        double b2 = ((wk[2] * wk[2]) + (wk[3] * wk[3])) + (wk[4] * wk[4]);
        double E = ((uk[1] / a) - (0.5 * b2)) / wk[0];
        wk[1] = mhd_p(wk[0], E - (0.5 * v2), prm + 2 * k);
        wk[5] = uk[5] / a;
    }
    W[0] = a1;
}
/* computeXFluxVector (:222-358); the reference has no Y flux for this model.  The interface field components are
 * pow(alpha1 B1^2 + alpha2 B2^2, 1/2) per component; each material's energy flux carries its own field. */
static void mmph_flux(const double* U, int axis, const double* prm, double* F) {
    (void)axis;
    double rho = U[0];
    double a1 = red_clamp(U[1] / rho), a2 = 1.0 - a1;
    double u = U[2] / rho, v = U[3] / rho, w = U[4] / rho;
    double r[2], B[2][3], psi[2], Et[2], p[2], b2[2];
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2;
        const double* uk = U + 5 + 6 * k;
        r[k] = uk[0] / a;
        for (int i = 0; i < 3; i++) B[k][i] = uk[2 + i] / pow(a, 1.0 / 2.0);
        psi[k] = uk[5] / a;
    }
    double IB2[3], IB[3];
    for (int i = 0; i < 3; i++) {
        IB2[i] = (a1 * (B[0][i] * B[0][i])) + (a2 * (B[1][i] * B[1][i]));
        IB[i] = pow(IB2[i], 1.0 / 2.0);
    }
    double v2 = ((u * u) + (v * v)) + (w * w);
    double ib2 = (IB2[0] + IB2[1]) + IB2[2];
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2;
        b2[k] = ((B[k][0] * B[k][0]) + (B[k][1] * B[k][1])) + (B[k][2] * B[k][2]);
        Et[k] = U[6 + 6 * k] / a;
        double e = ((Et[k] - (0.5 * b2[k])) / r[k]) - (0.5 * v2);
        p[k] = mhd_p(r[k], e, prm + 2 * k);
    }
    for (int i = 0; i < 17; i++) F[i] = 0.0;
    F[0] = rho * u;
    F[1] = rho * (u * a1);
    F[2] = (((rho * (u * u)) + ((a1 * p[0]) + (a2 * p[1]))) + (0.5 * ib2)) - IB2[0];
    F[3] = (rho * (u * v)) - (IB[0] * IB[1]);
    F[4] = (rho * (u * w)) - (IB[0] * IB[2]);
    for (int k = 0; k < 2; k++) {
        double a = k == 0 ? a1 : a2, ch = prm[4 + k];
        double* fk = F + 5 + 6 * k;
        fk[0] = a * (r[k] * u);
        double bv = ((0.0 + (u * B[k][0])) + (v * B[k][1])) + (w * B[k][2]);
        fk[1] = (a * (((Et[k] + p[k]) + (0.5 * b2[k])) * u)) - (a * (bv * B[k][0]));
        fk[2] = pow(a, 1.0 / 2.0) * psi[k];
        fk[3] = pow(a, 1.0 / 2.0) * ((B[k][1] * u) - (B[k][0] * v));
        fk[4] = pow(a, 1.0 / 2.0) * ((B[k][2] * u) - (B[k][0] * w));
        fk[5] = a * ((ch * ch) * B[k][0]);
    }
}
/* MHDSolvers::computeMaximumWaveSpeed for the multiphysics model (Solvers/mhdsolvers.cpp:305-323): each material's
 * fast magneto-acoustic speed at its own density, pressure and field */
static double mmph_wave1d(const double* W, const double* prm) {
    double V1[9] = {W[4], 0.0, 0.0, 0.0, W[5], W[6], W[7], W[8], 0.0};
    double V2[9] = {W[10], 0.0, 0.0, 0.0, W[11], W[12], W[13], W[14], 0.0};
    return fabs(W[1]) + smax(fabs(mhd_fast(V1, prm, W[6])), fabs(mhd_fast(V2, prm + 2, W[12])));
}
static double mmph_wave2d(const double* W, const double* prm) { (void)W; (void)prm; return NAN; }
/* MHDMultiphysicsStateVector() (:3-27) */
static void mmph_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 17; i++) W[i] = 0.0;
    W[0] = 0.999;
    W[4] = 1.0;
    W[5] = 1.0;
    W[10] = 1.0;
    W[11] = 1.0;
}
/* HPRReducedStateVector() (:3-19) */
static void hred_default(const double* prm, double* W) {
    (void)prm;
    for (int i = 0; i < 20; i++) W[i] = 0.0;
    W[0] = 0.999;
    W[1] = 1.0 / 1.4;
    W[2] = 1.0;
    W[6] = 1.0;
    W[10] = 1.0;
    W[17] = 1.0;
    W[18] = 1.0;
}

/* A cell of a reinitialisation window: relaxTotalDensity (reduced :281-287, multiphysics :308-314), for the
 * multiphysics model relaxTotalPressure (:316-329, which sets both pressures to the volume-fraction mean), then the
 * volume fraction.  Planes: reduced rho1 4, rho2 5; multiphysics rho1 4, p1 5, rho2 6, p2 7. */
static int g_reinit_mph = 0;
/* density and pressure planes: reduced models rho1 4, rho2 5 (HPR reduced 17, 18); multiphysics and MHD intermediate
 * rho1 4, p1 5, rho2 6, p2 7; HPR intermediate rho1 16, p1 17, rho2 18, p2 19 */
static int g_reinit_r1 = 4, g_reinit_r2 = 5, g_reinit_p1 = 5, g_reinit_p2 = 7;
static void red_reset_cell(double* planes, long plane, long idx, double alpha) {
    double a1 = planes[idx];
    int i1 = g_reinit_r1, i2 = g_reinit_r2;
    double rho = (a1 * planes[i1 * plane + idx]) + ((1.0 - a1) * planes[i2 * plane + idx]);
    planes[i1 * plane + idx] = rho;
    planes[i2 * plane + idx] = rho;
    if (g_reinit_mph) {
        double p = (a1 * planes[g_reinit_p1 * plane + idx]) + ((1.0 - a1) * planes[g_reinit_p2 * plane + idx]);
        planes[g_reinit_p1 * plane + idx] = p;
        planes[g_reinit_p2 * plane + idx] = p;
    }
    planes[idx] = alpha;
}
/* MultiphysicsSolvers::reinitialiseVolumeFraction for the reduced model (Solvers/multiphysicssolvers.cpp:164-191 in
 * 1D, :193-... in 2D).  1D: the last cell i >= 1 with alpha_i < 0.5 <= alpha_{i-1} (the loop's single-thread
 * outcome; i = 0 would read cell -1), or 0, and the window i-2 .. i+1.  2D: per row, then per column, every such
 * descending crossing (window set to 0.999 | 0.001) and every ascending one (alpha_j > 0.5 >= alpha_{j-1}; 0.001 |
 * 0.999), at most 100 of each kind per line.  Window cells outside the grid, which the reference writes out of
 * bounds, are skipped. */
static void red_reinit_line(double* planes, long plane, long start, long stride, int len) {
    int loc1[100], loc2[100], n1 = 0, n2 = 0;
    for (int j = 1; j < len; j++) {
        double a = planes[start + j * stride], b = planes[start + (j - 1) * stride];
        if (a < 0.5 && b >= 0.5 && n1 < 100) loc1[n1++] = j;
        if (a > 0.5 && b <= 0.5 && n2 < 100) loc2[n2++] = j;
    }
    for (int k = 0; k < n1; k++)
        for (int j = loc1[k] - 2; j < loc1[k] + 2; j++)
            if (j >= 0 && j < len) red_reset_cell(planes, plane, start + j * stride, j < loc1[k] ? 0.999 : 0.001);
    for (int k = 0; k < n2; k++)
        for (int j = loc2[k] - 2; j < loc2[k] + 2; j++)
            if (j >= 0 && j < len) red_reset_cell(planes, plane, start + j * stride, j < loc2[k] ? 0.001 : 0.999);
}
static void red_reinit(double* planes, int nx, int ny) {
    long plane = (long)nx * ny;
    if (ny == 1) {
        int loc = 0;
        for (int i = 1; i < nx; i++)
            if (planes[i] < 0.5 && planes[i - 1] >= 0.5) loc = i;
        for (int i = loc - 2; i < loc + 2; i++)
            if (i >= 0 && i < nx) red_reset_cell(planes, plane, i, i < loc ? 0.999 : 0.001);
        return;
    }
    for (int i = 0; i < ny; i++) red_reinit_line(planes, plane, (long)i * nx, 1, nx);
    for (int j = 0; j < nx; j++) red_reinit_line(planes, plane, j, nx, ny);
}

static const model M_EULER = {6, euler_cons, euler_setcons, euler_flux, euler_wave1d, euler_wave2d, euler_default, 0};
static const model M_MHD = {9, mhd_cons, mhd_setcons, mhd_flux, mhd_wave1d, mhd_wave2d, mhd_default, mhd_source};
static const model M_HPR = {17, hpr_cons, hpr_setcons, hpr_flux, hpr_wave1d, hpr_wave2d, hpr_default, hpr_source};
static const model M_RED = {8, red_cons, red_setcons, red_flux, red_wave1d, red_wave2d, red_default, 0};
static const model M_MPH = {9, mph_cons, mph_setcons, mph_flux, mph_wave1d, mph_wave2d, mph_default, 0};
static const model M_MRED = {12, mred_cons, mred_setcons, mred_flux, mred_wave1d, mred_wave2d, mred_default, mred_source};
static const model M_MINT = {13, mint_cons, mint_setcons, mint_flux, mint_wave1d, mint_wave2d, mint_default, mint_source};
static const model M_HRED = {20, hred_cons, hred_setcons, hred_flux, hred_wave1d, hred_wave2d, hred_default, hred_source};
static const model M_HINT = {21, hint_cons, hint_setcons, hint_flux, hint_wave1d, hint_wave2d, hint_default, hint_source};
static const model M_HMPH = {33, hmph_cons, hmph_setcons, hmph_flux, hmph_wave1d, hmph_wave2d, hmph_default, 0};
static const model M_MMPH = {17, mmph_cons, mmph_setcons, mmph_flux, mmph_wave1d, mmph_wave2d, mmph_default, 0};

static const model* model_of(int id) {
    switch (id) {
        case VO_EULER: return &M_EULER;
        case VO_MHD: return &M_MHD;
        case VO_HPR: return &M_HPR;
        case VO_EULER_REDUCED: return &M_RED;
        case VO_EULER_MULTIPHYSICS: return &M_MPH;
        case VO_MHD_REDUCED: return &M_MRED;
        case VO_MHD_INTERMEDIATE: return &M_MINT;
        case VO_HPR_REDUCED: return &M_HRED;
        case VO_HPR_INTERMEDIATE: return &M_HINT;
        case VO_HPR_MULTIPHYSICS: return &M_HMPH;
        case VO_MHD_MULTIPHYSICS: return &M_MMPH;
        default: return NULL;
    }
}

int vo_nvar(int id) { const model* m = model_of(id); return m ? m->nv : 0; }
int vo_nparams(int id) {
    return id == VO_EULER ? 6 : id == VO_MHD ? 3 : id == VO_HPR ? 20 : (id == VO_EULER_REDUCED || id == VO_EULER_MULTIPHYSICS) ? 4 : (id == VO_MHD_REDUCED || id == VO_MHD_INTERMEDIATE) ? 5 : id == VO_MHD_MULTIPHYSICS ? 6 : (id == VO_HPR_REDUCED || id == VO_HPR_INTERMEDIATE || id == VO_HPR_MULTIPHYSICS) ? 40 : 0;
}

/* ------------------------------------------------------------------------------- SLIC building blocks */

/* Solvers::evolveStateByHalf{X,Y}TimeStep + evolveStateByHalfTimeStep + computeEvolutionVector,
 * Solvers/solvers.cpp:454-466, :502-514, :550-565, :601-609.  Returns primitives (the reference
 * stores the evolved state in a default-constructed state vector). */
static void evolve_half(const model* m, const double* wl, const double* wm, const double* wr, int axis,
                        double dx, double dt, double w, int lim, int side, const double* prm, double* out) {
    double uL[MAXV], uM[MAXV], uR[MAXV], s[MAXV], xl[MAXV], xr[MAXV], fl[MAXV], fr[MAXV], ev[MAXV];
    int nv = m->nv;
    m->cons(wl, prm, uL);
    m->cons(wm, prm, uM);
    m->cons(wr, prm, uR);
    slope_vector(nv, uL, uM, uR, w, lim, s);
    for (int i = 0; i < nv; i++) {
        xl[i] = uM[i] + (-1.0 * (0.5 * s[i]));
        xr[i] = uM[i] + (0.5 * s[i]);
    }
    m->flux(xl, axis, prm, fl);
    m->flux(xr, axis, prm, fr);
    double c = 0.5 * (dt / dx);
    for (int i = 0; i < nv; i++) ev[i] = c * (fl[i] + (-1.0 * fr[i]));
    double sum[MAXV];
    for (int i = 0; i < nv; i++) sum[i] = (side == 0 ? xl[i] : xr[i]) + ev[i];
    m->default_state(prm, out);
    m->setcons(sum, prm, out);
}

/* FirstOrderSolver::compute{X,Y}FORCEFlux with its Lax-Friedrichs and Richtmyer halves,
 * Solvers/firstordersolver.cpp:7-17, :79-85, :87-98, :165-171, :173-180, :227-230. */
static void force_flux(const model* m, const double* wa, const double* wb, int axis, double dx, double dt,
                       const double* prm, double* F) {
    double ua[MAXV], ub[MAXV], fa[MAXV], fb[MAXV], uri[MAXV], fri[MAXV], lf[MAXV];
    int nv = m->nv;
    m->cons(wa, prm, ua);
    m->cons(wb, prm, ub);
    m->flux(ua, axis, prm, fa);
    m->flux(ub, axis, prm, fb);
    double rinv = dx / dt, r = dt / dx;
    for (int i = 0; i < nv; i++) lf[i] = 0.5 * ((fa[i] + fb[i]) + (rinv * (ua[i] + (-1.0 * ub[i]))));
    for (int i = 0; i < nv; i++) uri[i] = 0.5 * ((ua[i] + ub[i]) + (r * (fa[i] + (-1.0 * fb[i]))));
    m->flux(uri, axis, prm, fri);
    for (int i = 0; i < nv; i++) F[i] = 0.5 * (lf[i] + fri[i]);
}

/* SecondOrderSolver::compute{X,Y}SLICFlux, Solvers/secondordersolver.cpp:7-17, :43-53 */
static void slic_flux(const model* m, const double* wLL, const double* wL, const double* wR, const double* wRR,
                      int axis, double dx, double dt, double w, int lim, const double* prm, double* F) {
    double a[MAXV], b[MAXV];
    evolve_half(m, wLL, wL, wR, axis, dx, dt, w, lim, 1, prm, a);
    evolve_half(m, wL, wR, wRR, axis, dx, dt, w, lim, 0, prm, b);
    force_flux(m, a, b, axis, dx, dt, prm, F);
}

/* ------------------------------------------------------------------------------------ grids */

/* Ghost index along one axis of length n with 2 ghosts: transmissive mirror (Solvers/solvers.cpp:17-23)
 * or wrap-around; k runs over -2 .. n+1. */
static int ghost_index(int k, int n, int bc) {
    if (k >= 0 && k < n) return k;
    if (bc == VO_BC_PERIODIC) return (k < 0) ? k + n : k - n;
    return (k < 0) ? (-1 - k) : (2 * n - 1 - k);
}

static void load_cell(const double* planes, long plane, long idx, int nv, double* W) {
    for (int v = 0; v < nv; v++) W[v] = planes[v * plane + idx];
}

/* One sweep of compute{X,Y}SLICTimeStep2D (Solvers/secondordersolver.cpp:140-162, :214-236) over a
 * grid with ncol columns, nrow rows.  Each interface flux is a pure function of its 4-cell stencil, so
 * computing it once and using it for both neighbours gives the reference's values. */
static void sweep_grid(const model* m, double* planes, int nx, int ny, int axis, double dx, double dt,
                       double w, int lim, const double* prm, int bc) {
    long plane = (long)nx * ny;
    int nv = m->nv;
    int nline = axis == 0 ? ny : nx, len = axis == 0 ? nx : ny;
    double* out = (double*)malloc(sizeof(double) * nv * plane);
    double r = dt / dx;
#pragma omp parallel for schedule(static)
    for (int line = 0; line < nline; line++) {
        double* fl = (double*)malloc(sizeof(double) * MAXV * (len + 1));
        double st[4][MAXV];
        for (int f = 0; f <= len; f++) {
            /* interface f sits between cells f-1 and f; stencil cells f-2 .. f+1 */
            for (int s = 0; s < 4; s++) {
                int k = ghost_index(f - 2 + s, len, bc);
                long idx = axis == 0 ? (long)line * nx + k : (long)k * nx + line;
                load_cell(planes, plane, idx, nv, st[s]);
            }
            slic_flux(m, st[0], st[1], st[2], st[3], axis, dx, dt, w, lim, prm, fl + (long)f * MAXV);
        }
        for (int c = 0; c < len; c++) {
            long idx = axis == 0 ? (long)line * nx + c : (long)c * nx + line;
            double W[MAXV], U[MAXV], Un[MAXV];
            load_cell(planes, plane, idx, nv, W);
            m->cons(W, prm, U);
            /* FirstOrderSolver::computeFORCEUpdate, Solvers/firstordersolver.cpp:428-433 */
            for (int v = 0; v < nv; v++)
                Un[v] = U[v] + (r * (fl[(long)c * MAXV + v] + (-1.0 * fl[(long)(c + 1) * MAXV + v])));
            m->setcons(Un, prm, W);
            for (int v = 0; v < nv; v++) out[v * plane + idx] = W[v];
        }
        free(fl);
    }
    memcpy(planes, out, sizeof(double) * nv * plane);
    free(out);
}

void vo_sweep2d(int id, double* planes, int nx, int ny, int axis, double dx, double dt, double w, int lim,
                const double* prm, int bc) {
    const model* m = model_of(id);
    if (!m) return;
    sweep_grid(m, planes, nx, ny, axis, dx, dt, w, lim, prm, bc);
}

void vo_sweep1d(int id, double* planes, int n, double dx, double dt, double w, int lim, const double* prm,
                int bc) {
    const model* m = model_of(id);
    if (!m) return;
    sweep_grid(m, planes, n, 1, 0, dx, dt, w, lim, prm, bc);
}

/* computeMaximumWaveSpeed over the 2-ghost padded line: ghosts are copies of interior cells, so the
 * maximum is over the interior (Solvers/solvers.cpp:259-276; `if (s > max) max = s` from 0.0). */
static double max_wave(const model* m, const double* planes, long plane, int dims, const double* prm) {
    double best = 0.0;
    for (long k = 0; k < plane; k++) {
        double W[MAXV];
        load_cell(planes, plane, k, m->nv, W);
        double s = dims == 1 ? m->wave1d(W, prm) : m->wave2d(W, prm);
        if (s > best) best = s;
    }
    if (dims == 2) {
        /* the default-constructed corner ghosts of insertBoundaryCells2D (Solvers/solvers.cpp:92) */
        double W[MAXV];
        m->default_state(prm, W);
        double s = m->wave2d(W, prm);
        if (s > best) best = s;
    }
    return best;
}

double vo_max_wave1d(int id, const double* planes, int n, const double* prm) {
    const model* m = model_of(id);
    return m ? max_wave(m, planes, n, 1, prm) : 0.0;
}

double vo_max_wave2d(int id, const double* planes, int nx, int ny, const double* prm) {
    const model* m = model_of(id);
    return m ? max_wave(m, planes, (long)nx * ny, 2, prm) : 0.0;
}

/* ------------------------------------------------------------------------- HPR relaxation source (RK4) */

/* HPRSolvers::evolveStateByFractional{X,Y}TimeStep (Solvers/hprsolvers.cpp:606-620, :673-687) with
 * evolveStateByFractionalTimeStep (:791-797): the middle state advanced by frac * dt of the flux difference of
 * its own slope-limited edge values; returns primitives (default-constructed target). */
static void frac_evolve(const model* m, double frac, const double* wl, const double* wm, const double* wr, int axis,
                        double dx, double dt, double w, int lim, const double* prm, double* out) {
    double uL[MAXV], uM[MAXV], uR[MAXV], s[MAXV], xl[MAXV], xr[MAXV], fl[MAXV], fr[MAXV], sum[MAXV];
    int nv = m->nv;
    m->cons(wl, prm, uL);
    m->cons(wm, prm, uM);
    m->cons(wr, prm, uR);
    slope_vector(nv, uL, uM, uR, w, lim, s);
    for (int i = 0; i < nv; i++) {
        xl[i] = uM[i] + (-1.0 * (0.5 * s[i]));
        xr[i] = uM[i] + (0.5 * s[i]);
    }
    m->flux(xl, axis, prm, fl);
    m->flux(xr, axis, prm, fr);
    double c = frac * (dt / dx);   /* Solvers::computeFractionalEvolutionVector (Solvers/solvers.cpp:606-609) */
    for (int i = 0; i < nv; i++) sum[i] = uM[i] + (c * (fl[i] + (-1.0 * fr[i])));
    m->default_state(prm, out);
    m->setcons(sum, prm, out);
}

static void prim_of(const model* m, const double* u, const double* prm, double* w) {
    m->default_state(prm, w);
    m->setcons(u, prm, w);
}

/* HPRForcingSolver::evolveConservedVariableVector{,2D} (Solvers/hprforcingsolver.cpp:7-44, :134-194) and
 * computeEvolvedConservedVariableVector (:332-339); MHDForcingSolver's are the same steps with the MHD model
 * (Solvers/mhdforcingsolver.cpp:7-44, :134-194).  dims == 1 uses the X predictor alone with fractions
 * (1/2, 1/2, 1); dims == 2 the X(f/2) Y(f) X(f/2) predictor with f = 1/2, 1/2, 1. */
static void rk4_source(const model* m, const double* uLf, const double* uM, const double* uRf, const double* uTf,
                       const double* uBf, int dims, double dx, double dt, double w, int lim, const double* prm,
                       double* result) {
    int nv = m->nv;
    double wl[MAXV], wr[MAXV], wt[MAXV], wb[MAXV], wm[MAXV], e1[MAXV], e2[MAXV], e[MAXV], ue[MAXV], S[MAXV];
    double k[4][MAXV], ut[MAXV];
    prim_of(m, uLf, prm, wl);
    prim_of(m, uRf, prm, wr);
    if (dims == 2) {
        prim_of(m, uTf, prm, wt);
        prim_of(m, uBf, prm, wb);
    }
    m->default_state(prm, wm);
    m->source(uM, prm, S);
    for (int i = 0; i < nv; i++) k[0][i] = dt * S[i];
    static const double stage[3] = {0.5, 0.5, 1.0};
    for (int s = 0; s < 3; s++) {
        for (int i = 0; i < nv; i++) ut[i] = uM[i] + (s < 2 ? (0.5 * k[s][i]) : k[s][i]);
        m->setcons(ut, prm, wm);
        double f = stage[s];
        if (dims == 1) {
            frac_evolve(m, f, wl, wm, wr, 0, dx, dt, w, lim, prm, e);
        } else {
            frac_evolve(m, 0.5 * f, wl, wm, wr, 0, dx, dt, w, lim, prm, e1);
            frac_evolve(m, f, wt, e1, wb, 1, dx, dt, w, lim, prm, e2);
            frac_evolve(m, 0.5 * f, wl, e2, wr, 0, dx, dt, w, lim, prm, e);
        }
        m->cons(e, prm, ue);
        m->source(ue, prm, S);
        for (int i = 0; i < nv; i++) k[s + 1][i] = dt * S[i];
    }
    for (int i = 0; i < nv; i++)
        result[i] = uM[i] + ((1.0 / 6.0) * (k[0][i] + ((2.0 * k[1][i]) + ((2.0 * k[2][i]) + k[3][i]))));
}

/* 1-ghost boundary of insertBoundaryCells{,2D}(cells, 1): transmissive copies g[-1] = c[0], g[n] = c[n-1]
 * (Solvers/hprsolvers.cpp, same layout as Solvers/solvers.cpp:11-15) or wrap-around. */
static int ghost1(int k, int n, int bc) {
    if (k >= 0 && k < n) return k;
    if (bc == VO_BC_PERIODIC) return k < 0 ? k + n : k - n;
    return k < 0 ? 0 : n - 1;
}

/* HPRForcingSolver::computeRungeKuttaTimeStep{,2D} (Solvers/hprforcingsolver.cpp:341-357, :394-418) and
 * MHDForcingSolver's (Solvers/mhdforcingsolver.cpp:341-357, :394-418) */
static void forcing_grid(const model* m, double* planes, int nx, int ny, int dims, double dx, double dt, double w,
                         int lim, const double* prm, int bc) {
    long plane = (long)nx * ny;
    int nv = m->nv;
    double* out = (double*)malloc(sizeof(double) * nv * plane);
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < plane; idx++) {
        int i = (int)(idx / nx), j = (int)(idx - (long)i * nx);
        double W[MAXV], uL[MAXV], uM[MAXV], uR[MAXV], uT[MAXV], uB[MAXV], res[MAXV];
        load_cell(planes, plane, (long)i * nx + ghost1(j - 1, nx, bc), nv, W);
        m->cons(W, prm, uL);
        load_cell(planes, plane, (long)i * nx + ghost1(j + 1, nx, bc), nv, W);
        m->cons(W, prm, uR);
        if (dims == 2) {
            load_cell(planes, plane, (long)ghost1(i - 1, ny, bc) * nx + j, nv, W);
            m->cons(W, prm, uT);
            load_cell(planes, plane, (long)ghost1(i + 1, ny, bc) * nx + j, nv, W);
            m->cons(W, prm, uB);
        }
        load_cell(planes, plane, idx, nv, W);
        m->cons(W, prm, uM);
        rk4_source(m, uL, uM, uR, uT, uB, dims, dx, dt, w, lim, prm, res);
        m->setcons(res, prm, W);
        for (int v = 0; v < nv; v++) out[v * plane + idx] = W[v];
    }
    memcpy(planes, out, sizeof(double) * nv * plane);
    free(out);
}

void vo_forcing(int id, double* planes, int nx, int ny, double dx, double dt, double w, int lim, const double* prm,
                int bc) {
    const model* m = model_of(id);
    if (!m || !m->source) return;
    forcing_grid(m, planes, nx, ny, ny > 1 ? 2 : 1, dx, dt, w, lim, prm, bc);
}

void vo_hpr_cell(const double* w, const double* prm, double* u, double* fx, double* fy, double* src, double* speed_xy) {
    hpr_cons(w, prm, u);
    hpr_flux(u, 0, prm, fx);
    hpr_flux(u, 1, prm, fy);
    hpr_source(u, prm, src);
    speed_xy[0] = hpr_acoustic_speed(w, 0, prm);
    speed_xy[1] = hpr_acoustic_speed(w, 1, prm);
}

void vo_hpr_eos(const double* prm, const double* rho, const double* p, const double* e, int n, double* out) {
    for (int k = 0; k < n; k++) {
        double r = rho[k], *o = out + 13 * k;
        o[0] = mg_G(r, prm);
        o[1] = mg_pref(r, prm);
        o[2] = mg_eref(r, prm);
        o[3] = mg_dG(r, prm);
        o[4] = mg_dpref(r, prm);
        o[5] = mg_deref(r, prm);
        o[6] = mg_energy(r, p[k], prm);
        o[7] = mg_pressure(r, e[k], prm);
        o[8] = mg_temperature(r, p[k], prm);
        o[9] = mg_dedrho(r, p[k], prm);
        o[10] = mg_dedp(r, prm);
        o[11] = mg_dTdrho(r, p[k], prm);
        o[12] = mg_dTdp(r, prm);
    }
}

void vo_hpr_theta1(const double* prm, const double* rho, const double* a9, int n, double* out) {
    for (int k = 0; k < n; k++) {
        mat3 A = load_A(a9 + 9 * k);
        out[k] = hpr_theta1(rho[k], &A, prm);
    }
}

/* the stiff relaxation of every cell of the grid (see hpr_relax_cell) */
static void relax_grid(const model* m, double* planes, long plane, double h, const double* prm) {
    int nv = m->nv;
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < plane; idx++) {
        double W[MAXV], U[MAXV];
        load_cell(planes, plane, idx, nv, W);
        m->cons(W, prm, U);
        hpr_relax_cell(U, h, prm);
        m->setcons(U, prm, W);
        for (int v = 0; v < nv; v++) planes[v * plane + idx] = W[v];
    }
}

/* Solvers::computeStableTimeStep(dt, t, tEnd, it), Solvers/solvers.cpp:437-452 */
static double stable_dt(double dt, double t, double t_end, int it) {
    double d = dt;
    if (it <= 5) d *= 0.2;
    if ((t + d) > t_end) d = t_end - t;
    return d;
}

/* solve()/solve2D()'s loop: Solvers/secondordersolver.cpp:288-314 (1D), :392-424 (2D); MHD adds
 * c_h = padded-grid maximum wave speed before the sweeps (Solvers/mhdsecondordersolver.cpp:330-332,
 * :513-515). */
static double run(int id, double* planes, int nx, int ny, int dims, double dx, double cfl, double t_end,
                  int max_steps, double w, int lim, const double* prm_in, int bc, int subcycles, int* steps_out,
                  double* dt_log, int reinit_freq) {
    const model* m = model_of(id);
    if (!m) return -1.0;
    double prm[48];
    memcpy(prm, prm_in, sizeof(double) * vo_nparams(id));
    double tEnd = t_end > 0.0 ? t_end : 1.0e300;
    int limit = max_steps > 0 ? max_steps : 0x7fffffff;
    long plane = (long)nx * ny;
    double t = 0.0;
    int it = 0;
    /* subcycles < 0 (HPR): the stiff relaxation of dt/2 before and after the sweeps instead of the RK4 forcing */
    int stiff = id == VO_HPR && subcycles < 0;
    int sub = (m->source && subcycles > 0) ? subcycles : 0;
    while (t < tEnd && it < limit) {
        double smax_ = max_wave(m, planes, plane, dims, prm);
        double dt = stable_dt(cfl * (dx / smax_), t, tEnd, it);
        if (id == VO_MHD) prm[2] = smax_;
        if (id == VO_MHD_REDUCED || id == VO_MHD_INTERMEDIATE) prm[4] = smax_;
        if (dt_log) dt_log[it] = dt;
        /* HPR relaxation / MHD GLM damping: sub-cycled RK4 source before and after the sweeps
         * (Solvers/hprsecondordersolver.cpp:323-341, :514-541; Solvers/mhdsecondordersolver.cpp:334-348, :517-540) */
        for (int s = 0; s < sub; s++) forcing_grid(m, planes, nx, ny, dims, dx, 0.5 * (dt / sub), w, lim, prm, bc);
        if (stiff) relax_grid(m, planes, plane, 0.5 * dt, prm);
        if (dims == 1) {
            sweep_grid(m, planes, nx, 1, 0, dx, dt, w, lim, prm, bc);
        } else {
            sweep_grid(m, planes, nx, ny, 0, dx, 0.5 * dt, w, lim, prm, bc);
            sweep_grid(m, planes, nx, ny, 1, dx, dt, w, lim, prm, bc);
            sweep_grid(m, planes, nx, ny, 0, dx, 0.5 * dt, w, lim, prm, bc);
        }
        for (int s = 0; s < sub; s++) forcing_grid(m, planes, nx, ny, dims, dx, 0.5 * (dt / sub), w, lim, prm, bc);
        if (stiff) relax_grid(m, planes, plane, 0.5 * dt, prm);
        t += dt;
        it += 1;
        /* the reduced model's solve{,2D}: reinitialisation every reinit_freq steps (Solvers/secondordersolver.cpp) */
        if ((id == VO_EULER_REDUCED || id == VO_EULER_MULTIPHYSICS || id == VO_MHD_REDUCED ||
             id == VO_MHD_INTERMEDIATE || id == VO_HPR_REDUCED || id == VO_HPR_INTERMEDIATE) && reinit_freq != 0 &&
            (it % reinit_freq) == 0) {
            /* the multiphysics and both intermediate models also relax the pressures (relaxTotalPressure) */
            g_reinit_mph = id == VO_EULER_MULTIPHYSICS || id == VO_MHD_INTERMEDIATE || id == VO_HPR_INTERMEDIATE;
            g_reinit_r1 = id == VO_HPR_REDUCED ? 17 : id == VO_HPR_INTERMEDIATE ? 16 : 4;
            g_reinit_r2 = id == VO_HPR_REDUCED ? 18 : id == VO_HPR_INTERMEDIATE ? 18 : g_reinit_mph ? 6 : 5;
            g_reinit_p1 = id == VO_HPR_INTERMEDIATE ? 17 : 5;
            g_reinit_p2 = id == VO_HPR_INTERMEDIATE ? 19 : 7;
            red_reinit(planes, nx, dims == 1 ? 1 : ny);
        }
        if (id == VO_HPR_MULTIPHYSICS && reinit_freq != 0 && (it % reinit_freq) == 0) hmph_reinit(planes, nx);
    }
    if (steps_out) *steps_out = it;
    return t;
}

/* One sweep of FirstOrderSolver::computeFORCETimeStep / compute{X,Y}FORCETimeStep2D (Solvers/firstordersolver.cpp:
 * 232-247, :286-308, :357-379): FORCE fluxes of the cells themselves over the 1-ghost boundary (the ghosts -1 and
 * n are the 2-ghost mirror's), then computeFORCEUpdate (:428-433). */
static void sweep1_grid(const model* m, double* planes, int nx, int ny, int axis, double dx, double dt,
                        const double* prm, int bc) {
    long plane = (long)nx * ny;
    int nv = m->nv;
    int len = axis == 0 ? nx : ny, nlines = axis == 0 ? ny : nx;
    double r = dt / dx;
    double* out = (double*)malloc(sizeof(double) * nv * plane);
#pragma omp parallel for schedule(static)
    for (int line = 0; line < nlines; line++) {
        double* fl = (double*)malloc(sizeof(double) * (len + 1) * MAXV);
        for (int f = 0; f <= len; f++) {
            double wa[MAXV], wb[MAXV];
            int ka = ghost_index(f - 1, len, bc), kb = ghost_index(f, len, bc);
            load_cell(planes, plane, axis == 0 ? (long)line * nx + ka : (long)ka * nx + line, nv, wa);
            load_cell(planes, plane, axis == 0 ? (long)line * nx + kb : (long)kb * nx + line, nv, wb);
            force_flux(m, wa, wb, axis, dx, dt, prm, fl + (long)f * MAXV);
        }
        for (int c = 0; c < len; c++) {
            long idx = axis == 0 ? (long)line * nx + c : (long)c * nx + line;
            double W[MAXV], U[MAXV], Un[MAXV];
            load_cell(planes, plane, idx, nv, W);
            m->cons(W, prm, U);
            for (int v = 0; v < nv; v++)
                Un[v] = U[v] + (r * (fl[(long)c * MAXV + v] + (-1.0 * fl[(long)(c + 1) * MAXV + v])));
            m->setcons(Un, prm, W);
            for (int v = 0; v < nv; v++) out[v * plane + idx] = W[v];
        }
        free(fl);
    }
    memcpy(planes, out, sizeof(double) * nv * plane);
    free(out);
}

/* FirstOrderSolver::solve{,2D} (Solvers/firstordersolver.cpp:435-553) and the MHD / HPR twins
 * (Solvers/mhdfirstordersolver.cpp:457-478, Solvers/hprfirstordersolver.cpp:547-574): the parameters stay as
 * given (the MHD c_h = prm[2] is not reset), no source sub-cycles. */
double vo_run_first_order(int id, double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                          const double* prm, int bc, int* steps_out) {
    const model* m = model_of(id);
    if (!m) return -1.0;
    hred_drop_cold_heat_flux(id, planes, (long)nx * ny, prm);
    hmph_drop_cold_heat_flux(id, planes, (long)nx * ny, prm);
    int dims = ny > 1 ? 2 : 1;
    double tEnd = t_end > 0.0 ? t_end : 1.0e300;
    int limit = max_steps > 0 ? max_steps : 0x7fffffff;
    long plane = (long)nx * ny;
    double t = 0.0;
    int it = 0;
    while (t < tEnd && it < limit) {
        double smax_ = max_wave(m, planes, plane, dims, prm);
        double dt = stable_dt(cfl * (dx / smax_), t, tEnd, it);
        if (dims == 1) {
            sweep1_grid(m, planes, nx, 1, 0, dx, dt, prm, bc);
        } else {
            sweep1_grid(m, planes, nx, ny, 0, dx, 0.5 * dt, prm, bc);
            sweep1_grid(m, planes, nx, ny, 1, dx, dt, prm, bc);
            sweep1_grid(m, planes, nx, ny, 0, dx, 0.5 * dt, prm, bc);
        }
        t += dt;
        it += 1;
    }
    if (steps_out) *steps_out = it;
    return t;
}

double vo_run1d(int id, double* planes, int n, double dx, double cfl, double t_end, int max_steps, double w,
                int lim, const double* prm, int bc, int subcycles, int* steps_out, double* dt_log) {
    return run(id, planes, n, 1, 1, dx, cfl, t_end, max_steps, w, lim, prm, bc, subcycles, steps_out, dt_log, 0);
}

double vo_run2d(int id, double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                double w, int lim, const double* prm, int bc, int subcycles, int* steps_out, double* dt_log) {
    return run(id, planes, nx, ny, 2, dx, cfl, t_end, max_steps, w, lim, prm, bc, subcycles, steps_out, dt_log, 0);
}

double vo_run_two_material(int id, double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                           double w, int lim, const double* prm, int bc, int reinit_freq, int* steps_out) {
    if (id != VO_EULER_REDUCED && id != VO_EULER_MULTIPHYSICS) return -1.0;
    return run(id, planes, nx, ny, ny > 1 ? 2 : 1, dx, cfl, t_end, max_steps, w, lim, prm, bc, 0,
               steps_out, NULL, reinit_freq);
}

double vo_run_mhd_two_material(int id, double* planes, int nx, int ny, double dx, double cfl, double t_end,
                                int max_steps, double w, int lim, const double* prm, int bc, int subcycles,
                                int reinit_freq, int* steps_out) {
    if (id != VO_MHD_REDUCED && id != VO_MHD_INTERMEDIATE && id != VO_HPR_REDUCED && id != VO_HPR_INTERMEDIATE &&
        id != VO_HPR_MULTIPHYSICS && id != VO_MHD_MULTIPHYSICS)
        return -1.0;
    if ((id == VO_HPR_MULTIPHYSICS || id == VO_MHD_MULTIPHYSICS) && ny > 1) return -1.0;  /* 1D only, as the reference */
    hred_drop_cold_heat_flux(id, planes, (long)nx * ny, prm);
    hmph_drop_cold_heat_flux(id, planes, (long)nx * ny, prm);
    double t = run(id, planes, nx, ny, ny > 1 ? 2 : 1, dx, cfl, t_end, max_steps, w, lim, prm, bc, subcycles,
                   steps_out, NULL, reinit_freq);
    /* a cold material's J is state (the reinitialisation mixes it in) that computePrimitiveVariableVector does not
     * return: the returned planes hold 0 there */
    hmph_drop_cold_heat_flux(id, planes, (long)nx * ny, prm);
    return t;
}

/* ------------------------------------------------------------------------- unit-test building blocks */

void vo_prim_to_cons(int id, const double* w, const double* prm, double* u) {
    const model* m = model_of(id);
    if (m) m->cons(w, prm, u);
}

void vo_cons_to_prim(int id, const double* u, const double* prm, double* w) {
    const model* m = model_of(id);
    if (!m) return;
    m->default_state(prm, w);
    m->setcons(u, prm, w);
}

void vo_flux(int id, const double* u, int axis, const double* prm, double* f) {
    const model* m = model_of(id);
    if (m) m->flux(u, axis, prm, f);
}

void vo_slic_flux(int id, const double* wLL, const double* wL, const double* wR, const double* wRR, int axis,
                  double dx, double dt, double w, int lim, const double* prm, double* f) {
    const model* m = model_of(id);
    if (m) slic_flux(m, wLL, wL, wR, wRR, axis, dx, dt, w, lim, prm, f);
}
