// Vector-Jacobian products of the HPR relaxation source and of the conserved/primitive conversions, for the
// gas instantiation (StiffenedGas equation of state, elastic strain relaxation): the reverse pass of the
// homogeneous source batch (source_batch.cu).  No counterpart in the reference, which has no derivatives.
//
// Notation (HPR/hprstatevector.cpp:78-162): primitives W = [rho, p, A (9, row-major), u (3), J (3)], conserved
// U = [rho, rho E, A, rho u, rho J].  With the StiffenedGas branch of HPRMieGruneisen (HPR/hprmiegruneisen.cpp:
// 7-102: Gamma = gamma - 1, p_ref = -p_inf, e_ref = p_inf / rho) the pieces differentiated are
//   rho E = (p + gamma p_inf) / (gamma - 1) + rho m(A) + rho |u|^2 / 2 + alpha^2 rho |J|^2 / 2,
//   m(A)  = c_s^2 |dev(A^T A)|^2 / 4                  (HPR/hprequationofstate.cpp: the mesoscale distortion energy)
//   d(A)  = dm/dA = c_s^2 A dev(A^T A)                (HPR/hprderivatives.cpp:17-25)
//   T     = T_ref + (p + p_inf) / (rho (gamma - 1) c_v)
//   S_A   = -theta1^-1 d(A),  theta1^-1 = 3 det(A)^(5/3) / (c_s^2 tau1)          (HPR/hprsourceterms.cpp:7-27)
//   S_rhoJ = -rho theta2^-1 alpha^2 J = -(rho0 / (tau2 T0)) T (rho J) / rho     (HPR/hprsourceterms.cpp:29-39)
// (the thermal terms only for a thermal material).  The derivatives are those of these exact expressions; the
// forward's floating-point evaluation order does not enter them.  The source is smooth wherever det A > 0,
// rho > 0 and T > 0, so no subgradient choice arises.
#pragma once

#include "physics_hpr.cuh"

namespace vg {
namespace srcadj {

using H = HPRModel<false>;
using M3 = H::M3;

__device__ __forceinline__ M3 transpose(const M3& a) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.m[i][j] = a.m[j][i];
    return r;
}

// cofactor matrix: d det(A) / dA
__device__ __forceinline__ M3 cofactor(const M3& a) {
    M3 c;
    c.m[0][0] = a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1];
    c.m[0][1] = a.m[1][2] * a.m[2][0] - a.m[1][0] * a.m[2][2];
    c.m[0][2] = a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0];
    c.m[1][0] = a.m[0][2] * a.m[2][1] - a.m[0][1] * a.m[2][2];
    c.m[1][1] = a.m[0][0] * a.m[2][2] - a.m[0][2] * a.m[2][0];
    c.m[1][2] = a.m[0][1] * a.m[2][0] - a.m[0][0] * a.m[2][1];
    c.m[2][0] = a.m[0][1] * a.m[1][2] - a.m[0][2] * a.m[1][1];
    c.m[2][1] = a.m[0][2] * a.m[1][0] - a.m[0][0] * a.m[1][2];
    c.m[2][2] = a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0];
    return c;
}

// D = dev(A^T A) and d = c_s^2 A D
__device__ __forceinline__ void distortion(const M3& A, const H::P& q, M3& D, M3& d, double& meso) {
    D = H::dev(H::tmul(A, A));
    const M3 AD = H::mul(A, D);
    const double cs2 = q.cs * q.cs;
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            d.m[i][j] = cs2 * AD.m[i][j];
            sum += D.m[i][j] * D.m[i][j];
        }
    meso = 0.25 * cs2 * sum;
}

// gA += (d m / dA)-adjoint of a cotangent gd of d = c_s^2 A D(A): c_s^2 gd D + A (gG + gG^T), gG = dev(c_s^2 A^T gd)
__device__ __forceinline__ void d_vjp(const M3& A, const M3& D, const M3& gd, const H::P& q, M3& gA) {
    const double cs2 = q.cs * q.cs;
    M3 gD;
#pragma unroll
    for (int l = 0; l < 3; l++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < 3; i++) s += A.m[i][l] * gd.m[i][j];
            gD.m[l][j] = cs2 * s;
        }
    const double tr = (gD.m[0][0] + gD.m[1][1] + gD.m[2][2]) / 3.0;
#pragma unroll
    for (int i = 0; i < 3; i++) gD.m[i][i] -= tr;  // gG = dev(gD)
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            double s = 0.0, t = 0.0;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                s += gd.m[a][j] * D.m[b][j];
                t += A.m[a][j] * (gD.m[b][j] + gD.m[j][b]);
            }
            gA.m[a][b] += cs2 * s + t;
        }
}

// gU += (dS/dU)^T mu; gt1, gt2 += dS/dtau . mu, at the conserved state U.
__device__ __forceinline__ void source_vjp(const double* U, const H::P& q, const double* mu, double* gU, double& gt1,
                                           double& gt2) {
    const double rho = U[0];
    const M3 A = H::load(U + 2);
    M3 D, d;
    double meso;
    distortion(A, q, D, d, meso);
    const double det = H::det(A);
    const double th1 = 3.0 * (pow(det, 5.0 / 3.0) / ((q.cs * q.cs) * q.tau1));
    // S_A = -th1 d
    double g_th1 = 0.0;
    M3 gd, gA;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double m = mu[2 + 3 * i + j];
            g_th1 -= m * d.m[i][j];
            gd.m[i][j] = -th1 * m;
            gA.m[i][j] = 0.0;
        }
    d_vjp(A, D, gd, q, gA);
    const M3 cof = cofactor(A);
    const double dth = g_th1 * ((5.0 / 3.0) * (th1 / det));
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) gA.m[i][j] += dth * cof.m[i][j];
    gt1 += g_th1 * (-th1 / q.tau1);
    if (q.thermal) {
        // S_J = -kappa T UJ / rho,  T = T_ref + (e - p_inf / rho) / c_v,
        // e = U1 / rho - |m|^2 / (2 rho^2) - meso - alpha^2 |UJ|^2 / (2 rho^2)
        const double a2 = q.alpha * q.alpha, r2 = rho * rho, r3 = r2 * rho;
        const double m2 = U[11] * U[11] + U[12] * U[12] + U[13] * U[13];
        const double j2 = U[14] * U[14] + U[15] * U[15] + U[16] * U[16];
        const double e = U[1] / rho - 0.5 * m2 / r2 - meso - 0.5 * a2 * j2 / r2;
        const double T = q.Tref + (e - q.pinf / rho) / q.cv;
        const double kappa = q.rho0 / (q.tau2 * q.T0);
        double mJ = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) mJ += mu[14 + k] * U[14 + k];
        const double gT = -kappa * mJ / rho;
#pragma unroll
        for (int k = 0; k < 3; k++) gU[14 + k] += -kappa * (T / rho) * mu[14 + k];
        gU[0] += kappa * T * mJ / r2;
        gt2 += kappa * T * mJ / (q.tau2 * rho);
        const double ge = gT / q.cv;
        gU[0] += gT * (q.pinf / r2) / q.cv;
        gU[1] += ge / rho;
        gU[0] += ge * (-U[1] / r2 + m2 / r3 + a2 * j2 / r3);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            gU[11 + k] += ge * (-U[11 + k] / r2);
            gU[14 + k] += ge * (-a2 * U[14 + k] / r2);
        }
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) gA.m[i][j] -= ge * d.m[i][j];
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) gU[2 + 3 * i + j] += gA.m[i][j];
}

// gW = (dU/dW)^T gU at the primitive state W (HPRStateVector::computeConservedVariableVector).
__device__ __forceinline__ void cons_vjp(const double* W, const H::P& q, const double* gU, double* gW) {
    const double rho = W[0];
    const M3 A = H::load(W + 2);
    M3 D, d;
    double meso;
    distortion(A, q, D, d, meso);
    const double a2 = q.alpha * q.alpha;
    const double u2 = W[11] * W[11] + W[12] * W[12] + W[13] * W[13];
    const double j2 = q.thermal ? W[14] * W[14] + W[15] * W[15] + W[16] * W[16] : 0.0;
    double gr = gU[0] + gU[1] * (meso + 0.5 * u2 + 0.5 * a2 * j2);
    for (int k = 0; k < 3; k++) gr += gU[11 + k] * W[11 + k];
    if (q.thermal)
        for (int k = 0; k < 3; k++) gr += gU[14 + k] * W[14 + k];
    gW[0] = gr;
    gW[1] = gU[1] / (q.g - 1.0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) gW[2 + 3 * i + j] = gU[2 + 3 * i + j] + gU[1] * rho * d.m[i][j];
    for (int k = 0; k < 3; k++) {
        gW[11 + k] = gU[1] * rho * W[11 + k] + gU[11 + k] * rho;
        gW[14 + k] = q.thermal ? gU[1] * rho * a2 * W[14 + k] + gU[14 + k] * rho : 0.0;
    }
}

// gU = (dW/dU)^T gW at the conserved state U (HPRStateVector::setConservedVariableVector); for a non-thermal
// material J is not a function of U (the cell keeps its own) and gW's J part is not used here.
__device__ __forceinline__ void setcons_vjp(const double* U, const H::P& q, const double* gW, double* gU) {
    const double rho = U[0], r2 = rho * rho;
    const M3 A = H::load(U + 2);
    M3 D, d;
    double meso;
    distortion(A, q, D, d, meso);
    const double a2 = q.alpha * q.alpha, gm1 = q.g - 1.0;
    const double m2 = U[11] * U[11] + U[12] * U[12] + U[13] * U[13];
    const double j2 = q.thermal ? U[14] * U[14] + U[15] * U[15] + U[16] * U[16] : 0.0;
    const double gp = gW[1];
    double g0 = gW[0] + gp * gm1 * (0.5 * m2 / r2 - meso + 0.5 * a2 * j2 / r2);
    for (int k = 0; k < 3; k++) g0 -= gW[11 + k] * U[11 + k] / r2;
    if (q.thermal)
        for (int k = 0; k < 3; k++) g0 -= gW[14 + k] * U[14 + k] / r2;
    gU[0] = g0;
    gU[1] = gp * gm1;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) gU[2 + 3 * i + j] = gW[2 + 3 * i + j] - gp * gm1 * rho * d.m[i][j];
    for (int k = 0; k < 3; k++) {
        gU[11 + k] = gW[11 + k] / rho - gp * gm1 * U[11 + k] / rho;
        gU[14 + k] = q.thermal ? gW[14 + k] / rho - gp * gm1 * a2 * U[14 + k] / rho : 0.0;
    }
}

}  // namespace srcadj
}  // namespace vg
