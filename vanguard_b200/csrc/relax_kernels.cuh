// Stiff relaxation of the HPR source (no counterpart in the reference, whose only source integrator is the explicit
// RK4 forcing solver, stable for sub-steps up to ~2.8 tau).  It replaces the 2 x subcycles forcing passes of a step by
// one relaxation of dt/2 before and one after the sweeps, cell by cell, at any tau:
//   * distortion: S_A = -c A dev(A^T A), c = 3 det(A)^(5/3) / tau1 (HPR/hprsourceterms.cpp:7-39 with
//     dE/dA = c_s^2 A dev(A^T A)).  det A is conserved (dev is traceless), so c is constant; G = A^T A keeps its
//     eigenvectors and its eigenvalues obey d(ln l_i)/dt = -2 c (l_i - mean(l)).  That system is integrated by
//     implicit Euler (L-stable, Newton on three unknowns), then A <- A V diag(sqrt(l_i' / l_i)) V^T;
//   * heat flux: d(rho J)/dt = -(rho0 T / (tau2 T0 rho)) rho J with rho, v, E and the relaxed A fixed.  Every
//     equation of state here has T = T_ref + (e - e_ref(rho)) / c_v, and e = e_J0 - alpha^2 |J|^2 / 2, so
//     T = T_J0 - beta s with s = |J|^2, beta = alpha^2 / (2 c_v): s obeys the Bernoulli equation
//     ds/dt = -2 kappa (T_J0 - beta s) s (kappa = rho0 / (tau2 T0 rho)), whose exact solution over h scales J by
//     sqrt(E / ((1 - r) + r E)), E = exp(-2 kappa T_J0 h), r = beta s0 / T_J0.  J is left alone where T <= 0.
// rho, rho v and rho E do not change.  The eigen-decomposition is the published cyclic Jacobi method.
#pragma once

#include "physics_hpr.cuh"
#include "slic_kernels.cuh"
#include "vg_common.cuh"

namespace vg {

__device__ inline void sym_eig3(const double g[3][3], double l[3], double V[3][3]) {
    double a[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            a[i][j] = g[i][j];
            V[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 16; sweep++) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-32 * dia) break;
        for (int pq = 0; pq < 3; pq++) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            if (a[p][q] == 0.0) continue;
            const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
            const double apq = a[p][q];
            a[p][p] -= t * apq;
            a[q][q] += t * apq;
            a[p][q] = a[q][p] = 0.0;
            for (int r = 0; r < 3; r++) {
                if (r != p && r != q) {
                    const double arp = a[r][p], arq = a[r][q];
                    a[r][p] = a[p][r] = c * arp - s * arq;
                    a[r][q] = a[q][r] = s * arp + c * arq;
                }
                const double vrp = V[r][p], vrq = V[r][q];
                V[r][p] = c * vrp - s * vrq;
                V[r][q] = s * vrp + c * vrq;
            }
        }
    }
    for (int i = 0; i < 3; i++) l[i] = a[i][i];
}

// n implicit-Euler steps of d(mu_i)/dt = -2 c (exp(mu_i) - mean(exp(mu))), k = 2 c h / n per step.  Newton starts
// from the linear extrapolation of the last two step values and stops once a correction below 1e-8 has been
// applied: Newton converges quadratically here (the Jacobian is I plus a positive diagonal and a rank-one term),
// so the next correction would be of the order of its square, below the double resolution of mu.
__device__ inline void relax_log_eigs(double mu[3], double k, int n) {
    double prev[3] = {mu[0], mu[1], mu[2]};
    for (int s = 0; s < n; s++) {
        const double m0[3] = {mu[0], mu[1], mu[2]};
        double x[3];
        for (int i = 0; i < 3; i++) x[i] = m0[i] + (m0[i] - prev[i]);
        for (int i = 0; i < 3; i++) prev[i] = m0[i];
        for (int it = 0; it < 100; it++) {
            const double e[3] = {exp(x[0]), exp(x[1]), exp(x[2])};
            const double mean = (e[0] + e[1] + e[2]) / 3.0;
            // J dx = -F with J = diag(1 + k e_i) - (k / 3) 1 e^T, by the Sherman-Morrison formula:
            // dx = y + k z (e . y) / sum(z), z_i = 1 / (1 + k e_i), y_i = -F_i z_i
            // (1 - (k / 3) e . z = sum(z) / 3 exactly, so the denominator takes no cancellation)
            double z[3], y[3];
            for (int i = 0; i < 3; i++) {
                const double F = (x[i] - m0[i]) + k * (e[i] - mean);
                z[i] = 1.0 / (1.0 + k * e[i]);
                y[i] = -F * z[i];
            }
            const double g = k * (((e[0] * y[0]) + (e[1] * y[1]) + (e[2] * y[2])) / ((z[0] + z[1]) + z[2]));
            double dx[3], big = 0.0;
            for (int c = 0; c < 3; c++) {
                dx[c] = y[c] + z[c] * g;
                big = fmax(big, fabs(dx[c]));
            }
            const double damp = big > 0.5 ? 0.5 / big : 1.0;
            for (int i = 0; i < 3; i++) x[i] += damp * dx[i];
            if (big < 1e-8) break;
        }
        for (int i = 0; i < 3; i++) mu[i] = x[i];
    }
}

__device__ inline int clamp_steps(double v, int lo, int hi) {
    if (!(v > lo)) return lo;
    if (v > hi) return hi;
    return (int)ceil(v);
}

// Relax the conserved vector U of one cell over a time h (see the file comment).
template <class M>
__device__ inline void hpr_relax_cell(double* U, double h, const typename M::P& q) {
    const double rho = U[0];
    const typename M::M3 A = M::load(U + 2);
    const double d = M::det(A);
    if (!(d > 0.0) || !(h > 0.0)) return;
    const typename M::M3 G = M::tmul(A, A);
    double l[3], V[3][3], mu[3];
    sym_eig3(G.m, l, V);
    if (!(l[0] > 0.0 && l[1] > 0.0 && l[2] > 0.0)) return;
    const double c = 3.0 * (pow(d, 5.0 / 3.0) / q.tau1);
    const double lmax = fmax(l[0], fmax(l[1], l[2]));
    const int nA = clamp_steps((2.0 * c * lmax * h) / 0.25, 1, 256);
    for (int i = 0; i < 3; i++) mu[i] = log(l[i]);
    relax_log_eigs(mu, 2.0 * c * (h / nA), nA);
    double f[3], Mr[3][3];
    for (int i = 0; i < 3; i++) f[i] = exp(0.5 * (mu[i] - log(l[i])));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double sum = 0.0;
            for (int k = 0; k < 3; k++) sum += V[i][k] * f[k] * V[j][k];
            Mr[i][j] = sum;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double sum = 0.0;
            for (int k = 0; k < 3; k++) sum += A.m[i][k] * Mr[k][j];
            U[2 + 3 * i + j] = sum;
        }
    if (!q.thermal) return;
    const typename M::M3 An = M::load(U + 2);
    const double E = U[1] / rho, u = U[11] / rho, v = U[12] / rho, w = U[13] / rho;
    const double jx = U[14] / rho, jy = U[15] / rho, jz = U[16] / rho;
    const double s0 = ((jx * jx) + (jy * jy)) + (jz * jz);
    const double T = M::mg_temperature(rho, M::pressure_of(rho, E, u, v, w, An, jx, jy, jz, q), q);
    if (!(s0 > 0.0) || !(T > 0.0)) return;
    const double beta = (0.5 * (q.alpha * q.alpha)) / q.cv;
    const double TJ0 = T + (beta * s0);  // the temperature at J = 0
    const double kappa = q.rho0 / (q.tau2 * q.T0 * rho);
    const double Eh = exp(-2.0 * (kappa * (TJ0 * h)));
    const double r = (beta * s0) / TJ0;
    const double fac = sqrt(Eh / ((1.0 - r) + (r * Eh)));
    for (int i = 14; i < 17; i++) U[i] *= fac;
}

// One relaxation of length h = dt * a.dt_scale of every cell, in place on a.out (a.in == a.out allowed).
template <class M>
__global__ void __launch_bounds__(128, 4) relax_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW;
    const long n = (long)a.nx * a.ny;
    const long idx = blockIdx.x * 128L + threadIdx.x;
    if (idx >= n || (a.ctrl && !a.ctrl->active)) return;
    const int i = (int)(idx / a.nx), j = (int)(idx - (long)i * a.nx);
    const long self = (long)i * a.pitch + j;
    const typename M::P q = M::params(a.params, 0.0);
    const double h = (a.ctrl ? a.ctrl->dt : a.dt_host) * a.dt_scale;
    double W[NW], U[NU];
    for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + self];
    M::cons(W, q, U);
    hpr_relax_cell<M>(U, h, q);
    M::setcons(U, q, W);  // the cell keeps its own J when the material is not thermal
    for (int v = 0; v < NW; v++) a.out[v * a.plane + self] = W[v];
    if (bad_state<M>(W, q)) atomicOr(a.err, ERR_STATE);
}

}  // namespace vg
