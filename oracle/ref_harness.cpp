// Test-infrastructure harness around the reference's own, unmodified SLIC code.
//
// Compiled by oracle/Makefile together with the reference sources into oracle/_ref/libvgref.so.
// It exposes extern "C" entry points over structure-of-arrays PRIMITIVE planes (the reference stores
// primitives in its cells), so Python tests and the CPU baseline in bench.py can drive the reference
// with plain pointers.  Only tests/, bench.py's CPU legs and __graft_entry__.smoke() may load it.
//
// What it calls (paths relative to the reference tree):
//   * SecondOrderSolver::solve / solve2D              Solvers/secondordersolver.cpp:288,392
//   * the per-step functions that solve() is built from, to run a fixed number of steps:
//       Solvers::insertBoundaryCells{,2D}             Solvers/solvers.cpp:7,88
//       Solvers::computeStableTimeStep{,2D}           Solvers/solvers.cpp:388,413
//       SecondOrderSolver::computeSLICTimeStep        Solvers/secondordersolver.cpp:80
//       SecondOrderSolver::compute{X,Y}SLICTimeStep2D Solvers/secondordersolver.cpp:140,214
//   * the MHD equivalents (Solvers/mhdsecondordersolver.cpp:318,501 and Solvers/mhdsolvers.cpp), with
//     c_h set from the padded-grid maximum wave speed each step as solve() does (:330-332, :513-515).
//   * the HPR equivalents (Solvers/hprsecondordersolver.cpp, Solvers/hprsolvers.cpp,
//     Solvers/hprforcingsolver.cpp).
//   * the first-order FORCE solvers' loops (FirstOrderSolver::solve{,2D}, Solvers/firstordersolver.cpp:435,521;
//     MHDFirstOrderSolver, HPRFirstOrderSolver) from their per-step functions compute{,X,Y}FORCETimeStep{,2D}.
//
// The reference has no periodic boundary.  For periodic runs this harness builds the ghosted arrays
// itself (2 ghost cells, wrap-around) and leaves the 2D corner blocks default-constructed, exactly as
// insertBoundaryCells2D leaves them (Solvers/solvers.cpp:92), so the CFL maximum sees the same cells.
//
// Parity runs call vgref_set_threads(1): the reference's CFL maximum is an unsynchronised OpenMP
// update (Solvers/solvers.cpp:264-273) and is only reproducible on one thread.

#include "Solvers/firstordersolver.h"
#include "Solvers/hprfirstordersolver.h"
#include "Solvers/mhdfirstordersolver.h"
#include "Solvers/secondordersolver.h"
#include "Solvers/mhdsecondordersolver.h"
#include "Solvers/mhdforcingsolver.h"
#include "Solvers/hprsecondordersolver.h"
#include "Solvers/hprforcingsolver.h"
#include "Euler/eulertests.h"
#include "MHD/mhdtests.h"
#include "HPR/hprtests.h"
#include "Solvers/multiphysicssolvers.h"

#include <omp.h>
#include <iostream>
#include <limits>
#include <type_traits>
#include <vector>

using std::vector;

namespace {

// Per-step status lines go to cout in the reference (Solvers/solvers.cpp:611-614); drop them.
struct QuietCout {
    std::streambuf* saved;
    QuietCout() : saved(std::cout.rdbuf(nullptr)) {}
    ~QuietCout() { std::cout.clear(); std::cout.rdbuf(saved); }
};

const double kNoEnd = 1.0e300;

// ---------------------------------------------------------------------------------------------- Euler
// Plane order = EulerStateVector primitive order (Euler/eulerstatevector.cpp:47-55): rho,u,v,w,p,lambda.
EulerMaterialParameters eulerParams(const double* prm) {
    // prm = {gamma, p_inf, c_v, E0, T_ign, rate}  (Euler/eulermaterialparameters.cpp:36-46)
    return EulerMaterialParameters(prm[0], prm[1], prm[2], prm[3], prm[4], prm[5]);
}

EulerStateVector eulerCell(const double* planes, long plane, long k) {
    return EulerStateVector(planes[k], planes[plane + k], planes[2 * plane + k], planes[3 * plane + k],
                            planes[4 * plane + k], planes[5 * plane + k]);
}

void eulerStore(EulerStateVector& c, double* planes, long plane, long k) {
    vector<double> w = c.computePrimitiveVariableVector();
    for (int v = 0; v < 6; v++) planes[v * plane + k] = w[v];
}

vector<vector<EulerStateVector> > eulerGrid(const double* planes, int nx, int ny) {
    long plane = (long)nx * ny;
    vector<vector<EulerStateVector> > g(ny, vector<EulerStateVector>(nx));
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) g[i][j] = eulerCell(planes, plane, (long)i * nx + j);
    return g;
}

void eulerUngrid(vector<vector<EulerStateVector> >& g, double* planes, int nx, int ny) {
    long plane = (long)nx * ny;
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) eulerStore(g[i][j], planes, plane, (long)i * nx + j);
}

// Ghosted copy with 2 wrap-around ghosts per side; corners stay default-constructed.
template <class S>
vector<vector<S> > periodicGhosts2D(vector<vector<S> >& c, int b) {
    int ny = c.size(), nx = c[0].size();
    vector<vector<S> > g(ny + 2 * b, vector<S>(nx + 2 * b));
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) g[i + b][j + b] = c[i][j];
    for (int i = 0; i < ny; i++)
        for (int k = 0; k < b; k++) {
            g[i + b][k] = c[i][nx - b + k];
            g[i + b][nx + b + k] = c[i][k];
        }
    for (int j = 0; j < nx; j++)
        for (int k = 0; k < b; k++) {
            g[k][j + b] = c[ny - b + k][j];
            g[ny + b + k][j + b] = c[k][j];
        }
    return g;
}

// The reference's transmissive ghosts (insertBoundaryCells2D: g[-1-k] = c[k], g[n+k] = c[n-1-k], corner blocks
// default-constructed), built here for the MHD intermediate model, whose own insertBoundaryCells2D fills the outermost
// bottom row from the padded grid instead of the cells (Solvers/mhdsolvers.cpp:213).
template <class S>
vector<vector<S> > mirrorGhosts2D(vector<vector<S> >& c, int b) {
    int ny = c.size(), nx = c[0].size();
    vector<vector<S> > g(ny + 2 * b, vector<S>(nx + 2 * b));
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) g[i + b][j + b] = c[i][j];
    for (int i = 0; i < ny; i++)
        for (int k = 0; k < b; k++) {
            g[i + b][b - 1 - k] = c[i][k];
            g[i + b][nx + b + k] = c[i][nx - 1 - k];
        }
    for (int j = 0; j < nx; j++)
        for (int k = 0; k < b; k++) {
            g[b - 1 - k][j + b] = c[k][j];
            g[ny + b + k][j + b] = c[ny - 1 - k][j];
        }
    return g;
}

template <class S>
vector<S> periodicGhosts1D(vector<S>& c, int b) {
    int n = c.size();
    vector<S> g(n + 2 * b);
    for (int i = 0; i < n; i++) g[i + b] = c[i];
    for (int k = 0; k < b; k++) {
        g[k] = c[n - b + k];
        g[n + b + k] = c[k];
    }
    return g;
}

// ------------------------------------------------------------------------------------------------ MHD
// Plane order = MHDStateVector primitive order (MHD/mhdstatevector.cpp:35-47):
// rho,u,v,w,p,Bx,By,Bz,psi.
MHDStateVector mhdCell(const double* planes, long plane, long k) {
    return MHDStateVector(planes[k], planes[plane + k], planes[2 * plane + k], planes[3 * plane + k],
                          planes[4 * plane + k], planes[5 * plane + k], planes[6 * plane + k],
                          planes[7 * plane + k], planes[8 * plane + k]);
}

void mhdStore(MHDStateVector& c, double* planes, long plane, long k) {
    vector<double> w = c.computePrimitiveVariableVector();
    for (int v = 0; v < 9; v++) planes[v * plane + k] = w[v];
}

MHDMaterialParameters mhdParams(const double* prm) {
    MHDMaterialParameters mp(prm[0]);
    mp.setStiffeningParameter(prm[1]);
    return mp;
}

// ------------------------------------------------------------------------------------------------ HPR
// Plane order = HPRStateVector primitive order (HPR/hprstatevector.cpp:50-73):
// rho, p, A(9, row-major), u, v, w, Jx, Jy, Jz.
// prm = {gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, is_thermal, eos, Gamma0, c0, s,
// alpha_eos, is_plastic, sigma0, n} (HPR/hprmaterialparameters.cpp:34-69 argument order); eos 0 StiffenedGas,
// 1 ShockMieGruneisen, 2 GodunovRomenski.
HPRMaterialParameters hprParams(const double* prm) {
    static const char* eos[3] = {"StiffenedGas", "ShockMieGruneisen", "GodunovRomenski"};
    int id = (int)prm[12];
    return HPRMaterialParameters(eos[id >= 0 && id < 3 ? id : 0], prm[11] != 0.0, prm[17] != 0.0, 8.31445985, prm[3],
                                 prm[10], prm[9], prm[4], prm[2], prm[0], prm[1], prm[14], prm[13], prm[15], 0.0, prm[5],
                                 prm[7], prm[8], 1.0e-2, 0.75, prm[18], prm[19], prm[6], prm[16], 0.0, 0.0);
}

HPRStateVector hprCell(const double* planes, long plane, long k) {
    vector<vector<double> > A(3, vector<double>(3));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) A[i][j] = planes[(2 + 3 * i + j) * plane + k];
    return HPRStateVector(planes[k], planes[plane + k], A, planes[11 * plane + k], planes[12 * plane + k],
                          planes[13 * plane + k], planes[14 * plane + k], planes[15 * plane + k], planes[16 * plane + k]);
}

void hprStore(HPRStateVector& c, double* planes, long plane, long k) {
    planes[k] = c.getDensity();
    planes[plane + k] = c.getPressure();
    vector<vector<double> > A = c.getDistortionTensor();
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) planes[(2 + 3 * i + j) * plane + k] = A[i][j];
    planes[11 * plane + k] = c.getXVelocity();
    planes[12 * plane + k] = c.getYVelocity();
    planes[13 * plane + k] = c.getZVelocity();
    planes[14 * plane + k] = c.getXThermalImpulse();
    planes[15 * plane + k] = c.getYThermalImpulse();
    planes[16 * plane + k] = c.getZThermalImpulse();
}
}  // namespace

extern "C" {

// Set the OpenMP team size used by the reference loops (n <= 0: all host cores).  Returns the size.
int vgref_set_threads(int n) {
    if (n <= 0) n = omp_get_num_procs();
    omp_set_num_threads(n);
    return n;
}

// --------------------------------------------------------------------------------------- Euler 1D
// Runs SecondOrderSolver::solve's loop on n cells (planes: 6 x n, transmissive).  max_steps <= 0 calls
// the reference's solve() itself (time-driven); otherwise the same per-step calls are made by this
// loop so a fixed step count can be run.  Returns the time reached; *steps_out the steps taken.
double vgref_euler1d_run(double* planes, int n, double dx, double cfl, double t_end, int max_steps,
                         double bias, int limiter, const double* prm, int* steps_out) {
    QuietCout quiet;
    EulerMaterialParameters mp = eulerParams(prm);
    vector<EulerStateVector> cells(n);
    for (int i = 0; i < n; i++) cells[i] = eulerCell(planes, n, i);
    double t = 0.0;
    int it = 0;
    if (max_steps <= 0) {
        cells = SecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, 0, mp);
        t = -1.0;  // solve() does not report its step count or final time
        it = -1;
    } else {
        double tEnd = t_end > 0.0 ? t_end : kNoEnd;
        while (t < tEnd && it < max_steps) {
            vector<EulerStateVector> withB = Solvers::insertBoundaryCells(cells, 2);
            double dt = Solvers::computeStableTimeStep(withB, dx, cfl, t, tEnd, it, mp);
            SecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, mp);
            t += dt;
            it += 1;
        }
    }
    for (int i = 0; i < n; i++) eulerStore(cells[i], planes, n, i);
    if (steps_out) *steps_out = it;
    return t;
}

// Many independent 1D problems, each run by SecondOrderSolver::solve's per-step loop as vgref_euler1d_run runs it
// (`steps` steps, no end time), the problems spread over the OpenMP team with one thread per problem (the
// reference's own loops inside run single-threaded as nested regions).  planes: 6 x total, the problems'
// primitive planes concatenated in order (total = sum of ncell); problem k has ncell[k] cells of width dx[k] and
// adiabatic index gamma[k] (p_inf 0).  This is the reference's way to solve a ragged batch: one solve per problem.
void vgref_euler1d_batch_run(double* planes, int ninst, const int* ncell, const double* dx, const double* gamma,
                             double cfl, int steps, double bias, int limiter) {
    QuietCout quiet;
    std::vector<long> off(ninst + 1, 0);
    for (int k = 0; k < ninst; k++) off[k + 1] = off[k] + ncell[k];
    const long total = off[ninst];
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < ninst; k++) {
        const double prm[6] = {gamma[k], 0.0, 25.0, 0.0, 0.25, 250.0};  // EulerMaterialParameters(gamma)'s defaults
        EulerMaterialParameters mp = eulerParams(prm);
        const int n = ncell[k];
        vector<EulerStateVector> cells(n);
        for (int i = 0; i < n; i++) cells[i] = eulerCell(planes, total, off[k] + i);
        double t = 0.0;
        for (int it = 0; it < steps; it++) {
            vector<EulerStateVector> withB = Solvers::insertBoundaryCells(cells, 2);
            double dt = Solvers::computeStableTimeStep(withB, dx[k], cfl, t, kNoEnd, it, mp);
            SecondOrderSolver::computeSLICTimeStep(cells, withB, dx[k], dt, bias, limiter, mp);
            t += dt;
        }
        for (int i = 0; i < n; i++) eulerStore(cells[i], planes, total, off[k] + i);
    }
}

// --------------------------------------------------------------------------------------- Euler 2D
// nx columns (x, inner index j) by ny rows (y, row index i); planes: 6 x (ny*nx), row-major.
// bc: 0 transmissive (reference ghosts), 1 periodic (harness ghosts).
double vgref_euler2d_run(double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                         double bias, int limiter, const double* prm, int bc, int* steps_out) {
    QuietCout quiet;
    EulerMaterialParameters mp = eulerParams(prm);
    vector<vector<EulerStateVector> > cells = eulerGrid(planes, nx, ny);
    double t = 0.0;
    int it = 0;
    if (max_steps <= 0 && bc == 0) {
        cells = SecondOrderSolver::solve2D(cells, dx, cfl, t_end, bias, limiter, 0, mp);
        t = -1.0;
        it = -1;
    } else {
        double tEnd = t_end > 0.0 ? t_end : kNoEnd;
        int limit = max_steps > 0 ? max_steps : 0x7fffffff;
        auto ghosts = [&](vector<vector<EulerStateVector> >& c) {
            return bc == 1 ? periodicGhosts2D(c, 2) : Solvers::insertBoundaryCells2D(c, 2);
        };
        while (t < tEnd && it < limit) {
            vector<vector<EulerStateVector> > withB = ghosts(cells);
            double dt = Solvers::computeStableTimeStep2D(withB, dx, cfl, t, tEnd, it, mp);
            SecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, bias, limiter, mp);
            withB = ghosts(cells);
            SecondOrderSolver::computeYSLICTimeStep2D(cells, withB, dx, dt, bias, limiter, mp);
            withB = ghosts(cells);
            SecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, bias, limiter, mp);
            t += dt;
            it += 1;
        }
    }
    eulerUngrid(cells, planes, nx, ny);
    if (steps_out) *steps_out = it;
    return t;
}

// One sweep (axis 0 = X, 1 = Y) with time step dt, on the ghosted grid the reference builds.
void vgref_euler2d_sweep(double* planes, int nx, int ny, int axis, double dx, double dt, double bias,
                         int limiter, const double* prm, int bc) {
    EulerMaterialParameters mp = eulerParams(prm);
    vector<vector<EulerStateVector> > cells = eulerGrid(planes, nx, ny);
    vector<vector<EulerStateVector> > withB =
        bc == 1 ? periodicGhosts2D(cells, 2) : Solvers::insertBoundaryCells2D(cells, 2);
    if (axis == 0)
        SecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, dt, bias, limiter, mp);
    else
        SecondOrderSolver::computeYSLICTimeStep2D(cells, withB, dx, dt, bias, limiter, mp);
    eulerUngrid(cells, planes, nx, ny);
}

// computeMaximumWaveSpeed2D over the ghosted grid (corner blocks default-constructed).
double vgref_euler2d_max_wave_speed(const double* planes, int nx, int ny, const double* prm, int bc) {
    EulerMaterialParameters mp = eulerParams(prm);
    vector<vector<EulerStateVector> > cells = eulerGrid(planes, nx, ny);
    vector<vector<EulerStateVector> > withB =
        bc == 1 ? periodicGhosts2D(cells, 2) : Solvers::insertBoundaryCells2D(cells, 2);
    return Solvers::computeMaximumWaveSpeed2D(withB, mp);
}

// ----------------------------------------------------------------------------------------- MHD 1D/2D
// planes: 9 x cells.  prm = {gamma, p_inf}.  subcycles > 0 adds MHDForcingSolver's RK4 GLM damping
// around the sweeps as solve()/solve2D() do (Solvers/mhdsecondordersolver.cpp:334-348, :517-540);
// only with transmissive boundaries.
double vgref_mhd1d_run(double* planes, int n, double dx, double cfl, double t_end, int max_steps,
                       double bias, int limiter, const double* prm, int bc, int subcycles, int* steps_out) {
    QuietCout quiet;
    MHDMaterialParameters mp = mhdParams(prm);
    vector<MHDStateVector> cells(n);
    for (int i = 0; i < n; i++) cells[i] = mhdCell(planes, n, i);
    double t = 0.0;
    int it = 0;
    if (max_steps <= 0 && bc == 0) {
        cells = MHDSecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, subcycles, mp);
        t = -1.0;
        it = -1;
    } else {
        double tEnd = t_end > 0.0 ? t_end : kNoEnd;
        int limit = max_steps > 0 ? max_steps : 0x7fffffff;
        auto ghosts = [&](vector<MHDStateVector>& c, int b) {
            return bc == 1 ? periodicGhosts1D(c, b) : MHDSolvers::insertBoundaryCells(c, b);
        };
        while (t < tEnd && it < limit) {
            vector<MHDStateVector> withB = ghosts(cells, 2);
            double dt = MHDSolvers::computeStableTimeStep(withB, dx, cfl, t, tEnd, it, mp);
            double smax = MHDSolvers::computeMaximumWaveSpeed(withB, mp);
            mp.setHyperbolicWaveSpeed(smax);
            mp.configureParabolicDamping();
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                MHDForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            withB = ghosts(cells, 2);
            MHDSecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, mp);
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                MHDForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            t += dt;
            it += 1;
        }
    }
    for (int i = 0; i < n; i++) mhdStore(cells[i], planes, n, i);
    if (steps_out) *steps_out = it;
    return t;
}

double vgref_mhd2d_run(double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                       double bias, int limiter, const double* prm, int bc, int subcycles, int* steps_out) {
    QuietCout quiet;
    MHDMaterialParameters mp = mhdParams(prm);
    long plane = (long)nx * ny;
    vector<vector<MHDStateVector> > cells(ny, vector<MHDStateVector>(nx));
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) cells[i][j] = mhdCell(planes, plane, (long)i * nx + j);
    double t = 0.0;
    int it = 0;
    if (max_steps <= 0 && bc == 0) {
        cells = MHDSecondOrderSolver::solve2D(cells, dx, cfl, t_end, bias, limiter, subcycles, mp);
        t = -1.0;
        it = -1;
    } else {
        double tEnd = t_end > 0.0 ? t_end : kNoEnd;
        int limit = max_steps > 0 ? max_steps : 0x7fffffff;
        auto ghosts = [&](vector<vector<MHDStateVector> >& c, int b) {
            return bc == 1 ? periodicGhosts2D(c, b) : MHDSolvers::insertBoundaryCells2D(c, b);
        };
        while (t < tEnd && it < limit) {
            vector<vector<MHDStateVector> > withB = ghosts(cells, 2);
            double dt = MHDSolvers::computeStableTimeStep2D(withB, dx, cfl, t, tEnd, it, mp);
            double smax = MHDSolvers::computeMaximumWaveSpeed2D(withB, mp);
            mp.setHyperbolicWaveSpeed(smax);
            mp.configureParabolicDamping();
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                MHDForcingSolver::computeRungeKuttaTimeStep2D(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            withB = ghosts(cells, 2);
            MHDSecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, bias, limiter, mp);
            withB = ghosts(cells, 2);
            MHDSecondOrderSolver::computeYSLICTimeStep2D(cells, withB, dx, dt, bias, limiter, mp);
            withB = ghosts(cells, 2);
            MHDSecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, bias, limiter, mp);
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                MHDForcingSolver::computeRungeKuttaTimeStep2D(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            t += dt;
            it += 1;
        }
    }
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) mhdStore(cells[i][j], planes, plane, (long)i * nx + j);
    if (steps_out) *steps_out = it;
    return t;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------- HPR 1D/2D
// planes: 17 x cells.  subcycles > 0 runs HPRForcingSolver's RK4 relaxation source around the sweeps as
// solve()/solve2D() do (Solvers/hprsecondordersolver.cpp:323-341, :514-541).
extern "C" double vgref_hpr1d_run(double* planes, int n, double dx, double cfl, double t_end, int max_steps,
                                  double bias, int limiter, const double* prm, int bc, int subcycles, int* steps_out) {
    QuietCout quiet;
    HPRMaterialParameters mp = hprParams(prm);
    vector<HPRStateVector> cells(n);
    for (int i = 0; i < n; i++) cells[i] = hprCell(planes, n, i);
    double t = 0.0;
    int it = 0;
    if (max_steps <= 0 && bc == 0) {
        cells = HPRSecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, subcycles, mp);
        t = -1.0;
        it = -1;
    } else {
        double tEnd = t_end > 0.0 ? t_end : kNoEnd;
        int limit = max_steps > 0 ? max_steps : 0x7fffffff;
        auto ghosts = [&](vector<HPRStateVector>& c, int b) {
            return bc == 1 ? periodicGhosts1D(c, b) : HPRSolvers::insertBoundaryCells(c, b);
        };
        while (t < tEnd && it < limit) {
            vector<HPRStateVector> withB = ghosts(cells, 2);
            double dt = HPRSolvers::computeStableTimeStep(withB, dx, cfl, t, tEnd, it, mp);
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                HPRForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            withB = ghosts(cells, 2);
            HPRSecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, mp);
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                HPRForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            t += dt;
            it += 1;
        }
    }
    for (int i = 0; i < n; i++) hprStore(cells[i], planes, n, i);
    if (steps_out) *steps_out = it;
    return t;
}

extern "C" double vgref_hpr2d_run(double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                                  double bias, int limiter, const double* prm, int bc, int subcycles, int* steps_out) {
    QuietCout quiet;
    HPRMaterialParameters mp = hprParams(prm);
    long plane = (long)nx * ny;
    vector<vector<HPRStateVector> > cells(ny, vector<HPRStateVector>(nx));
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) cells[i][j] = hprCell(planes, plane, (long)i * nx + j);
    double t = 0.0;
    int it = 0;
    if (max_steps <= 0 && bc == 0) {
        cells = HPRSecondOrderSolver::solve2D(cells, dx, cfl, t_end, bias, limiter, subcycles, mp);
        t = -1.0;
        it = -1;
    } else {
        double tEnd = t_end > 0.0 ? t_end : kNoEnd;
        int limit = max_steps > 0 ? max_steps : 0x7fffffff;
        auto ghosts = [&](vector<vector<HPRStateVector> >& c, int b) {
            return bc == 1 ? periodicGhosts2D(c, b) : HPRSolvers::insertBoundaryCells2D(c, b);
        };
        while (t < tEnd && it < limit) {
            vector<vector<HPRStateVector> > withB = ghosts(cells, 2);
            double dt = HPRSolvers::computeStableTimeStep2D(withB, dx, cfl, t, tEnd, it, mp);
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                HPRForcingSolver::computeRungeKuttaTimeStep2D(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            withB = ghosts(cells, 2);
            HPRSecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, bias, limiter, mp);
            withB = ghosts(cells, 2);
            HPRSecondOrderSolver::computeYSLICTimeStep2D(cells, withB, dx, dt, bias, limiter, mp);
            withB = ghosts(cells, 2);
            HPRSecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, bias, limiter, mp);
            for (int s = 0; s < subcycles; s++) {
                withB = ghosts(cells, 1);
                HPRForcingSolver::computeRungeKuttaTimeStep2D(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, mp);
            }
            t += dt;
            it += 1;
        }
    }
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) hprStore(cells[i][j], planes, plane, (long)i * nx + j);
    if (steps_out) *steps_out = it;
    return t;
}

// Single-cell probes of the HPR model for unit tests: cons (U[17]), x/y flux of a conserved vector,
// source term of a conserved vector, and the acoustic-tensor wave speed in a direction.
extern "C" void vgref_hpr_cell(const double* w, const double* prm, double* u, double* fx, double* fy, double* src,
                               double* speed_xy) {
    HPRMaterialParameters mp = hprParams(prm);
    HPRStateVector s = hprCell(w, 1, 0);
    vector<double> U = s.computeConservedVariableVector(mp);
    vector<double> Fx = HPRStateVector::computeXFluxVector(U, mp);
    vector<double> Fy = HPRStateVector::computeYFluxVector(U, mp);
    vector<double> S = HPRStateVector::computeSourceTermVector(U, mp);
    for (int i = 0; i < 17; i++) {
        u[i] = U[i];
        fx[i] = Fx[i];
        fy[i] = Fy[i];
        src[i] = S[i];
    }
    speed_xy[0] = HPRAcousticTensor::computeMaximumWaveSpeed(s, mp, 0);
    speed_xy[1] = HPRAcousticTensor::computeMaximumWaveSpeed(s, mp, 1);
}

// ---------------------------------------------------------------------------------------- first order
// FirstOrderSolver / MHDFirstOrderSolver / HPRFirstOrderSolver::solve{,2D} (Solvers/firstordersolver.cpp:435-553,
// Solvers/mhdfirstordersolver.cpp:457-478, Solvers/hprfirstordersolver.cpp:547-574): 1-ghost boundary, stable
// time step, one FORCE step in 1D or X(dt/2) Y(dt) X(dt/2) in 2D.  The material parameters are not touched
// between steps (the MHD c_h stays what the caller gave, prm[2]).
namespace {

template <class S, class P, class Sol, class FO>
double firstOrder1D(vector<S>& cells, double dx, double cfl, double t_end, int max_steps, P mp, int bc, int* steps) {
    QuietCout quiet;
    double t = 0.0, tEnd = t_end > 0.0 ? t_end : kNoEnd;
    int it = 0, limit = max_steps > 0 ? max_steps : 0x7fffffff;
    while (t < tEnd && it < limit) {
        vector<S> withB = bc == 1 ? periodicGhosts1D(cells, 1) : Sol::insertBoundaryCells(cells, 1);
        double dt = Sol::computeStableTimeStep(withB, dx, cfl, t, tEnd, it, mp);
        FO::computeFORCETimeStep(cells, withB, dx, dt, mp);
        t += dt;
        it += 1;
    }
    if (steps) *steps = it;
    return t;
}

template <class S, class P, class Sol, class FO>
double firstOrder2D(vector<vector<S> >& cells, double dx, double cfl, double t_end, int max_steps, P mp, int bc,
                    int* steps) {
    QuietCout quiet;
    auto ghosts = [&](vector<vector<S> >& c) { return bc == 1 ? periodicGhosts2D(c, 1) : Sol::insertBoundaryCells2D(c, 1); };
    double t = 0.0, tEnd = t_end > 0.0 ? t_end : kNoEnd;
    int it = 0, limit = max_steps > 0 ? max_steps : 0x7fffffff;
    while (t < tEnd && it < limit) {
        vector<vector<S> > withB = ghosts(cells);
        double dt = Sol::computeStableTimeStep2D(withB, dx, cfl, t, tEnd, it, mp);
        FO::computeXFORCETimeStep2D(cells, withB, dx, 0.5 * dt, mp);
        withB = ghosts(cells);
        FO::computeYFORCETimeStep2D(cells, withB, dx, dt, mp);
        withB = ghosts(cells);
        FO::computeXFORCETimeStep2D(cells, withB, dx, 0.5 * dt, mp);
        t += dt;
        it += 1;
    }
    if (steps) *steps = it;
    return t;
}

}  // namespace

// model 0 Euler (prm as eulerParams), 1 MHD (prm = {gamma, p_inf, c_h}), 2 HPR (prm as hprParams); ny == 1: 1D.
extern "C" double vgref_first_order_run(int model, double* planes, int nx, int ny, double dx, double cfl,
                                        double t_end, int max_steps, const double* prm, int bc, int* steps_out) {
    const long plane = (long)nx * ny;
    double t = 0.0;
    if (model == 0) {
        EulerMaterialParameters mp = eulerParams(prm);
        vector<vector<EulerStateVector> > g = eulerGrid(planes, nx, ny);
        if (ny == 1)
            t = firstOrder1D<EulerStateVector, EulerMaterialParameters, Solvers, FirstOrderSolver>(g[0], dx, cfl, t_end, max_steps, mp, bc, steps_out);
        else
            t = firstOrder2D<EulerStateVector, EulerMaterialParameters, Solvers, FirstOrderSolver>(g, dx, cfl, t_end, max_steps, mp, bc, steps_out);
        eulerUngrid(g, planes, nx, ny);
    } else if (model == 1) {
        MHDMaterialParameters mp = mhdParams(prm);
        mp.setHyperbolicWaveSpeed(prm[2]);
        vector<vector<MHDStateVector> > g(ny, vector<MHDStateVector>(nx));
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) g[i][j] = mhdCell(planes, plane, (long)i * nx + j);
        if (ny == 1)
            t = firstOrder1D<MHDStateVector, MHDMaterialParameters, MHDSolvers, MHDFirstOrderSolver>(g[0], dx, cfl, t_end, max_steps, mp, bc, steps_out);
        else
            t = firstOrder2D<MHDStateVector, MHDMaterialParameters, MHDSolvers, MHDFirstOrderSolver>(g, dx, cfl, t_end, max_steps, mp, bc, steps_out);
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) mhdStore(g[i][j], planes, plane, (long)i * nx + j);
    } else {
        HPRMaterialParameters mp = hprParams(prm);
        vector<vector<HPRStateVector> > g(ny, vector<HPRStateVector>(nx));
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) g[i][j] = hprCell(planes, plane, (long)i * nx + j);
        if (ny == 1)
            t = firstOrder1D<HPRStateVector, HPRMaterialParameters, HPRSolvers, HPRFirstOrderSolver>(g[0], dx, cfl, t_end, max_steps, mp, bc, steps_out);
        else
            t = firstOrder2D<HPRStateVector, HPRMaterialParameters, HPRSolvers, HPRFirstOrderSolver>(g, dx, cfl, t_end, max_steps, mp, bc, steps_out);
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) hprStore(g[i][j], planes, plane, (long)i * nx + j);
    }
    return t;
}

// ------------------------------------------------------------------------------------ HPR EOS / source probes
// The 13 values of vo_hpr_eos from HPRMieGruneisen's own functions.  For GodunovRomenski the three values that go
// through computeGruneisenCoefficientDerivative (dGamma, de/drho, dT/drho) are NaN: that function has no
// GodunovRomenski return (HPR/hprmiegruneisen.cpp:104-119), and compiled with -O2 a call to it does not return.
extern "C" void vgref_hpr_eos(const double* prm, const double* rho, const double* p, const double* e, int n, double* out) {
    HPRMaterialParameters mp = hprParams(prm);
    const bool gr = (int)prm[12] == 2;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (int k = 0; k < n; k++) {
        double r = rho[k], *o = out + 13 * k;
        o[0] = HPRMieGruneisen::computeGruneisenCoefficient(r, mp);
        o[1] = HPRMieGruneisen::computeReferencePressure(r, mp);
        o[2] = HPRMieGruneisen::computeReferenceInternalEnergy(r, mp);
        o[3] = gr ? nan : HPRMieGruneisen::computeGruneisenCoefficientDerivative(r, mp);
        o[4] = HPRMieGruneisen::computeReferencePressureDerivative(r, mp);
        o[5] = HPRMieGruneisen::computeReferenceInternalEnergyDerivative(r, mp);
        o[6] = HPRMieGruneisen::computeInternalEnergy(r, p[k], mp);
        o[7] = HPRMieGruneisen::computePressure(r, e[k], mp);
        o[8] = HPRMieGruneisen::computeTemperature(r, p[k], mp);
        o[9] = gr ? nan : HPRMieGruneisen::computeInternalEnergyDerivativeDensity(r, p[k], mp);
        o[10] = HPRMieGruneisen::computeInternalEnergyDerivativePressure(r, mp);
        o[11] = gr ? nan : HPRMieGruneisen::computeTemperatureDerivativeDensity(r, p[k], mp);
        o[12] = HPRMieGruneisen::computeTemperatureDerivativePressure(r, mp);
    }
}

// HPRSourceTerms::computeTheta1Reciprocal of (rho[k], A = a9[9k..9k+8] row-major).
extern "C" void vgref_hpr_theta1(const double* prm, const double* rho, const double* a9, int n, double* out) {
    HPRMaterialParameters mp = hprParams(prm);
    for (int k = 0; k < n; k++) {
        vector<vector<double> > A(3, vector<double>(3));
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) A[i][j] = a9[9 * k + 3 * i + j];
        out[k] = HPRSourceTerms::computeTheta1Reciprocal(rho[k], A, mp);
    }
}

// ------------------------------------------------------------------------------------ .dat writers
// The reference scenarios' solution writers, writing density.dat etc. into the current working directory:
// EulerTests::outputSolution (Euler/eulertests.cpp:54-80), MHDTests::outputSolution{,2D} (MHD/mhdtests.cpp:123-161),
// HPRTests::outputSolution{,2D} (HPR/hprtests.cpp:219-269).  planes: the model's primitive planes, nx x ny cells.
extern "C" void vgref_write_euler(const double* planes, int n) {
    vector<EulerStateVector> cells(n);
    for (int i = 0; i < n; i++) cells[i] = eulerCell(planes, n, i);
    EulerTests::outputSolution(cells);
}

extern "C" void vgref_write_mhd(const double* planes, int nx, int ny) {
    const long plane = (long)nx * ny;
    if (ny == 1) {
        vector<MHDStateVector> cells(nx);
        for (int i = 0; i < nx; i++) cells[i] = mhdCell(planes, plane, i);
        MHDTests::outputSolution(cells);
        return;
    }
    vector<vector<MHDStateVector> > g(ny, vector<MHDStateVector>(nx));
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) g[i][j] = mhdCell(planes, plane, (long)i * nx + j);
    MHDTests::outputSolution2D(g);
}

extern "C" void vgref_write_hpr(const double* planes, int nx, int ny, const double* prm) {
    HPRMaterialParameters mp = hprParams(prm);
    const long plane = (long)nx * ny;
    if (ny == 1) {
        vector<HPRStateVector> cells(nx);
        for (int i = 0; i < nx; i++) cells[i] = hprCell(planes, plane, i);
        HPRTests::outputSolution(cells, mp);
        return;
    }
    vector<vector<HPRStateVector> > g(ny, vector<HPRStateVector>(nx));
    for (int i = 0; i < ny; i++)
        for (int j = 0; j < nx; j++) g[i][j] = hprCell(planes, plane, (long)i * nx + j);
    HPRTests::outputSolution2D(g, mp);
}

// ------------------------------------------------------------------------------ Euler reduced two-material model
// planes: the 7 primitive planes of EulerReducedStateVector (alpha1, u, v, w, rho1, rho2, p; :30-41), nx x ny cells;
// prm = {gamma1, p_inf1, gamma2, p_inf2}.  max_steps <= 0: the reference's own SecondOrderSolver::solve{,2D} to t_end;
// else its per-step functions for max_steps steps, in solve's order (Solvers/secondordersolver.cpp:354-385, :470-...),
// with the volume-fraction reinitialisation every reinit_freq steps.
static EulerReducedStateVector redCell(const double* planes, long plane, long k) {
    return EulerReducedStateVector(planes[k], planes[plane + k], planes[2 * plane + k], planes[3 * plane + k],
                                   planes[4 * plane + k], planes[5 * plane + k], planes[6 * plane + k]);
}
static void redStore(EulerReducedStateVector& c, double* planes, long plane, long k) {
    vector<double> w = c.computePrimitiveVariableVector();
    for (int v = 0; v < 7; v++) planes[v * plane + k] = w[v];
}

extern "C" double vgref_reduced_run(double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                                    double bias, int limiter, const double* prm, int reinit_freq, int* steps_out) {
    EulerMaterialParameters m1(prm[0], prm[1]), m2(prm[2], prm[3]);
    const long plane = (long)nx * ny;
    double t = 0.0;
    int it = 0;
    if (ny == 1) {
        vector<EulerReducedStateVector> cells(nx);
        for (int i = 0; i < nx; i++) cells[i] = redCell(planes, plane, i);
        if (max_steps <= 0) {
            cells = SecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, 0, reinit_freq, m1, m2);
            t = t_end;
        } else {
            for (; it < max_steps; it++) {
                vector<EulerReducedStateVector> withB = Solvers::insertBoundaryCells(cells, 2);
                double dt = Solvers::computeStableTimeStep(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                SecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, m1, m2);
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(cells, m1, m2);
            }
        }
        for (int i = 0; i < nx; i++) redStore(cells[i], planes, plane, i);
    } else {
        vector<vector<EulerReducedStateVector> > g(ny, vector<EulerReducedStateVector>(nx));
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) g[i][j] = redCell(planes, plane, (long)i * nx + j);
        if (max_steps <= 0) {
            g = SecondOrderSolver::solve2D(g, dx, cfl, t_end, bias, limiter, 0, reinit_freq, m1, m2);
            t = t_end;
        } else {
            for (; it < max_steps; it++) {
                vector<vector<EulerReducedStateVector> > withB = Solvers::insertBoundaryCells2D(g, 2);
                double dt = Solvers::computeStableTimeStep2D(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                SecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                withB = Solvers::insertBoundaryCells2D(g, 2);
                SecondOrderSolver::computeYSLICTimeStep2D(g, withB, dx, dt, bias, limiter, m1, m2);
                withB = Solvers::insertBoundaryCells2D(g, 2);
                SecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(g, m1, m2);
            }
        }
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) redStore(g[i][j], planes, plane, (long)i * nx + j);
    }
    if (steps_out) *steps_out = it;
    return t;
}

// ------------------------------------------------------------------------- Euler multiphysics two-material model
// planes: the 8 primitive planes of EulerMultiphysicsStateVector (alpha1, u, v, w, rho1, p1, rho2, p2; :32-44);
// prm = {gamma1, p_inf1, gamma2, p_inf2}.  max_steps <= 0: the reference's own SecondOrderSolver::solve{,2D} to t_end;
// else its per-step functions for max_steps steps, in solve's order (Solvers/secondordersolver.cpp:354-385, :470-...),
// with the volume-fraction reinitialisation every reinit_freq steps.
static EulerMultiphysicsStateVector mphCell(const double* planes, long plane, long k) {
    return EulerMultiphysicsStateVector(planes[k], planes[plane + k], planes[2 * plane + k], planes[3 * plane + k],
                                        planes[4 * plane + k], planes[5 * plane + k], planes[6 * plane + k],
                                        planes[7 * plane + k]);
}
static void mphStore(EulerMultiphysicsStateVector& c, double* planes, long plane, long k) {
    vector<double> w = c.computePrimitiveVariableVector();
    for (int v = 0; v < 8; v++) planes[v * plane + k] = w[v];
}

extern "C" double vgref_multiphysics_run(double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                                    double bias, int limiter, const double* prm, int reinit_freq, int* steps_out) {
    EulerMaterialParameters m1(prm[0], prm[1]), m2(prm[2], prm[3]);
    const long plane = (long)nx * ny;
    double t = 0.0;
    int it = 0;
    if (ny == 1) {
        vector<EulerMultiphysicsStateVector> cells(nx);
        for (int i = 0; i < nx; i++) cells[i] = mphCell(planes, plane, i);
        if (max_steps <= 0) {
            cells = SecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, 0, reinit_freq, m1, m2);
            t = t_end;
        } else {
            for (; it < max_steps; it++) {
                vector<EulerMultiphysicsStateVector> withB = Solvers::insertBoundaryCells(cells, 2);
                double dt = Solvers::computeStableTimeStep(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                SecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, m1, m2);
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(cells, m1, m2);
            }
        }
        for (int i = 0; i < nx; i++) mphStore(cells[i], planes, plane, i);
    } else {
        vector<vector<EulerMultiphysicsStateVector> > g(ny, vector<EulerMultiphysicsStateVector>(nx));
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) g[i][j] = mphCell(planes, plane, (long)i * nx + j);
        if (max_steps <= 0) {
            g = SecondOrderSolver::solve2D(g, dx, cfl, t_end, bias, limiter, 0, reinit_freq, m1, m2);
            t = t_end;
        } else {
            for (; it < max_steps; it++) {
                vector<vector<EulerMultiphysicsStateVector> > withB = Solvers::insertBoundaryCells2D(g, 2);
                double dt = Solvers::computeStableTimeStep2D(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                SecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                withB = Solvers::insertBoundaryCells2D(g, 2);
                SecondOrderSolver::computeYSLICTimeStep2D(g, withB, dx, dt, bias, limiter, m1, m2);
                withB = Solvers::insertBoundaryCells2D(g, 2);
                SecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(g, m1, m2);
            }
        }
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) mphStore(g[i][j], planes, plane, (long)i * nx + j);
    }
    if (steps_out) *steps_out = it;
    return t;
}



// ---------------------------------------------------------------- MHD reduced and intermediate two-material models
// planes: the primitive planes of MHDReducedStateVector (11: alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi;
// MHD/Multiphysics/mhdreducedstatevector.cpp:91-111) or of MHDIntermediateStateVector (12: alpha1, u, v, w, rho1, p1,
// rho2, p2, Bx, By, Bz, psi; MHD/Multiphysics/mhdintermediatestatevector.cpp:108-130); prm = {gamma1, p_inf1, gamma2,
// p_inf2}.  max_steps <= 0: the reference's own MHDSecondOrderSolver::solve{,2D} to t_end (Solvers/
// mhdsecondordersolver.cpp:387-440, :445-495, :552-..., :615-675); else its per-step functions for max_steps steps in
// solve's order: c_h of both materials = the padded grid's maximum wave speed, RK4 GLM damping sub-cycles around the
// sweeps, reinitialisation every reinit_freq steps.  The intermediate model in 2D: per-step only (its solve2D pads the
// grid with the defective insertBoundaryCells2D, see mirrorGhosts2D), with mirror ghosts built here.
template <class SV>
static SV mhdTwoCell(const double* planes, long plane, long k);
template <>
MHDReducedStateVector mhdTwoCell<MHDReducedStateVector>(const double* planes, long plane, long k) {
    return MHDReducedStateVector(planes[k], planes[plane + k], planes[2 * plane + k], planes[3 * plane + k],
                                 planes[4 * plane + k], planes[5 * plane + k], planes[6 * plane + k],
                                 planes[7 * plane + k], planes[8 * plane + k], planes[9 * plane + k],
                                 planes[10 * plane + k]);
}
template <>
MHDIntermediateStateVector mhdTwoCell<MHDIntermediateStateVector>(const double* planes, long plane, long k) {
    MHDIntermediateStateVector c;
    vector<double> w(12);
    for (int v = 0; v < 12; v++) w[v] = planes[v * plane + k];
    c.setPrimitiveVariableVector(w);
    return c;
}
template <class SV>
static void mhdTwoStore(SV& c, double* planes, long plane, long k) {
    vector<double> w = c.computePrimitiveVariableVector();
    for (size_t v = 0; v < w.size(); v++) planes[v * plane + k] = w[v];
}

template <class SV>
static double mhdTwoMaterialRun(double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                                double bias, int limiter, const double* prm, int subcycles, int reinit_freq,
                                int* steps_out) {
    QuietCout quiet;
    MHDMaterialParameters m1 = mhdParams(prm), m2 = mhdParams(prm + 2);
    const long plane = (long)nx * ny;
    double t = 0.0;
    int it = 0;
    auto glm = [&](double smax) {
        m1.setHyperbolicWaveSpeed(smax);
        m2.setHyperbolicWaveSpeed(smax);
        m1.configureParabolicDamping();
        m2.configureParabolicDamping();
    };
    if (ny == 1) {
        vector<SV> cells(nx);
        for (int i = 0; i < nx; i++) cells[i] = mhdTwoCell<SV>(planes, plane, i);
        if (max_steps <= 0) {
            cells = MHDSecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, subcycles, reinit_freq, m1, m2);
            t = t_end;
        } else {
            for (; it < max_steps; it++) {
                vector<SV> withB = MHDSolvers::insertBoundaryCells(cells, 2);
                double dt = MHDSolvers::computeStableTimeStep(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                glm(MHDSolvers::computeMaximumWaveSpeed(withB, m1, m2));
                for (int s = 0; s < subcycles; s++) {
                    withB = MHDSolvers::insertBoundaryCells(cells, 1);
                    MHDForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                withB = MHDSolvers::insertBoundaryCells(cells, 2);
                MHDSecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, m1, m2);
                for (int s = 0; s < subcycles; s++) {
                    withB = MHDSolvers::insertBoundaryCells(cells, 1);
                    MHDForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(cells, m1, m2);
            }
        }
        for (int i = 0; i < nx; i++) mhdTwoStore(cells[i], planes, plane, i);
    } else {
        vector<vector<SV> > g(ny, vector<SV>(nx));
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) g[i][j] = mhdTwoCell<SV>(planes, plane, (long)i * nx + j);
        if (max_steps <= 0) {
            g = MHDSecondOrderSolver::solve2D(g, dx, cfl, t_end, bias, limiter, subcycles, reinit_freq, m1, m2);
            t = t_end;
        } else {
            // the intermediate model's own 2-ghost insertion has the defect above: mirror ghosts built here instead
            auto ghosts = [&](vector<vector<SV> >& c, int b) {
                return (b == 2 && std::is_same<SV, MHDIntermediateStateVector>::value) ? mirrorGhosts2D(c, b)
                                                                                       : MHDSolvers::insertBoundaryCells2D(c, b);
            };
            for (; it < max_steps; it++) {
                vector<vector<SV> > withB = ghosts(g, 2);
                double dt = MHDSolvers::computeStableTimeStep2D(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                glm(MHDSolvers::computeMaximumWaveSpeed2D(withB, m1, m2));
                for (int s = 0; s < subcycles; s++) {
                    withB = ghosts(g, 1);
                    MHDForcingSolver::computeRungeKuttaTimeStep2D(g, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                withB = ghosts(g, 2);
                MHDSecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                withB = ghosts(g, 2);
                MHDSecondOrderSolver::computeYSLICTimeStep2D(g, withB, dx, dt, bias, limiter, m1, m2);
                withB = ghosts(g, 2);
                MHDSecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                for (int s = 0; s < subcycles; s++) {
                    withB = ghosts(g, 1);
                    MHDForcingSolver::computeRungeKuttaTimeStep2D(g, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(g, m1, m2);
            }
        }
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) mhdTwoStore(g[i][j], planes, plane, (long)i * nx + j);
    }
    if (steps_out) *steps_out = it;
    return t;
}

extern "C" double vgref_mhd_reduced_run(double* planes, int nx, int ny, double dx, double cfl, double t_end,
                                        int max_steps, double bias, int limiter, const double* prm, int subcycles,
                                        int reinit_freq, int* steps_out) {
    return mhdTwoMaterialRun<MHDReducedStateVector>(planes, nx, ny, dx, cfl, t_end, max_steps, bias, limiter, prm,
                                                    subcycles, reinit_freq, steps_out);
}

extern "C" double vgref_mhd_intermediate_run(double* planes, int nx, int ny, double dx, double cfl, double t_end,
                                             int max_steps, double bias, int limiter, const double* prm, int subcycles,
                                             int reinit_freq, int* steps_out) {
    return mhdTwoMaterialRun<MHDIntermediateStateVector>(planes, nx, ny, dx, cfl, t_end, max_steps, bias, limiter,
                                                         prm, subcycles, reinit_freq, steps_out);
}

// ------------------------------------------------------------------------------------ HPR reduced two-material
// Planes: the 19 primitives of HPRReducedStateVector (alpha1, p, A(9), u, v, w, Jx, Jy, Jz, rho1, rho2;
// HPR/Multiphysics/hprreducedstatevector.cpp:154-185).  prm holds each material's HPRMaterialParameters as the 20-value
// block of hprParams, material k at prm[20 k].
// max_steps <= 0: the reference's own HPRSecondOrderSolver::solve{,2D} to t_end (Solvers/hprsecondordersolver.cpp:
// 452-..., :604-...); else its per-step functions for max_steps steps in solve's order: the RK4 forcing sub-cycles
// around the sweeps and the reinitialisation every reinit_freq steps.
static HPRMaterialParameters hredParams(const double* prm, int k) { return hprParams(prm + 20 * k); }
template <class SV>
static SV hprTwoCell(const double* planes, long plane, long k, int nw, HPRMaterialParameters& m1,
                     HPRMaterialParameters& m2) {
    SV c;
    vector<double> w(nw);
    for (int v = 0; v < nw; v++) w[v] = planes[v * plane + k];
    c.setPrimitiveVariableVector(w, m1, m2);
    return c;
}
template <class SV>
static void hprTwoStore(SV& c, double* planes, long plane, long k, int nw, HPRMaterialParameters& m1,
                        HPRMaterialParameters& m2) {
    vector<double> w = c.computePrimitiveVariableVector(m1, m2);
    for (int v = 0; v < nw; v++) planes[v * plane + k] = w[v];
}

// The HPR two-material solve loop of HPRSecondOrderSolver::solve{,2D} (Solvers/hprsecondordersolver.cpp:402-450,
// :452-500 in 1D, :548-602, :604-658 in 2D) for a state type SV with nw primitives: the reference's own solve to t_end
// when max_steps <= 0, else its per-step functions for max_steps steps in solve's order.
template <class SV>
static double hprTwoMaterialRun(double* planes, int nw, int nx, int ny, double dx, double cfl, double t_end,
                                int max_steps, double bias, int limiter, const double* prm, int subcycles,
                                int reinit_freq, int* steps_out) {
    QuietCout quiet;
    HPRMaterialParameters m1 = hredParams(prm, 0), m2 = hredParams(prm, 1);
    const long plane = (long)nx * ny;
    double t = 0.0;
    int it = 0;
    if (ny == 1) {
        vector<SV> cells(nx);
        for (int i = 0; i < nx; i++) cells[i] = hprTwoCell<SV>(planes, plane, i, nw, m1, m2);
        if (max_steps <= 0) {
            cells = HPRSecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, subcycles, reinit_freq, m1, m2);
            t = t_end;
        } else {
            for (; it < max_steps; it++) {
                vector<SV> withB = HPRSolvers::insertBoundaryCells(cells, 2);
                double dt = HPRSolvers::computeStableTimeStep(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                for (int s = 0; s < subcycles; s++) {
                    withB = HPRSolvers::insertBoundaryCells(cells, 1);
                    HPRForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                withB = HPRSolvers::insertBoundaryCells(cells, 2);
                HPRSecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, m1, m2);
                for (int s = 0; s < subcycles; s++) {
                    withB = HPRSolvers::insertBoundaryCells(cells, 1);
                    HPRForcingSolver::computeRungeKuttaTimeStep(cells, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(cells, m1, m2);
            }
        }
        for (int i = 0; i < nx; i++) hprTwoStore(cells[i], planes, plane, i, nw, m1, m2);
    } else {
        vector<vector<SV> > g(ny, vector<SV>(nx));
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) g[i][j] = hprTwoCell<SV>(planes, plane, (long)i * nx + j, nw, m1, m2);
        if (max_steps <= 0) {
            g = HPRSecondOrderSolver::solve2D(g, dx, cfl, t_end, bias, limiter, subcycles, reinit_freq, m1, m2);
            t = t_end;
        } else {
            for (; it < max_steps; it++) {
                vector<vector<SV> > withB = HPRSolvers::insertBoundaryCells2D(g, 2);
                double dt = HPRSolvers::computeStableTimeStep2D(withB, dx, cfl, t, 1.0e300, it, m1, m2);
                for (int s = 0; s < subcycles; s++) {
                    withB = HPRSolvers::insertBoundaryCells2D(g, 1);
                    HPRForcingSolver::computeRungeKuttaTimeStep2D(g, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                withB = HPRSolvers::insertBoundaryCells2D(g, 2);
                HPRSecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                withB = HPRSolvers::insertBoundaryCells2D(g, 2);
                HPRSecondOrderSolver::computeYSLICTimeStep2D(g, withB, dx, dt, bias, limiter, m1, m2);
                withB = HPRSolvers::insertBoundaryCells2D(g, 2);
                HPRSecondOrderSolver::computeXSLICTimeStep2D(g, withB, dx, 0.5 * dt, bias, limiter, m1, m2);
                for (int s = 0; s < subcycles; s++) {
                    withB = HPRSolvers::insertBoundaryCells2D(g, 1);
                    HPRForcingSolver::computeRungeKuttaTimeStep2D(g, withB, dx, 0.5 * (dt / subcycles), bias, limiter, m1, m2);
                }
                t += dt;
                if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                    MultiphysicsSolvers::reinitialiseVolumeFraction(g, m1, m2);
            }
        }
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) hprTwoStore(g[i][j], planes, plane, (long)i * nx + j, nw, m1, m2);
    }
    if (steps_out) *steps_out = it;
    return t;
}

extern "C" double vgref_hpr_reduced_run(double* planes, int nx, int ny, double dx, double cfl, double t_end,
                                        int max_steps, double bias, int limiter, const double* prm, int subcycles,
                                        int reinit_freq, int* steps_out) {
    return hprTwoMaterialRun<HPRReducedStateVector>(planes, 19, nx, ny, dx, cfl, t_end, max_steps, bias, limiter, prm,
                                                    subcycles, reinit_freq, steps_out);
}

// ------------------------------------------------------------------------------- HPR intermediate two-material
// Planes: the 20 primitives of HPRIntermediateStateVector (alpha1, A(9), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2;
// HPR/Multiphysics/hprintermediatestatevector.cpp:161-193); prm as for the reduced model.
extern "C" double vgref_hpr_intermediate_run(double* planes, int nx, int ny, double dx, double cfl, double t_end,
                                             int max_steps, double bias, int limiter, const double* prm, int subcycles,
                                             int reinit_freq, int* steps_out) {
    return hprTwoMaterialRun<HPRIntermediateStateVector>(planes, 20, nx, ny, dx, cfl, t_end, max_steps, bias, limiter,
                                                         prm, subcycles, reinit_freq, steps_out);
}

// ------------------------------------------------------------------------------- HPR multiphysics two-material
// Planes: the 32 primitives of HPRMultiphysicsStateVector (alpha1, u, v, w, rho1, p1, A1(9), J1(3), rho2, p2, A2(9),
// J2(3); HPR/Multiphysics/hprmultiphysicsstatevector.cpp:204-249); prm as for the reduced model; 1D only, as the
// reference has it.  max_steps <= 0: the reference's own HPRSecondOrderSolver::solve to t_end (Solvers/
// hprsecondordersolver.cpp:354-400, whose sub-cycle loops only pad the grid); else its per-step functions for max_steps
// steps in solve's order, with the reinitialisation every reinit_freq steps.
extern "C" double vgref_hpr_multiphysics_run(double* planes, int nx, double dx, double cfl, double t_end, int max_steps,
                                             double bias, int limiter, const double* prm, int subcycles,
                                             int reinit_freq, int* steps_out) {
    QuietCout quiet;
    HPRMaterialParameters m1 = hredParams(prm, 0), m2 = hredParams(prm, 1);
    const long plane = nx;
    double t = 0.0;
    int it = 0;
    vector<HPRMultiphysicsStateVector> cells(nx);
    for (int i = 0; i < nx; i++) cells[i] = hprTwoCell<HPRMultiphysicsStateVector>(planes, plane, i, 32, m1, m2);
    if (max_steps <= 0) {
        cells = HPRSecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, subcycles, reinit_freq, m1, m2);
        t = t_end;
    } else {
        for (; it < max_steps; it++) {
            vector<HPRMultiphysicsStateVector> withB = HPRSolvers::insertBoundaryCells(cells, 2);
            double dt = HPRSolvers::computeStableTimeStep(withB, dx, cfl, t, 1.0e300, it, m1, m2);
            withB = HPRSolvers::insertBoundaryCells(cells, 2);
            HPRSecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, m1, m2);
            t += dt;
            if (reinit_freq != 0 && ((it + 1) % reinit_freq) == 0)
                MultiphysicsSolvers::reinitialiseVolumeFraction(cells, m1, m2);
        }
    }
    for (int i = 0; i < nx; i++) hprTwoStore(cells[i], planes, plane, i, 32, m1, m2);
    if (steps_out) *steps_out = it;
    return t;
}

// ------------------------------------------------------------------------------- MHD multiphysics two-material
// Planes: the 16 primitives of MHDMultiphysicsStateVector (alpha1, u, v, w, rho1, p1, B1(3), psi1, rho2, p2, B2(3),
// psi2; MHD/Multiphysics/mhdmultiphysicsstatevector.cpp:135-163); prm = {gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2};
// 1D only, as the reference has it.  max_steps <= 0: the reference's own MHDSecondOrderSolver::solve to t_end
// (Solvers/mhdsecondordersolver.cpp:362-385: no source, no reinitialisation, the materials' c_h as given); else its
// per-step functions for max_steps steps in solve's order.
extern "C" double vgref_mhd_multiphysics_run(double* planes, int nx, double dx, double cfl, double t_end, int max_steps,
                                             double bias, int limiter, const double* prm, int* steps_out) {
    QuietCout quiet;
    MHDMaterialParameters m1 = mhdParams(prm), m2 = mhdParams(prm + 2);
    m1.setHyperbolicWaveSpeed(prm[4]);
    m2.setHyperbolicWaveSpeed(prm[5]);
    double t = 0.0;
    int it = 0;
    vector<MHDMultiphysicsStateVector> cells(nx);
    for (int i = 0; i < nx; i++) {
        vector<double> w(16);
        for (int v = 0; v < 16; v++) w[v] = planes[(long)v * nx + i];
        cells[i].setPrimitiveVariableVector(w);
    }
    if (max_steps <= 0) {
        cells = MHDSecondOrderSolver::solve(cells, dx, cfl, t_end, bias, limiter, 0, 0, m1, m2);
        t = t_end;
    } else {
        for (; it < max_steps; it++) {
            vector<MHDMultiphysicsStateVector> withB = MHDSolvers::insertBoundaryCells(cells, 2);
            double dt = MHDSolvers::computeStableTimeStep(withB, dx, cfl, t, 1.0e300, it, m1, m2);
            MHDSecondOrderSolver::computeSLICTimeStep(cells, withB, dx, dt, bias, limiter, m1, m2);
            t += dt;
        }
    }
    for (int i = 0; i < nx; i++) {
        vector<double> w = cells[i].computePrimitiveVariableVector();
        for (int v = 0; v < 16; v++) planes[(long)v * nx + i] = w[v];
    }
    if (steps_out) *steps_out = it;
    return t;
}
