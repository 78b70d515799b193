// A Vanguard-style caller of the drop-in C++ surface: it uses only the reference's class names and
// signatures (as EulerTests::solveToroTest1 and RGFM's per-sweep calls do) and writes the resulting primitive
// planes to a binary file for tests/test_shim_gpu.py to compare with the oracle.
//   shim_driver <out.bin>
// Output, in order (float64): Euler 1D solve (6 x 200), Euler 2D per-sweep loop (6 x 24 x 20),
// MHD solve2D (9 x 16 x 16), HPR solve (17 x 50), Euler 1D step-count solve (6 x 150), Euler 1D first-order solve
// (6 x 150), HPR GodunovRomenski plastic solve (17 x 60), reduced two-material solve (7 x 120), multiphysics
// two-material solve (8 x 100), MHD reduced two-material solve2D (11 x 24 x 24), MHD intermediate two-material solve
// (12 x 80), the 2D maximum wave speed of an interior-only cold gas (1), whether solve2D refused a single row (1),
// HPR reduced two-material solve2D (19 x 16 x 16), HPR intermediate two-material solve (20 x 60), HPR multiphysics
// two-material solve (32 x 60), MHD multiphysics two-material solve (16 x 80), then the number of 2D steps the
// per-sweep loop took.
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "Solvers/firstordersolver.h"
#include "Solvers/secondordersolver.h"
#include "Solvers/mhdsecondordersolver.h"
#include "MHD/Multiphysics/mhdreducedstatevector.h"
#include "MHD/Multiphysics/mhdintermediatestatevector.h"
#include "MHD/Multiphysics/mhdmultiphysicsstatevector.h"
#include "Solvers/hprsecondordersolver.h"
#include "HPR/Multiphysics/hprreducedstatevector.h"
#include "HPR/Multiphysics/hprintermediatestatevector.h"
#include "HPR/Multiphysics/hprmultiphysicsstatevector.h"

using std::vector;

static void put(FILE* f, const vector<double>& v) { std::fwrite(v.data(), sizeof(double), v.size(), f); }

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    FILE* f = std::fopen(argv[1], "wb");
    if (!f) return 3;

    // 1) SecondOrderSolver::solve on a shock tube (minbee, CFL 0.9, to t = 0.1)
    {
        int n = 200;
        vector<EulerStateVector> cells(n);
        EulerMaterialParameters mp(1.4);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n ? EulerStateVector(1.0, 0.0, 0.0, 0.0, 1.0) : EulerStateVector(0.125, 0.0, 0.0, 0.0, 0.1);
        vector<EulerStateVector> out = SecondOrderSolver::solve(cells, 1.0 / n, 0.9, 0.1, 0.0, 2, 0, mp);
        vector<double> v;
        for (int k = 0; k < 6; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 2) the per-step functions, as solve2D is built from them (Solvers/secondordersolver.cpp:399-410)
    int steps = 0;
    {
        int nx = 24, ny = 20;
        vector<vector<EulerStateVector> > cells(ny, vector<EulerStateVector>(nx));
        EulerMaterialParameters mp(1.4);
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++)
                cells[i][j] = (i < ny / 2) == (j < nx / 2) ? EulerStateVector(1.0, 0.1, -0.2, 0.0, 1.0)
                                                           : EulerStateVector(0.3, -0.1, 0.3, 0.0, 0.4);
        double t = 0.0, dx = 1.0 / nx;
        for (steps = 0; steps < 6; steps++) {
            vector<vector<EulerStateVector> > withB = Solvers::insertBoundaryCells2D(cells, 2);
            double dt = Solvers::computeStableTimeStep2D(withB, dx, 0.8, t, 1.0, steps, mp);
            SecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, 0.0, 0, mp);
            withB = Solvers::insertBoundaryCells2D(cells, 2);
            SecondOrderSolver::computeYSLICTimeStep2D(cells, withB, dx, dt, 0.0, 0, mp);
            withB = Solvers::insertBoundaryCells2D(cells, 2);
            SecondOrderSolver::computeXSLICTimeStep2D(cells, withB, dx, 0.5 * dt, 0.0, 0, mp);
            t += dt;
        }
        vector<double> v;
        for (int k = 0; k < 6; k++)
            for (auto& row : cells)
                for (auto& c : row) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 3) MHDSecondOrderSolver::solve2D (to t = 0.02)
    {
        int n = 16;
        const double pi = 3.14159265358979323846, g = 5.0 / 3.0, s = 1.0 / std::sqrt(4.0 * pi);
        vector<vector<MHDStateVector> > cells(n, vector<MHDStateVector>(n));
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double x = (j + 0.5) / n, y = (i + 0.5) / n;
                cells[i][j] = MHDStateVector(g * g, -std::sin(2 * pi * y), std::sin(2 * pi * x), 0.0, g, -std::sin(2 * pi * y) * s,
                                             std::sin(4 * pi * x) * s, 0.0, 0.0);
            }
        vector<vector<MHDStateVector> > out = MHDSecondOrderSolver::solve2D(cells, 1.0 / n, 0.8, 0.02, 0.0, 0, 0, MHDMaterialParameters(g));
        vector<double> v;
        for (int k = 0; k < 9; k++)
            for (auto& row : out)
                for (auto& c : row) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 4) HPRSecondOrderSolver::solve with the heat-conduction material (HPR/hprtests.cpp:33-57), 1 sub-cycle, t = 0.02
    {
        int n = 50;
        HPRMaterialParameters mp("StiffenedGas", true, false, 8.31445985, 1.0, 1.0, 0.0, 1.0, 2.5, 1.4, 0.0, 0.0, 0.0, 0.0, 0.0,
                                 1.0, 0.0, 0.0, std::pow(10.0, -2.0), 0.75, 0.0, 1.0, 2.0, 0.0, 0.0, 0.0);
        mp.configureStrainDissipationTime();
        mp.configureThermalImpulseRelaxationTime(std::pow(10.0, -2.0));
        vector<HPRStateVector> cells(n);
        for (int i = 0; i < n; i++) {
            double r = i <= 0.5 * n ? 2.0 : 0.5, a = std::pow(r, 1.0 / 3.0);
            vector<vector<double> > A = {{a, 0.0, 0.0}, {0.0, a, 0.0}, {0.0, 0.0, a}};
            cells[i] = HPRStateVector(r, 1.0, A, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
        }
        vector<HPRStateVector> out = HPRSecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.02, 0.0, 0, 1, mp);
        vector<double> v;
        for (int k = 0; k < 17; k++)
            for (auto& c : out) v.push_back(c.data()[k]);
        put(f, v);
    }
    // 5) the step-count overload: SecondOrderSolver::solve(..., maxSteps) with no end time, superbee, 37 steps
    {
        int n = 150;
        vector<EulerStateVector> cells(n);
        EulerMaterialParameters mp(1.4);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n ? EulerStateVector(1.0, 0.0, 0.0, 0.0, 1.0) : EulerStateVector(0.125, 0.0, 0.0, 0.0, 0.1);
        vector<EulerStateVector> out = SecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.0, 0.0, 0, 0, mp, 37);
        vector<double> v;
        for (int k = 0; k < 6; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 6) FirstOrderSolver::solve on the same shock tube, to t = 0.05
    {
        int n = 150;
        vector<EulerStateVector> cells(n);
        EulerMaterialParameters mp(1.4);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n ? EulerStateVector(1.0, 0.0, 0.0, 0.0, 1.0) : EulerStateVector(0.125, 0.0, 0.0, 0.0, 0.1);
        vector<EulerStateVector> out = FirstOrderSolver::solve(cells, 1.0 / n, 0.8, 0.05, 0, mp);
        vector<double> v;
        for (int k = 0; k < 6; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 7) HPRSecondOrderSolver::solve, step-count overload, with the reference's Zhang elastic-plastic material
    //    (GodunovRomenski, plastic; HPR/hprtests.cpp:109-115), A = I, rho = rho0, u = +-0.75, p = 0, 2 sub-cycles
    {
        int n = 60;
        HPRMaterialParameters mp("GodunovRomenski", false, true, 8.31445985, 2.71, 73.0, 300.0, 300.0, 9.0 * std::pow(10.0, -4.0),
                                 1.0, 0.0, 5.037, 1.0, 1.338, 0.0, 3.16, std::pow(10.0, -9.0), 0.0, 24.8 * std::pow(10.0, 9.0),
                                 0.75, 0.2976 * std::pow(10.0, 9.0), 1.338, 2.0, 1.0, 3.577, 2.088);
        vector<vector<double> > I = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
        vector<HPRStateVector> cells(n);
        for (int i = 0; i < n; i++)
            cells[i] = HPRStateVector(2.71, 0.0, I, i <= 0.5 * n ? 0.75 : -0.75, 0.0, 0.0, 0.0, 0.0, 0.0);
        vector<HPRStateVector> out = HPRSecondOrderSolver::solve(cells, 10.0 / n, 0.8, 0.0, 0.0, 0, 2, mp, 20);
        vector<double> v;
        for (int k = 0; k < 17; k++)
            for (auto& c : out) v.push_back(c.data()[k]);
        put(f, v);
    }
    // 8) SecondOrderSolver::solve of the reduced two-material model (EulerReducedTests::solveToroTest1's layout),
    //    gamma 1.4 | 1.67, reinitialisation every 5 steps, to t = 0.05
    {
        int n = 120;
        vector<EulerReducedStateVector> cells(n);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n ? EulerReducedStateVector(0.999, 0.0, 0.0, 0.0, 1.0, 0.125, 1.0)
                                    : EulerReducedStateVector(0.001, 0.0, 0.0, 0.0, 1.0, 0.125, 0.1);
        vector<EulerReducedStateVector> out = SecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.05, 0.0, 0, 0, 5,
                                                                       EulerMaterialParameters(1.4),
                                                                       EulerMaterialParameters(1.67));
        vector<double> v;
        for (int k = 0; k < 7; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 9) SecondOrderSolver::solve of the multiphysics two-material model, reinitialisation every 4 steps, t = 0.04
    {
        int n = 100;
        vector<EulerMultiphysicsStateVector> cells(n);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n ? EulerMultiphysicsStateVector(0.999, 0.0, 0.0, 0.0, 1.0, 2.0, 0.1379, 2.0)
                                    : EulerMultiphysicsStateVector(0.001, 0.0, 0.0, 0.0, 1.0, 1.0, 0.1379, 1.0);
        vector<EulerMultiphysicsStateVector> out = SecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.04, 0.0, 0, 0, 4,
                                                                            EulerMaterialParameters(1.4),
                                                                            EulerMaterialParameters(1.67));
        vector<double> v;
        for (int k = 0; k < 8; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 10) MHDSecondOrderSolver::solve2D of the MHD reduced two-material model (MHDReducedTests::
    //     solve2DDumbserMultimaterialTest1's layout), gamma 1.4 | 1.67, one GLM sub-cycle, reinitialisation every 3
    //     steps, 6 steps
    {
        int n = 24;
        vector<vector<MHDReducedStateVector> > cells(n, vector<MHDReducedStateVector>(n));
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double r = std::sqrt(((i - (0.5 * n)) * (i - (0.5 * n))) + ((j - (0.5 * n)) * (j - (0.5 * n))));
                cells[i][j] = r <= 0.2 * n ? MHDReducedStateVector(0.999, 0.0, 0.0, 0.0, 1.0, 0.125, 1.0, 0.75, 1.0, 0.0, 0.0)
                                           : MHDReducedStateVector(0.001, 0.0, 0.0, 0.0, 1.0, 0.125, 0.1, 0.75, -1.0, 0.0, 0.0);
            }
        vector<vector<MHDReducedStateVector> > out = MHDSecondOrderSolver::solve2D(
            cells, 1.0 / n, 0.8, 1.0, 0.0, 0, 1, 3, MHDMaterialParameters(1.4), MHDMaterialParameters(1.67), 6);
        vector<double> v;
        for (int k = 0; k < 11; k++)
            for (auto& row : out)
                for (auto& c : row) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 11) MHDSecondOrderSolver::solve of the MHD intermediate two-material model, gamma 1.4 | 1.67, one GLM sub-cycle,
    //     reinitialisation every 5 steps, to t = 0.05
    {
        int n = 80;
        vector<MHDIntermediateStateVector> cells(n);
        for (int i = 0; i < n; i++) {
            bool left = i <= 0.5 * n;
            cells[i].setPrimitiveVariableVector(left ? vector<double>{0.999, 0.0, 0.0, 0.0, 1.0, 1.0, 0.125, 1.0, 0.75, 1.0, 0.0, 0.0}
                                                     : vector<double>{0.001, 0.0, 0.0, 0.0, 1.0, 0.1, 0.125, 0.1, 0.75, -1.0, 0.0, 0.0});
        }
        vector<MHDIntermediateStateVector> out = MHDSecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.05, 0.0, 2, 1, 5,
                                                                             MHDMaterialParameters(1.4),
                                                                             MHDMaterialParameters(1.67));
        vector<double> v;
        for (int k = 0; k < 12; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 12) Solvers::computeMaximumWaveSpeed2D over interior cells only (no ghosts, so no default-state corners): a cold
    //     gas whose own speeds are below the default state's; then solve2D on a single row, which the reference's 2D
    //     ghost insertion does not define: the shim must refuse it (1.0 written when it throws invalid_argument)
    {
        int nx = 8, ny = 6;
        vector<vector<EulerStateVector> > cells(ny, vector<EulerStateVector>(nx));
        for (int i = 0; i < ny; i++)
            for (int j = 0; j < nx; j++) cells[i][j] = EulerStateVector(1.0 + 0.01 * j, 0.01 * i, -0.02 * j, 0.0, 0.01 + 0.001 * i);
        double smax = Solvers::computeMaximumWaveSpeed2D(cells, EulerMaterialParameters(1.4));
        put(f, vector<double>{smax});
        vector<vector<EulerStateVector> > row(1, vector<EulerStateVector>(10, EulerStateVector(1.0, 0.0, 0.0, 0.0, 1.0)));
        double refused = 0.0;
        try {
            SecondOrderSolver::solve2D(row, 0.1, 0.8, 0.01, 0.0, 0, 0, EulerMaterialParameters(1.4));
        } catch (const std::invalid_argument&) {
            refused = 1.0;
        }
        put(f, vector<double>{refused});
    }
    // 13) HPRSecondOrderSolver::solve2D of the HPR reduced two-material model: a disc of material 1 in material 2
    //     (ideal gas gamma 1.4 | stiffened gas gamma 2, p_inf 0.5, both thermal), one relaxation sub-cycle,
    //     reinitialisation every 2 steps, 4 steps
    HPRMaterialParameters hm1("StiffenedGas", true, false, 8.31445985, 1.0, 1.0, 0.0, 1.0, 2.5, 1.4, 0.0, 0.0, 0.0, 0.0,
                              0.0, 1.0, 1e-2, 1e-2, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0);
    HPRMaterialParameters hm2("StiffenedGas", true, false, 8.31445985, 1.0, 1.0, 0.0, 1.0, 2.5, 2.0, 0.5, 0.0, 0.0, 0.0,
                              0.0, 1.0, 1e-2, 1e-2, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0);
    vector<vector<double> > eye = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    {
        int n = 16;
        vector<vector<HPRReducedStateVector> > cells(n, vector<HPRReducedStateVector>(n));
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double r = std::sqrt(((i - (0.5 * n)) * (i - (0.5 * n))) + ((j - (0.5 * n)) * (j - (0.5 * n))));
                cells[i][j] = r <= 0.3 * n ? HPRReducedStateVector(0.999, 1.0, eye, 0.2, 0.0, 0.0, 0.02, 0.0, 0.0, 1.0, 0.5)
                                           : HPRReducedStateVector(0.001, 0.3, eye, -0.1, 0.0, 0.0, 0.0, 0.01, 0.0, 0.8, 0.25);
            }
        vector<vector<HPRReducedStateVector> > out =
            HPRSecondOrderSolver::solve2D(cells, 1.0 / n, 0.8, 1.0, 0.0, 2, 1, 2, hm1, hm2, 4);
        vector<double> v;
        for (int k = 0; k < 19; k++)
            for (auto& row : out)
                for (auto& c : row) v.push_back(c.computePrimitiveVariableVector(hm1, hm2)[k]);
        put(f, v);
    }
    // 14) HPRSecondOrderSolver::solve of the HPR intermediate two-material model: a shock tube with unequal material
    //     pressures, one relaxation sub-cycle, reinitialisation every 4 steps, to t = 0.02
    {
        int n = 60;
        vector<HPRIntermediateStateVector> cells(n);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n ? HPRIntermediateStateVector(0.999, eye, 0.2, 0.0, 0.0, 0.02, 0.0, 0.0, 1.0, 1.0, 0.5, 1.0)
                                    : HPRIntermediateStateVector(0.001, eye, -0.1, 0.0, 0.0, 0.0, 0.01, 0.0, 0.8, 0.3, 0.25, 0.36);
        vector<HPRIntermediateStateVector> out = HPRSecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.02, 0.0, 2, 1, 4, hm1, hm2);
        vector<double> v;
        for (int k = 0; k < 20; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector(hm1, hm2)[k]);
        put(f, v);
    }
    // 15) HPRSecondOrderSolver::solve of the HPR multiphysics two-material model (1D): a distortion and a heat flux per
    //     material, two sub-cycles (empty in the reference's loop for this model), to t = 0.015
    {
        int n = 60;
        vector<vector<double> > A2 = {{1.01, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 0.99}};
        vector<HPRMultiphysicsStateVector> cells(n);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n ? HPRMultiphysicsStateVector(0.999, 0.2, 0.0, 0.0, 1.0, 1.0, eye, 0.02, 0.0, 0.0, 0.5,
                                                                 1.1, A2, 0.01, 0.0, 0.0)
                                    : HPRMultiphysicsStateVector(0.001, -0.1, 0.0, 0.0, 0.8, 0.3, eye, 0.0, 0.01, 0.0,
                                                                 0.25, 0.33, A2, 0.0, 0.005, 0.0);
        vector<HPRMultiphysicsStateVector> out = HPRSecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.015, 0.0, 2, 2, 0, hm1, hm2);
        vector<double> v;
        for (int k = 0; k < 32; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector(hm1, hm2)[k]);
        put(f, v);
    }
    // 16) MHDSecondOrderSolver::solve of the MHD multiphysics two-material model (1D), MHDMultiphysicsTests::
    //     solveDumbserMultimaterialTest1's layout (gamma 1.4 | 1.67), to t = 0.05
    {
        int n = 80;
        vector<MHDMultiphysicsStateVector> cells(n);
        for (int i = 0; i < n; i++)
            cells[i] = MHDMultiphysicsStateVector(i <= 0.5 * n ? 0.999 : 0.001, 0.0, 0.0, 0.0, 1.0, 1.0, 0.75, 1.0, 0.0, 0.0,
                                                  0.125, 0.1, 0.75, -1.0, 0.0, 0.0);
        vector<MHDMultiphysicsStateVector> out = MHDSecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.05, 0.0, 0, 0, 0,
                                                                             MHDMaterialParameters(1.4),
                                                                             MHDMaterialParameters(1.67));
        vector<double> v;
        for (int k = 0; k < 16; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector()[k]);
        put(f, v);
    }
    // 17) HPRSecondOrderSolver::solve of the HPR intermediate two-material model with GodunovRomenski solids:
    //     HPRIntermediateTests::solveZhangTest's aluminium | copper and its deformation gradients (A = F^-1 on each
    //     side, each material at rho0 det A and the interface at the dominant material's cold pressure), one
    //     relaxation sub-cycle, reinitialisation every 3 steps, to t = 0.01
    {
        HPRMaterialParameters al("GodunovRomenski", false, false, 8.31445985, 2.71, 73.0, 300.0, 300.0, 9.0e-4, 1.0, 0.0,
                                 5.037, 1.0, 1.338, 0.0, 3.16, 1e8, 0.0, 0.0, 0.75, 0.0, 1.338, 2.0, 1.0, 3.577, 2.088);
        HPRMaterialParameters cu("GodunovRomenski", false, false, 8.31445985, 8.9, 0.0, 300.0, 300.0, 3.94e-4, 1.0, 0.0,
                                 3.909, 0.0, 0.0, 0.0, 2.1, 1e8, 0.0, 0.0, 0.75, 0.0, 1.0,
                                 8.9 * 3.909 * std::sqrt(4.0e-4 / 300.0), 1.0, 3.0, 2.0);
        vector<vector<double> > AL = {{1.0, 0.0, 0.0},
                                      {0.010175438596491228, 1.0526315789473684, -0.023391812865497075},
                                      {0.016666666666666666, 0.0, 1.1111111111111112}};
        vector<vector<double> > AR = {{1.0, 0.0, 0.0},
                                      {-0.015789473684210523, 1.0526315789473684, 0.0},
                                      {0.011111111111111112, 0.0, 1.1111111111111112}};
        int n = 60;
        vector<HPRIntermediateStateVector> cells(n);
        for (int i = 0; i < n; i++)
            cells[i] = i <= 0.5 * n
                           ? HPRIntermediateStateVector(0.999, AL, 2.0, 0.0, 0.1, 0.0, 0.0, 0.0, 3.1695906432748537,
                                                        15.950813993329472, 10.409356725146198, 15.950813993329472)
                           : HPRIntermediateStateVector(0.001, AR, 0.0, -0.03, -0.01, 0.0, 0.0, 0.0, 3.1695906432748537,
                                                        31.54939282442279, 10.409356725146198, 31.54939282442279);
        vector<HPRIntermediateStateVector> out = HPRSecondOrderSolver::solve(cells, 1.0 / n, 0.8, 0.01, 0.0, 2, 1, 3, al, cu);
        vector<double> v;
        for (int k = 0; k < 20; k++)
            for (auto& c : out) v.push_back(c.computePrimitiveVariableVector(al, cu)[k]);
        put(f, v);
    }
    double st = steps;
    std::fwrite(&st, sizeof(double), 1, f);
    std::fclose(f);
    return 0;
}
