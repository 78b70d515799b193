/* CPU restatement of Vanguard's single-material SLIC/FORCE path (test infrastructure only).
 *
 * This is the checker the CUDA path is compared against.  It is a plain-C restatement of the
 * reference's algorithm with the reference's floating-point operation order, so that on x86-64 (no
 * FMA contraction, -ffp-contract=off) it reproduces the reference bit for bit; it is itself pinned
 * against the compiled reference (oracle/_ref/libvgref.so) and against committed golden vectors.
 * Only tests/, bench.py's CPU baseline leg and __graft_entry__.smoke() may load it; the product path
 * never calls it.
 *
 * Layout: structure-of-arrays PRIMITIVE planes in the reference's primitive order, row-major
 * (index = row * nx + column; X runs along the column index, Y along the row index):
 *   Euler (6):  rho, u, v, w, p, lambda                 Euler/eulerstatevector.cpp:36-45
 *   MHD   (9):  rho, u, v, w, p, Bx, By, Bz, psi        MHD/mhdstatevector.cpp:35-47
 *   HPR  (17):  rho, p, A(9 row-major), u, v, w, Jx, Jy, Jz   HPR/hprstatevector.cpp:50-73
 *   Euler reduced (8): alpha1, u, v, w, rho1, rho2, p, unused  Euler/Multiphysics/eulerreducedstatevector.cpp:30-41
 *   Euler multiphysics (9): alpha1, u, v, w, rho1, p1, rho2, p2, unused  .../eulermultiphysicsstatevector.cpp:32-44
 */
#ifndef VANGUARD_SLIC_ORACLE_H
#define VANGUARD_SLIC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { VO_EULER = 0, VO_MHD = 1, VO_HPR = 2, VO_EULER_REDUCED = 3, VO_EULER_MULTIPHYSICS = 4, VO_MHD_REDUCED = 5, VO_MHD_INTERMEDIATE = 6,
       VO_HPR_REDUCED = 7, VO_HPR_INTERMEDIATE = 8,
       VO_HPR_MULTIPHYSICS = 9, VO_MHD_MULTIPHYSICS = 10 };
enum { VO_BC_TRANSMISSIVE = 0, VO_BC_PERIODIC = 1 };

/* Number of primitive planes of a model (6, 9, 17). */
int vo_nvar(int model);

/* Length of the parameter block each model takes:
 *   Euler: {gamma, p_inf, c_v, E0, T_ign, reaction_rate}     (Euler/eulermaterialparameters.cpp:36-46)
 *   MHD:   {gamma, p_inf, c_h}   c_h is only read by vo_sweep*; vo_run* sets it every step
 *   HPR:   20 values, see slic_oracle.c; trailing zeros select StiffenedGas, non-plastic      */
int vo_nparams(int model);

/* Fixed-step or time-driven run of solve()/solve2D()'s loop (max_steps <= 0: run until t_end;
 * t_end <= 0: no end time).  Returns the time reached, *steps_out = steps taken, dt_log (nullable,
 * max_steps entries) receives each step's dt.  subcycles > 0 is only defined for the HPR model
 * (RK4 relaxation source around the sweeps, Solvers/hprsecondordersolver.cpp:514-541). */
double vo_run1d(int model, double* planes, int n, double dx, double cfl, double t_end, int max_steps,
                double bias, int limiter, const double* prm, int bc, int subcycles, int* steps_out,
                double* dt_log);
double vo_run2d(int model, double* planes, int nx, int ny, double dx, double cfl, double t_end,
                int max_steps, double bias, int limiter, const double* prm, int bc, int subcycles,
                int* steps_out, double* dt_log);

/* One SLIC sweep (axis 0: X, 1: Y) of length dt over the whole grid, in place. */
void vo_sweep1d(int model, double* planes, int n, double dx, double dt, double bias, int limiter,
                const double* prm, int bc);
void vo_sweep2d(int model, double* planes, int nx, int ny, int axis, double dx, double dt, double bias,
                int limiter, const double* prm, int bc);

/* Maximum wave speed over the ghosted grid, as computeMaximumWaveSpeed{,2D} sees it. */
double vo_max_wave1d(int model, const double* planes, int n, const double* prm);
double vo_max_wave2d(int model, const double* planes, int nx, int ny, const double* prm);

/* One sub-cycle of the HPR RK4 relaxation-source solver over the grid (HPRForcingSolver::
 * computeRungeKuttaTimeStep{,2D}, Solvers/hprforcingsolver.cpp:341-357, :394-418), in place. */
void vo_forcing(int model, double* planes, int nx, int ny, double dx, double dt, double bias, int limiter,
                const double* prm, int bc);

/* SecondOrderSolver::solve{,2D} of the Euler two-material models, id VO_EULER_REDUCED (8 planes: alpha1, u, v, w, rho1,
 * rho2, p, unused) or VO_EULER_MULTIPHYSICS (9 planes: alpha1, u, v, w, rho1, p1, rho2, p2, unused), prm = {gamma1,
 * p_inf1, gamma2, p_inf2}; reinit_freq > 0 reinitialises the volume fraction every reinit_freq steps
 * (MultiphysicsSolvers::reinitialiseVolumeFraction). */
/* MHDSecondOrderSolver::solve{,2D} of the MHD two-material models, id VO_MHD_REDUCED (12 planes: alpha1, u, v, w, rho1,
 * rho2, p, Bx, By, Bz, psi, unused) or VO_MHD_INTERMEDIATE (13 planes: alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz,
 * psi, unused), prm = {gamma1, p_inf1, gamma2, p_inf2, c_h (set every step)}: RK4 GLM damping sub-cycles around the
 * sweeps and the volume-fraction reinitialisation every reinit_freq steps. */
double vo_run_mhd_two_material(int id, double* planes, int nx, int ny, double dx, double cfl, double t_end,
                                int max_steps, double w, int lim, const double* prm, int bc, int subcycles,
                                int reinit_freq, int* steps_out);
double vo_run_two_material(int id, double* planes, int nx, int ny, double dx, double cfl, double t_end, int max_steps,
                           double w, int lim, const double* prm, int bc, int reinit_freq, int* steps_out);

/* HPR Mie-Grueneisen probe (HPR/hprmiegruneisen.cpp), 13 values per point k:
 *   Gamma, p_ref(rho), e_ref(rho), dGamma, dp_ref, de_ref, e(rho, p), p(rho, e), T(rho, p), de/drho(rho, p),
 *   de/dp, dT/drho(rho, p), dT/dp. */
void vo_hpr_eos(const double* prm, const double* rho, const double* p, const double* e, int n, double* out);
/* HPRSourceTerms::computeTheta1Reciprocal of density rho[k] and distortion a9[9k..9k+8] (row-major). */
void vo_hpr_theta1(const double* prm, const double* rho, const double* a9, int n, double* out);

/* HPR single-cell probe: conserved vector, x/y fluxes, source and acoustic-tensor speeds of primitives w. */
void vo_hpr_cell(const double* w, const double* prm, double* u, double* fx, double* fy, double* src, double* speed_xy);

/* Single-interface building blocks, exposed for unit tests of the device functions. */
double vo_slope_limiter(double r, double bias, int limiter);
void vo_prim_to_cons(int model, const double* w, const double* prm, double* u);
void vo_cons_to_prim(int model, const double* u, const double* prm, double* w);
void vo_flux(int model, const double* u, int axis, const double* prm, double* f);
void vo_slic_flux(int model, const double* wLL, const double* wL, const double* wR, const double* wRR,
                  int axis, double dx, double dt, double bias, int limiter, const double* prm, double* f);

/* FirstOrderSolver::solve{,2D} and the MHD / HPR twins (ny == 1: 1D); the MHD c_h stays prm[2]. */
double vo_run_first_order(int model, double* planes, int nx, int ny, double dx, double cfl, double t_end,
                          int max_steps, const double* prm, int bc, int* steps_out);

#ifdef __cplusplus
}
#endif
#endif
