/* vanguard_slic.h -- C ABI of the B200-native SLIC/FORCE finite-volume update.
 *
 * This is the drop-in boundary for Vanguard's single-material second-order solvers.  The reference
 * has no C ABI (its interface is static C++ methods, see each entry point below); callers reach this
 * ABI through the C++ shim in vanguard_b200/shim (same class names and signatures as the reference)
 * or directly through ctypes / any FFI.  No C++ or torch types cross this boundary: plain pointers,
 * sizes and status codes, no exceptions.
 *
 * Data layout at the boundary: structure-of-arrays PRIMITIVE planes, float64, in the reference's
 * primitive order, row-major (index = row * nx + column; X runs along the column index j, Y along
 * the row index i -- the reference's currentCells[i][j]):
 *   VG_MODEL_EULER (6 planes): rho, u, v, w, p, lambda           Euler/eulerstatevector.cpp:36-45
 *   VG_MODEL_MHD   (9 planes): rho, u, v, w, p, Bx, By, Bz, psi  MHD/mhdstatevector.cpp:35-47
 *   VG_MODEL_HPR  (17 planes): rho, p, A(9, row-major), u, v, w, Jx, Jy, Jz   HPR/hprstatevector.cpp:50-73
 *   VG_MODEL_EULER_REDUCED (7 planes): alpha1, u, v, w, rho1, rho2, p     the reduced two-material model,
 *                                      Euler/Multiphysics/eulerreducedstatevector.cpp:30-41 (w must be 0)
 *   VG_MODEL_EULER_MULTIPHYSICS (8 planes): alpha1, u, v, w, rho1, p1, rho2, p2   the multiphysics two-material
 *                                      model, Euler/Multiphysics/eulermultiphysicsstatevector.cpp:32-44 (w = 0)
 *   VG_MODEL_MHD_REDUCED (11 planes): alpha1, u, v, w, rho1, rho2, p, Bx, By, Bz, psi   the MHD reduced
 *                                      two-material model, MHD/Multiphysics/mhdreducedstatevector.cpp:91-111
 *   VG_MODEL_MHD_INTERMEDIATE (12 planes): alpha1, u, v, w, rho1, p1, rho2, p2, Bx, By, Bz, psi   the MHD
 *                                      intermediate two-material model, mhdintermediatestatevector.cpp:108-130
 *   VG_MODEL_HPR_REDUCED (19 planes): alpha1, p, A(9, row-major), u, v, w, Jx, Jy, Jz, rho1, rho2   the HPR
 *                                      reduced two-material model, HPR/Multiphysics/hprreducedstatevector.cpp:
 *                                      154-185 (VG_FP64 only)
 *   VG_MODEL_HPR_INTERMEDIATE (20 planes): alpha1, A(9, row-major), u, v, w, Jx, Jy, Jz, rho1, p1, rho2, p2   the
 *                                      HPR intermediate two-material model, HPR/Multiphysics/
 *                                      hprintermediatestatevector.cpp:161-193 (VG_FP64 only)
 *   VG_MODEL_HPR_MULTIPHYSICS (32 planes): alpha1, u, v, w, rho1, p1, A1(9), J1(3), rho2, p2, A2(9), J2(3)   the HPR
 *                                      multiphysics two-material model, HPR/Multiphysics/
 *                                      hprmultiphysicsstatevector.cpp:204-249 (VG_FP64 only; 1D: ny = 1; a cold
 *                                      material's J is taken and returned as 0)
 *   VG_MODEL_MHD_MULTIPHYSICS (16 planes): alpha1, u, v, w, rho1, p1, B1(3), psi1, rho2, p2, B2(3), psi2   the MHD
 *                                      multiphysics two-material model, MHD/Multiphysics/
 *                                      mhdmultiphysicsstatevector.cpp:135-163 (VG_FP64 only; 1D: ny = 1)
 * Ownership: a vg_solver owns all device memory it allocates; the caller owns every host buffer.
 * Threading: calls on different solvers are independent and re-entrant; one solver must not be used
 * from two host threads at once.  All work is enqueued on the stream given (NULL: the legacy default
 * stream) and the call returns after that stream has finished unless a function says otherwise.
 */
#ifndef VANGUARD_SLIC_H
#define VANGUARD_SLIC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vg_status {
    VG_OK = 0,
    VG_EINVAL = 1,       /* bad argument: null pointer, size, model, limiter, plane count */
    VG_ENAN = 2,         /* the run produced a non-finite value, a non-positive density, or a pressure at or
                          * below -p_inf (no real sound speed; 0 for ideal gases) */
    VG_ETIMEOUT = 3,     /* a bounded device-side wait gave up (the TMA-staged sweep): treat the CUDA context as
                          * lost (a copy may still be in flight), launch nothing more on it and reset the device */
    VG_ECUDA = 4,        /* a CUDA runtime call failed; vg_last_error_string() has the text */
    VG_ENOMEM = 5,       /* device allocation failed */
    VG_EUNSUPPORTED = 6  /* the input needs a variant this build does not provide (see below) */
} vg_status;

typedef enum vg_model {
    VG_MODEL_EULER = 0,
    VG_MODEL_MHD = 1,
    VG_MODEL_HPR = 2,
    VG_MODEL_EULER_REDUCED = 3,
    VG_MODEL_EULER_MULTIPHYSICS = 4,
    VG_MODEL_MHD_REDUCED = 5,
    VG_MODEL_MHD_INTERMEDIATE = 6,
    VG_MODEL_HPR_REDUCED = 7,
    VG_MODEL_HPR_INTERMEDIATE = 8,
    VG_MODEL_HPR_MULTIPHYSICS = 9,
    VG_MODEL_MHD_MULTIPHYSICS = 10
} vg_model;

/* VG_FP64: every operation in float64, in the reference's order, no FMA: matches the reference.
 * VG_MIXED: reconstruction, half-step evolution and FORCE flux in float32; pressure recovery, the CFL
 * reduction, source integration and the cell-update accumulation in float64. */
typedef enum vg_precision { VG_FP64 = 0, VG_MIXED = 1 } vg_precision;

/* VG_TRANSMISSIVE: the reference's mirror ghosts g[-1] = c[0], g[-2] = c[1] (Solvers/solvers.cpp:17-23).
 * VG_PERIODIC: wrap-around ghosts (the reference has none; its corner blocks stay default states). */
typedef enum vg_boundary { VG_TRANSMISSIVE = 0, VG_PERIODIC = 1 } vg_boundary;

/* SlopeLimiters::computeSlopeLimiter ids (Solvers/slopelimiters.cpp:60-74): 0 superbee, 1 van Leer,
 * any other value minbee. */
enum { VG_SUPERBEE = 0, VG_VANLEER = 1, VG_MINBEE = 2 };

#define VG_MAX_PARAMS 48

/* Material parameter blocks (params[] below):
 *   Euler: {gamma, p_inf, c_v, E0, T_ign, rate}   EulerMaterialParameters (Euler/eulermaterialparameters.h)
 *   MHD:   {gamma, p_inf, c_h}                    MHDMaterialParameters; c_h is recomputed every step by
 *                                                 vg_run as solve() does, and read from here by vg_sweep
 *   Euler reduced, multiphysics: {gamma1, p_inf1, gamma2, p_inf2}   the two materials' EulerMaterialParameters
 *   MHD reduced, intermediate: {gamma1, p_inf1, gamma2, p_inf2, c_h}   the two materials'
 *                                                 MHDMaterialParameters; c_h (both
 *                                                 materials) as MHD's: recomputed every step by the second-order
 *                                                 loop, read from here by the first-order loop and vg_sweep
 *   HPR:   {gamma, p_inf, c_v, rho0, T0, c_s, alpha, tau1, tau2, T_ref, p_ref, is_thermal,
 *           eos, Gamma0, c0, s, alpha_eos, is_plastic, sigma0, n}
 *                                                 HPRMaterialParameters (HPR/hprmaterialparameters.cpp:34-69):
 *                                                 eos 0 StiffenedGas, 1 ShockMieGruneisen (reference Grueneisen
 *                                                 coefficient Gamma0, reference sound speed c0, Hugoniot slope s,
 *                                                 with p_ref the reference pressure), 2 GodunovRomenski (c0 and
 *                                                 the exponent alpha_eos); is_plastic selects the plastic strain
 *                                                 relaxation with transition stress sigma0 and power-law index n
 *                                                 (HPR/hprsourceterms.cpp:12-23).
 *   MHD multiphysics: {gamma1, p_inf1, gamma2, p_inf2, c_h1, c_h2}   each material's c_h stays as given
 *   HPR reduced, intermediate, multiphysics: the HPR block above for each material, material k at params[20 k]
 *                (40 values): any equation of state, elastic or plastic
 * The last slot is reserved. */
typedef struct vg_grid_desc {
    int model;                        /* vg_model */
    int nx;                           /* cells along X (columns) */
    int ny;                           /* cells along Y (rows); 1 selects the 1D solver */
    int precision;                    /* vg_precision */
    int boundary;                     /* vg_boundary */
    int device;                       /* CUDA device ordinal */
    double params[VG_MAX_PARAMS];     /* material parameters, see above */
} vg_grid_desc;

typedef struct vg_run_config {
    double dx;          /* cellSpacing */
    double cfl;         /* CFLCoefficient */
    double t_end;       /* finalTime; <= 0: no end time (max_steps must then be > 0) */
    int max_steps;      /* > 0: stop after this many steps; <= 0: run until t_end */
    double bias;        /* slope-limiter bias omega */
    int limiter;        /* slopeLimiter id */
    int subcycles;      /* subcyclingIterations (source integration; HPR, the HPR two-material models, MHD and the
                         * MHD two-material models; second order only) */
    int order;          /* 2 (or 0): SecondOrderSolver's SLIC loop; 1: FirstOrderSolver's FORCE loop
                         * (Solvers/firstordersolver.cpp:435-553 and the MHD / HPR twins: 1-ghost boundary, FORCE
                         * of the cells themselves, no source, the MHD c_h kept at params[2], the MHD two-material
                         * models' at params[4]; both forms) */
    int stiff_source;   /* HPR only, no counterpart in the reference: 1 replaces the RK4 forcing sub-cycles by a
                         * stiff relaxation of dt/2 before and after the sweeps, cell by cell (distortion by implicit
                         * Euler on the eigenvalues of A^T A, heat flux by exponential sub-steps), stable at any tau;
                         * subcycles is then ignored.  Results approach the forcing's as its sub-cycles grow, not bit
                         * for bit. */
    int reinit_frequency;  /* two-material models: reinitialisationFrequency of (MHD, HPR)SecondOrderSolver::
                            * solve{,2D} (Solvers/secondordersolver.cpp:314-350, :354-385; Solvers/
                            * mhdsecondordersolver.cpp:445-495, :615-675; Solvers/hprsecondordersolver.cpp:402-500,
                            * :548-658): MultiphysicsSolvers::reinitialiseVolumeFraction after every
                            * reinit_frequency-th step; 0: never */
} vg_run_config;

typedef struct vg_solver vg_solver;

/* Create a solver for one grid.  Allocates device memory for two state buffers and a control block.
 * Replaces the allocation the reference does inside solve()/solve2D() (Solvers/secondordersolver.cpp:293). */
vg_status vg_create(const vg_grid_desc* desc, vg_solver** out);
vg_status vg_destroy(vg_solver* s);

/* Number of primitive planes the model takes at this boundary (6, 9, 17, 7, 8, 11, 12, 19, 20, 32, 16). */
int vg_model_nvar(int model);

/* Copy the state in / out.  planes: vg_model_nvar(model) planes of nx*ny float64, host or device
 * memory (is_device).  Upload returns VG_EUNSUPPORTED if the state uses fields the compiled variants
 * do not carry: Euler needs w == 0 and lambda == 1 in every cell; MHD needs w == 0 and Bz == 0 unless
 * the solver was created for the full 9-component variant (it chooses it automatically when they are
 * non-zero).  Where those checks do not decide the variant they run on host threads while the copies are in
 * flight; a failed upload leaves the solver without a state until the next successful one. */
vg_status vg_upload_primitive(vg_solver* s, const double* planes, int is_device, void* stream);
vg_status vg_download_primitive(vg_solver* s, double* planes, int is_device, void* stream);

/* The time loop of SecondOrderSolver::solve / solve2D (Solvers/secondordersolver.cpp:288-314, :392-424)
 * and its MHD/HPR counterparts, on the uploaded state, entirely on the device: CFL maximum, dt schedule
 * (x0.2 for the first six steps, clamp to t_end; Solvers/solvers.cpp:437-452), X(dt/2) Y(dt) X(dt/2)
 * sweeps in 2D, one sweep in 1D.  The loop is replayed from captured CUDA graphs; dt never returns to
 * the host.  A plain second-order exact-FP64 Euler run of a 1D row of 16 .. 2032 cells runs instead as one kernel
 * launch (the whole loop inside one thread-block cluster), with the same results; a run there that stops advancing
 * ends after 2^22 steps with VG_EINVAL.  steps_taken / t_reached may be NULL. */
vg_status vg_run(vg_solver* s, const vg_run_config* cfg, int* steps_taken, double* t_reached, void* stream);

/* Host-buffer convenience: upload, vg_run, download (the reference's solve(): copy in, return by value). */
vg_status vg_solve(vg_solver* s, const double* planes_in, double* planes_out, const vg_run_config* cfg,
                   int* steps_taken, double* t_reached, void* stream);

/* One sweep of compute{X,Y}SLICTimeStep2D (Solvers/secondordersolver.cpp:140-162, :214-236) or of the
 * 1D computeSLICTimeStep (:80-98) with a host-given time step, in place on the uploaded state.
 * axis: 0 = X, 1 = Y.  Enqueued asynchronously on `stream`. */
vg_status vg_sweep(vg_solver* s, int axis, double dx, double dt, double bias, int limiter, void* stream);

/* Solvers::computeMaximumWaveSpeed{,2D} over the ghosted grid (Solvers/solvers.cpp:259-339; MHD
 * Solvers/mhdsolvers.cpp:286-388), including the default-state corner ghosts in 2D. */
vg_status vg_max_wave_speed(vg_solver* s, double* out, void* stream);

/* The helper itself, Solvers::computeMaximumWaveSpeed2D (Solvers/solvers.cpp:318-339): the maximum over
 * exactly the uploaded cells, without adding the default-state corners.  A caller that uploads the
 * reference's ghosted array (corners included) gets the reference's value; one that uploads interior cells
 * only gets the maximum over those.  Equal to vg_max_wave_speed on 1D grids. */
vg_status vg_max_wave_speed_cells(vg_solver* s, double* out, void* stream);

/* Device pointer of plane 0 of the current state buffer and the plane/row strides in elements, so a
 * caller can read or write the resident state without a host round trip.  The carried planes are the
 * non-trivial subset (Euler: rho, u, [v], p; MHD: rho, u, v, [w], p, Bx, By, [Bz], psi). */
vg_status vg_state_device(vg_solver* s, double** plane0, long* plane_stride, long* row_stride, int* nplanes);

/* Number of CUDA kernels the last vg_run/vg_sweep/vg_max_wave_speed call launched (graph nodes count). */
long vg_last_launch_count(vg_solver* s);

/* Launch configurations of the sweeps.  No counterpart in the reference (its sweeps are OpenMP loops).
 * Each model and precision is compiled for VG_NUM_XCFG X-sweep tile shapes (cells per segment, segments
 * per block, register cap) and VG_NUM_YCFG Y-sweep tile shapes (columns per block, rows marched per
 * thread, register cap).  Each Y shape runs either with its own rows per thread or with row segments sized so
 * that its blocks fill whole waves of the device's resident slots; the tuner times both and keeps the faster
 * (a Y configuration's reported time is the better of the two).  The tile shape never changes a cell's
 * arithmetic, so every configuration gives identical results.
 * vg_autotune times every candidate on the uploaded state (`reps` launches each, CUDA events on `stream`),
 * keeps the fastest per axis and caches it (with the schedule below) by (variant, precision, boundary, nx,
 * ny, SM count) in
 * process memory and, when the environment variable VG_TUNE_CACHE names a file, on disk.  With
 * times_ms == NULL a cached choice is applied without timing; otherwise times_ms receives
 * VG_NUM_XCFG + VG_NUM_YCFG + VG_NUM_SCHED averages (X configurations, Y configurations, then the step's tail
 * under each schedule below, fused first).
 * The tuner also picks the step's schedule: where the next step's CFL maximum (Solvers/solvers.cpp:413-452) is
 * taken.  0 folds it into the last X sweep's epilogue (no extra pass over the state, but the wave speed's
 * registers ride in the sweep); 1 runs a separate reduction after the step (one more read of the state, a
 * leaner sweep).  The reference's split order X(dt/2) Y(dt) X(dt/2) itself is fixed: it defines the results.
 * Both schedules give identical results.  Runs with a source pass or a reinitialisation after the sweeps
 * always take the separate reduction.  vg_set_schedule / vg_get_schedule set and read it directly. */
#define VG_NUM_XCFG 5
#define VG_NUM_YCFG 6
#define VG_NUM_SCHED 2
vg_status vg_autotune(vg_solver* s, const vg_run_config* cfg, int reps, float* times_ms, void* stream);
vg_status vg_set_launch_config(vg_solver* s, int xcfg, int ycfg);
vg_status vg_get_launch_config(vg_solver* s, int* xcfg, int* ycfg, const char** xname, const char** yname);
vg_status vg_set_schedule(vg_solver* s, int cfl_separate);
vg_status vg_get_schedule(vg_solver* s, int* cfl_separate);

/* ---- Ragged batches of independent 1D Euler problems.  No counterpart in the reference, whose scenario drivers
 * call SecondOrderSolver::solve (Solvers/secondordersolver.cpp:288-314) once per problem; a batch runs that same
 * per-problem loop for many problems at once, each instance bit-equal to its own solve().
 * Instance k has ncell[k] >= 2 cells of width dx[k], adiabatic index gamma[k] and stiffening p_inf[k] (p_inf may be
 * NULL: 0), transmissive boundaries.  State planes at this boundary are the 6 Euler primitive planes of all
 * instances concatenated in instance order (total = sum of ncell), with v == w == 0 and lambda == 1.
 * vg_batch_run advances every instance by `steps` steps, each with its own dt_k = CFL dx_k / S_k (x0.2 for the
 * first six steps) computed on the device; the whole loop is one captured CUDA graph of one persistent kernel
 * per step.  dt_last (nullable, ninst entries) receives each instance's last time step. */
typedef struct vg_batch vg_batch;
vg_status vg_batch_create(int ninst, const int* ncell, const double* dx, const double* gamma, const double* p_inf,
                          int device, vg_batch** out);
vg_status vg_batch_destroy(vg_batch* b);
long vg_batch_total_cells(vg_batch* b);
vg_status vg_batch_upload(vg_batch* b, const double* planes, int is_device, void* stream);
vg_status vg_batch_download(vg_batch* b, double* planes, int is_device, void* stream);
vg_status vg_batch_run(vg_batch* b, double cfl, int steps, double bias, int limiter, double* dt_last, void* stream);
long vg_batch_last_launch_count(vg_batch* b);

/* No counterpart in the reference (it has no derivatives): the discrete adjoint of vg_batch_run.
 * Loss L = sum over all cells of all instances of (rho(T) - target_rho)^2 after `steps` steps of vg_batch_run
 * (same cfl, bias, limiter) from the batch's current state.  Returns L, dL/d(initial primitives) in the 6-plane
 * layout (rho, u, p planes filled; v, w, lambda planes 0: held fixed) and dL/dgamma per instance.  The dt of
 * every step depends on the state through the CFL maximum and that dependence is differentiated (the first cell
 * attaining the maximum carries it).  Non-smooth points take the derivative of the branch the forward step took.
 * `checkpoints` >= 1 state slots on the device (slot 0 holds the initial state; capped at `steps`) bound the
 * memory to (checkpoints + 3) states; steps are recomputed on Griewank's binomial schedule, so checkpoints ==
 * steps stores every state and recomputes nothing.  forward_steps / adjoint_steps (nullable) receive the number
 * of forward steps advanced (recomputation and the final step included) and of reversed steps.  The batch keeps
 * its initial state.  target_rho (total), grad_planes (6 x total, nullable) and grad_gamma (ninst, nullable) are
 * host arrays, or device arrays when is_device != 0; loss (nullable) is a host scalar.  Returns when done. */
vg_status vg_batch_gradient(vg_batch* b, const double* target_rho, double cfl, int steps, double bias, int limiter,
                            int checkpoints, double* loss, double* grad_planes, double* grad_gamma, int is_device,
                            long* forward_steps, long* adjoint_steps, void* stream);

/* ---- Homogeneous HPR relaxation batches and their discrete adjoint.  No counterpart in the reference (it has no
 * batches and no derivatives); each step is the reference's own source step on a spatially uniform field: one
 * sub-cycle of HPRForcingSolver's RK4 (Solvers/hprforcingsolver.cpp:332-357, the source terms of
 * HPRStateVector::computeSourceTermVector, HPR/hprstatevector.cpp:312-366, and HPRSourceTerms,
 * HPR/hprsourceterms.cpp:7-39) with zero limiter bias, where the fractional flux predictor reduces to its
 * primitive round trip; steps equal that forcing bit for bit up to pow's last place.  A batch holds `ncell`
 * independent cells of one HPR material (params: the HPR block of vg_grid_desc; StiffenedGas equation of state and
 * elastic strain relaxation only) with relaxation times tau1, tau2 per cell.
 * Planes at this boundary: the 17 HPR primitive planes of all cells (17 x ncell, HPR/hprstatevector.cpp:50-73);
 * tau: 2 x ncell (all tau1, then all tau2), or NULL for the params' tau1 and tau2 in every cell.
 * vg_source_batch_run advances the batch's state by `steps` steps of length h.
 * vg_source_batch_gradient is the adjoint of vg_source_batch_run(h, steps) from the batch's current state, which
 * it leaves unchanged: given the cotangent dL/dW(T) (17 x ncell) of any loss of the final primitives, it returns
 * dL/dW(0) (17 x ncell, nullable) and dL/dtau (2 x ncell, nullable).  The source is smooth where det A > 0, so no
 * subgradient choice arises; the primitive round trips are identities of exact arithmetic and are differentiated
 * as such; a non-thermal material's J passes through unchanged.  `checkpoints` >= 1 state slots per cell (slot 0
 * the initial state; capped at steps) bound the memory to (checkpoints + 1) states; steps are recomputed on
 * Griewank's binomial schedule (checkpoints == steps stores every state).  forward_steps / adjoint_steps
 * (nullable) receive the forward steps advanced (recomputation included) and the steps reversed.  Host or device
 * arrays per is_device; returns when done. */
typedef struct vg_source_batch vg_source_batch;
vg_status vg_source_batch_create(int ncell, const double* params, int device, vg_source_batch** out);
vg_status vg_source_batch_destroy(vg_source_batch* b);
vg_status vg_source_batch_upload(vg_source_batch* b, const double* planes, const double* tau, int is_device,
                                 void* stream);
vg_status vg_source_batch_download(vg_source_batch* b, double* planes, int is_device, void* stream);
vg_status vg_source_batch_run(vg_source_batch* b, double h, int steps, void* stream);
vg_status vg_source_batch_gradient(vg_source_batch* b, const double* cotangent, double h, int steps, int checkpoints,
                                   double* grad_planes, double* grad_tau, int is_device, long* forward_steps,
                                   long* adjoint_steps, void* stream);

/* Rows accepted by vg_max_wave_speed_noalloc: the size of its static scratch array (8 bytes per row,
 * 512 KiB, held on every GPU that loads the library until the process exits). */
#define VG_NOALLOC_MAX_ROWS 65536

/* No counterpart in the reference: an allocation-free variant of vg_max_wave_speed for callers that may
 * not allocate device memory themselves or let a library do so (applications that own all device memory
 * through their own pool allocator, where cudaMalloc/cudaFree would escape the pool's budget and
 * cudaFree would synchronise the device under their other streams).  Computes the maximum wave speed
 * of the padded grid exactly as vg_max_wave_speed does, from a state the caller already holds in device
 * memory: `planes` = the model's reference-order primitive planes (Euler 6, MHD 9) with the given plane
 * and row strides (elements; rows may be padded, row_stride >= nx, plane_stride >= row_stride * ny),
 * `params` = the model's parameter block (gamma, p_inf first) in HOST memory (read on the host before the
 * launch), `out` = a device pointer to one double.  Calls neither cudaMalloc nor cudaFree: per-row partial
 * maxima go to a file-scope __device__ array of VG_NOALLOC_MAX_ROWS doubles, so ny > VG_NOALLOC_MAX_ROWS
 * returns VG_EINVAL.  Uses the current device.  Every call looks up the array's device address in the
 * current context (cudaGetSymbolAddress, which allocates nothing); the first call on a device may load the
 * library's device code there, so make that first call before any stream capture.  Enqueued asynchronously
 * on `stream`.  All calls on a device share the array, so calls that may overlap on the GPU (different
 * streams without ordering between them) race and must be serialised by the caller. */
vg_status vg_max_wave_speed_noalloc(int model, const double* planes, long plane_stride, long row_stride, int nx,
                                    int ny, const double* params, double* out, void* stream);

/* Text of the last error on this thread. */
const char* vg_last_error_string(void);
const char* vg_status_string(vg_status st);

#ifdef __cplusplus
}
#endif
#endif /* VANGUARD_SLIC_H */
