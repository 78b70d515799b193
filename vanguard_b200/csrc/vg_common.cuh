// Shared device-side definitions of the SLIC/FORCE kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vg {

// Per-run control block in device memory.  The time loop runs entirely on the device: step_begin
// turns the previous step's wave-speed maximum into dt, the sweeps read dt, the last sweep of a step
// accumulates the next maximum and advances t / it.
struct Ctrl {
    double t;                        // time reached
    double dt;                       // this step's time step
    double t_end;                    // finalTime (1e300 for step-count runs)
    double cfl;                      // CFLCoefficient
    double dx;                       // cellSpacing
    double ch;                       // MHD GLM speed c_h of this step (= padded-grid maximum wave speed)
    unsigned long long smax_next;    // bit pattern of the running maximum wave speed (>= 0 doubles order as integers)
    int it;                          // steps taken
    int max_steps;                   // stop after this many steps
    int active;                      // 1 while the current step runs (t < t_end and it < max_steps)
    unsigned int err;                // bit 0: non-finite or non-positive density / pressure written
    int dims;                        // 1 or 2
    int pad;
    // sweep constants of this step, computed once by step_begin for the two sweep lengths dt/2 (slot 0) and
    // dt (slot 1): ts / dx, dx / ts, 0.5 * (ts / dx), and their float roundings
    double kr[2], krinv[2], khalf_r[2];
    float kr_f[2], krinv_f[2], khalf_r_f[2];
};

enum : unsigned int { ERR_STATE = 1u, ERR_TIMEOUT = 2u };  // bits of Ctrl::err

// Ghost-cell index along one axis of length n with 2 ghost cells per side (k in [-2, n+1]):
// transmissive mirror g[-1] = c[0], g[-2] = c[1], g[n] = c[n-1], g[n+1] = c[n-2] (Solvers/solvers.cpp:17-23)
// or periodic wrap-around.  Indices outside [-2, n+1] only occur in the unused halo of a partial tile and
// are clamped so every load stays in bounds.
__device__ __forceinline__ int ghost_index(int k, int n, int periodic) {
    if (k >= 0 && k < n) return k;
    if (k < -2) return 0;
    if (k > n + 1) return n - 1;
    if (periodic) return (k < 0) ? k + n : k - n;
    return (k < 0) ? (-1 - k) : (2 * n - 1 - k);
}

// std::min / std::max tie behaviour (min(a,b) = b < a ? b : a).
__device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ float std_minf(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float std_maxf(float a, float b) { return (a < b) ? b : a; }

// Kernel-wide constants of one sweep.
struct SweepConst {
    double r;        // timeStep / cellSpacing
    double rinv;     // cellSpacing / timeStep
    double half_r;   // 0.5 * (timeStep / cellSpacing)    (Solvers/solvers.cpp:606-609)
    double cm;       // 0.5 * (1 + bias)
    double cp;       // 0.5 * (1 - bias)
    double bias;
    double floor5;   // pow(10.0, -5.0), computed on the host with the same libm call as the reference
    int limiter;
};

constexpr int kParams = 48;           // VG_MAX_PARAMS
constexpr int kTmaTile = 128;         // threads (cells per row, halo included: kTmaTile + 2) of the TMA X sweep
constexpr int kInvGm1 = kParams - 1;  // slot the host fills with 1 / (gamma - 1)

// Launch-independent description of one sweep.
struct SweepArgs {
    const double* in;        // plane 0 of the input state
    double* out;             // plane 0 of the output state
    long plane;              // plane stride (elements)
    long pitch;              // row stride (elements)
    int nx, ny;              // grid size
    int periodic;            // boundary kind
    Ctrl* ctrl;              // device control block, or null for a host-given dt
    double dt_host;          // time step when ctrl == null
    double dt_scale;         // 0.5 for the X half sweeps of a 2D step, else 1
    int kslot;               // ctrl->kr[] slot of dt_scale (0: 0.5, 1: 1.0)
    double r_host, rinv_host, half_r_host;  // the same constants for ctrl == null (set by the host)
    float r_host_f, rinv_host_f, half_r_host_f;
    double ch_host;          // MHD c_h when ctrl == null
    double dx;
    double bias;
    double floor5;
    int limiter;
    int accumulate_wave;     // fold max wave speed of the output into *wave_acc
    int advance_time;        // last sweep of a step: ctrl->t += dt, ctrl->it += 1
    int dims;                // 1 or 2 (selects the wave-speed formula)
    int ch_fixed;            // step_begin keeps ctrl->ch = ch_host instead of this step's maximum (first order)
    unsigned long long* wave_acc;  // running maximum (bit pattern), usually &ctrl->smax_next
    unsigned int* err;             // error word (always valid)
    double* aux;                   // model scratch planes (HPR forcing neighbours), or null
    double params[kParams];  // model parameters (model-specific layout); params[kInvGm1] = 1 / (params[0] - 1)
    // device CUtensorMap over `in` for the TMA-staged X sweep (null: none); kept last, since a field ahead of
    // params[] changed the register allocation of the two-row X sweep (56 -> 60)
    const void* tmap;
    int reinit_freq;  // volume-fraction reinitialisation every reinit_freq steps (Euler reduced model; 0: none)
    int ty_rows;      // rows marched per Y-sweep block (0: the shape's TY), set by launch_y
    int y_waves;      // launch_y sizes the Y segments for whole waves of resident blocks (else the shape's TY)
};

// Sweep constants of one sweep of length ts = dt * scale, formed as the reference forms them
// (Solvers/solvers.cpp:606-609, Solvers/firstordersolver.cpp:79-85): one place for the device and the host.
__host__ __device__ __forceinline__ void sweep_scale(double ts, double dx, double& r, double& rinv, double& half_r) {
    r = ts / dx;
    rinv = dx / ts;
    half_r = 0.5 * (ts / dx);
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double v) {
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// Block-wide max of non-negative doubles into *acc; call from all threads of the block.
template <int NT>
__device__ __forceinline__ void block_max_to(double v, unsigned long long* acc) {
    __shared__ double red[32];
    const unsigned full = 0xffffffffu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(full, v, o);
        v = (w > v) ? w : v;
    }
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        constexpr int NWARP = (NT + 31) / 32;
        v = (lane < NWARP) ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double w = __shfl_xor_sync(full, v, o);
            v = (w > v) ? w : v;
        }
        if (lane == 0 && v > 0.0) atomic_max_nonneg(acc, v);
    }
}

}  // namespace vg
