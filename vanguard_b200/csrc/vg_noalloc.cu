// Allocation-free entry point: CFL maximum wave speed of a caller-owned device state.
//
// Some host applications own every byte of device memory through their own pool allocator and do not
// let a library call cudaMalloc or cudaFree: cudaFree synchronises the whole device and stalls the
// application's other streams, and a foreign allocation escapes the pool's accounting and memory budget.
// vg_max_wave_speed needs a vg_solver, whose creation allocates; this entry point computes the same value
// from device planes the caller already holds, and uses a fixed scratch array that is part of the library
// image instead of allocated memory.
//
// Compiled with -fmad=false like the FP64 sweeps: it reuses their exact wave-speed functions, so the
// result equals vg_max_wave_speed bit for bit.
#include <cuda_runtime.h>

#include <string>

#include "../../include/vanguard_slic.h"
#include "physics_fp64.cuh"
#include "vg_ops.h"

namespace {

// Per-row partial maxima of one call.  Every GPU that loads the library holds this array (512 KiB)
// until the process exits.  All calls on a device share it: a call writes slots [0, ny) before reading
// them, so nothing needs to start at zero, and calls that overlap on the GPU (different streams, no
// ordering between them) race on it.
__device__ __align__(256) double g_row_max[VG_NOALLOC_MAX_ROWS];

vg_status noalloc_fail(vg_status st, const std::string& msg) {
    vg::set_last_error(msg);
    return st;
}

// Reference plane of each wave-speed input (Euler: rho, u, v, p; MHD: all nine).
struct PlaneMap {
    int idx[9];
};

// Row maxima.  Reads the reference-order primitive planes directly (Euler: rho, u, v, w, p, lambda;
// MHD: rho, u, v, w, p, Bx, By, Bz, psi) and skips non-finite speeds like the reference's
// `if (waveSpeed > maximumWaveSpeed)` loop (Solvers/solvers.cpp:264-273).
template <class M, int NT>
__global__ void __launch_bounds__(NT) row_max_kernel(const double* __restrict__ planes, long plane, long pitch, int nx,
                                                     int dims, vg::SweepArgs a, PlaneMap map,
                                                     double* __restrict__ scratch) {
    const int row = blockIdx.x;
    const typename M::P q = M::params(a.params, 0.0);
    double best = 0.0;
    for (int c = threadIdx.x; c < nx; c += NT) {
        double W[M::NW];
#pragma unroll
        for (int v = 0; v < M::NW; v++) W[v] = planes[(long)map.idx[v] * plane + (long)row * pitch + c];
        double s = M::wave(W, q, dims);
        if (s > best) best = s;
    }
    __shared__ double red[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, best, o);
        best = (w > best) ? w : best;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < NT / 32; w++) m = (red[w] > m) ? red[w] : m;
        scratch[row] = m;
    }
}

// Reduce the row maxima, fold in the default-constructed corner ghosts of the 2D padded grid
// (Solvers/solvers.cpp:92) and write the result to the caller's output.
template <class M, int NT>
__global__ void __launch_bounds__(NT) row_max_finish_kernel(const double* __restrict__ scratch, int ny, int dims,
                                                            vg::SweepArgs a, double* __restrict__ out) {
    double best = 0.0;
    for (int r = threadIdx.x; r < ny; r += NT) best = (scratch[r] > best) ? scratch[r] : best;
    __shared__ double red[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, best, o);
        best = (w > best) ? w : best;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < NT / 32; w++) m = (red[w] > m) ? red[w] : m;
        if (dims == 2) {
            double W[M::NW];
            M::default_state(W);
            const typename M::P q = M::params(a.params, 0.0);
            double sd = M::wave(W, q, 2);
            if (sd > m) m = sd;
        }
        *out = m;
    }
}

// Device address of the scratch array in the current device's context.  Looked up on every call: the lookup is a
// host-side table query that allocates nothing, and a cached address would outlive the module it points into if the
// host reset the device (cudaDeviceReset) between calls.  The first lookup on a device may load the library's device
// code into that context, which is why the first call must come before any stream capture.
vg_status scratch_for_current_device(double** out) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_row_max);
    if (e != cudaSuccess) return noalloc_fail(VG_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = p;
    return VG_OK;
}

template <class M>
vg_status launch(const double* planes, long plane, long pitch, int nx, int ny, const vg::SweepArgs& a,
                 PlaneMap map, double* scratch, double* out, cudaStream_t st) {
    const int dims = ny > 1 ? 2 : 1;
    row_max_kernel<M, 256><<<ny, 256, 0, st>>>(planes, plane, pitch, nx, dims, a, map, scratch);
    row_max_finish_kernel<M, 1024><<<1, 1024, 0, st>>>(scratch, ny, dims, a, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(VG_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return VG_OK;
}

}  // namespace

extern "C" vg_status vg_max_wave_speed_noalloc(int model, const double* planes, long plane_stride, long row_stride,
                                                int nx, int ny, const double* params, double* out, void* stream) {
    if (!planes || !params || !out) return noalloc_fail(VG_EINVAL, "null argument");
    if (model != VG_MODEL_EULER && model != VG_MODEL_MHD)
        return noalloc_fail(VG_EUNSUPPORTED, "vg_max_wave_speed_noalloc supports the Euler and MHD models");
    if (nx < 1 || ny < 1) return noalloc_fail(VG_EINVAL, "empty grid");
    if (ny > VG_NOALLOC_MAX_ROWS)
        return noalloc_fail(VG_EINVAL, "ny = " + std::to_string(ny) + " rows exceeds VG_NOALLOC_MAX_ROWS = " +
                                           std::to_string(VG_NOALLOC_MAX_ROWS) + " (size of the static scratch array)");
    if (row_stride < nx || plane_stride < row_stride * (long)ny)
        return noalloc_fail(VG_EINVAL, "row_stride must be >= nx and plane_stride >= row_stride * ny");
    double* scratch = nullptr;
    vg_status st = scratch_for_current_device(&scratch);
    if (st != VG_OK) return st;
    const PlaneMap euler_map = {{0, 1, 2, 4}}, mhd_map = {{0, 1, 2, 3, 4, 5, 6, 7, 8}};
    vg::SweepArgs a{};
    a.params[0] = params[0];  // gamma
    a.params[1] = params[1];  // p_inf
    cudaStream_t s = (cudaStream_t)stream;
    if (model == VG_MODEL_EULER)
        return launch<vg::EulerF64<2>>(planes, plane_stride, row_stride, nx, ny, a, euler_map, scratch, out, s);
    return launch<vg::MHDF64<true>>(planes, plane_stride, row_stride, nx, ny, a, mhd_map, scratch, out, s);
}
