// Ragged batches of independent 1D Euler problems in one persistent launch per time step.
//
// Instances k = 0..K-1 have n_k cells (any sizes), their own gamma / p_inf and cell width dx_k, and are
// concatenated into structure-of-arrays planes (rho, u, p) with a cell-offset table.  The work is cut into
// tiles of BP - 2 consecutive cells of one instance; a persistent grid strides over the tile table, so no block
// straddles two instances and the transmissive ghosts of each instance are synthesised by the loader exactly as
// Solvers::insertBoundaryCells builds them (Solvers/solvers.cpp:7-32).  Every instance takes its own time step
// dt_k = CFL * dx_k / S_k (x0.2 for the first six steps, Solvers/solvers.cpp:437-452) from its own maximum wave
// speed S_k, kept on the device in a three-slot ring: step s reads slot s % 3, accumulates the next maximum into
// (s + 1) % 3 in the update epilogue and clears (s + 2) % 3.  The last block to finish a step advances the step
// counter, so one kernel per step and a captured CUDA graph of many steps run the whole time loop with no host
// involvement.  Each instance reproduces SecondOrderSolver::solve's step (Solvers/secondordersolver.cpp:288-314)
// bit for bit.  Compiled with -fmad=false.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vanguard_slic.h"
#include "host_planes.h"
#include "batch_internal.cuh"
#include "physics_fp64.cuh"
#include "slic_kernels.cuh"
#include "vg_ops.h"

namespace vg {
namespace {

using M1 = EulerF64<1>;

__device__ __forceinline__ double instance_dt(const BatchArgs& a, int k, int s) {
    double S = __longlong_as_double((long long)a.smax[(s % 3) * a.ninst + k]);
    double dt = a.cfl * (a.dx[k] / S);
    if (s <= 5) dt *= 0.2;
    return dt;
}

__global__ void __launch_bounds__(BP) batch_step_kernel(BatchArgs a) {
    constexpr int NU = M1::NU, NW = M1::NW;
    __shared__ double Us[NU][BP + 2];
    __shared__ double Es[NU][BP];
    __shared__ double Fs[NU][BP];
    __shared__ double red[BP / 32];
    __shared__ double tile_k[4];  // dt, dt/dx, dx/dt, 0.5 (dt/dx) of the tile's instance
    const int p = threadIdx.x;
    const int s = *a.step;
    const bool active = s < a.max_steps;
    const int slot_next = ((s + 1) % 3) * a.ninst;

    for (int t = blockIdx.x; t < a.ntiles && active; t += gridDim.x) {
        const Tile tile = a.tiles[t];
        const int k = tile.inst, len = a.ncell[k], s0 = tile.s0;
        const long base = a.offset[k];
        const int cell = s0 - 1 + p;
        const bool out_ok = p >= 1 && p <= BP - 2 && cell < len;
        // the instance's step constants, formed once per tile by one thread and shared after the first barrier
        if (p == 0) {
            const double dt = instance_dt(a, k, s);
            tile_k[0] = dt;
            tile_k[1] = dt / a.dx[k];
            tile_k[2] = a.dx[k] / dt;
            tile_k[3] = 0.5 * (dt / a.dx[k]);
            if (s0 == 0) a.dt_out[k] = dt;
        }
        SweepConst kc;
        kc.cm = 0.5 * (1.0 + a.bias);
        kc.cp = 0.5 * (1.0 - a.bias);
        kc.bias = a.bias;
        kc.floor5 = a.floor5;
        kc.limiter = a.limiter;
        M1::P q{a.gam[2 * k], a.gam[2 * k + 1], 0.0};

        auto conserve = [&](int slot) {
            int c = ghost_index(s0 - 2 + slot, len, 0);
            double W[NW], U[NU];
            for (int v = 0; v < NW; v++) W[v] = a.in[v * a.plane + base + c];
            M1::cons(W, q, U);
            for (int v = 0; v < NU; v++) Us[v][slot] = U[v];
        };
        conserve(p + 1);
        if (p == 0) conserve(0);
        if (p == BP - 1) conserve(BP + 1);
        __syncthreads();
        kc.r = tile_k[1];
        kc.rinv = tile_k[2];
        kc.half_r = tile_k[3];
        double ub[NU];
        {
            double uL[NU], u[NU], uR[NU], ua[NU];
            for (int v = 0; v < NU; v++) {
                uL[v] = Us[v][p];
                u[v] = Us[v][p + 1];
                uR[v] = Us[v][p + 2];
            }
            evolve_edges<M1, 0>(uL, u, uR, kc, q, ub, ua, p >= 1, p <= BP - 2);
            for (int v = 0; v < NU; v++) Es[v][p] = ua[v];
        }
        __syncthreads();
        if (p >= 1) {
            double ua[NU], F[NU];
            for (int v = 0; v < NU; v++) ua[v] = Es[v][p - 1];
            force_flux<M1, 0>(ua, ub, kc, q, F);
            for (int v = 0; v < NU; v++) Fs[v][p] = F[v];
        }
        __syncthreads();
        double wave = 0.0;
        if (out_ok) {
            double Un[NU], W[NW];
            for (int v = 0; v < NU; v++) Un[v] = Us[v][p + 1] + (kc.r * (Fs[v][p] - Fs[v][p + 1]));
            M1::setcons(Un, q, W);
            for (int v = 0; v < NW; v++) a.out[v * a.plane + base + cell] = W[v];
            if (bad_state<M1>(W, q)) atomicOr(a.err, ERR_STATE);
            double sw = M1::wave(W, q, 1);
            if (sw > wave) wave = sw;
        }
        // per-tile maximum into the instance's next slot
        for (int o = 16; o > 0; o >>= 1) {
            double w = __shfl_xor_sync(0xffffffffu, wave, o);
            wave = (w > wave) ? w : wave;
        }
        if ((p & 31) == 0) red[p >> 5] = wave;
        __syncthreads();
        if (p == 0) {
            double m = 0.0;
            for (int w = 0; w < BP / 32; w++) m = (red[w] > m) ? red[w] : m;
            if (m > 0.0) atomic_max_nonneg(&a.smax[slot_next + k], m);
        }
        __syncthreads();
    }
    if (!active) {  // past the last step: carry the state over so the buffer parity stays fixed
        for (long i = blockIdx.x * (long)BP + threadIdx.x; i < a.plane; i += (long)gridDim.x * BP)
            for (int v = 0; v < NW; v++) a.out[v * a.plane + i] = a.in[v * a.plane + i];
    }
    // the last block to finish clears (with all its threads) the slot the step after next will fill and advances
    // the step
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(a.done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        const int clear = ((s + 2) % 3) * a.ninst;
        for (int k = threadIdx.x; k < a.ninst; k += blockDim.x) a.smax[clear + k] = 0ull;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            if (active) *a.step = s + 1;
            *a.done = 0u;
            __threadfence();
        }
    }
}

// Initial maxima: slot a.wave_slot <- max over each instance's cells (one block per instance, no atomics).
// Also resets the step counter to a.step_init and the finished-block counter.
__global__ void __launch_bounds__(256) batch_max_wave_kernel(BatchArgs a) {
    const int k = blockIdx.x;
    if (k == 0 && threadIdx.x == 0) {
        *a.step = a.step_init;
        *a.done = 0u;
    }
    const long base = a.offset[k];
    const int n = a.ncell[k];
    const M1::P q{a.gam[2 * k], a.gam[2 * k + 1], 0.0};
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) {
        double W[M1::NW];
        for (int v = 0; v < M1::NW; v++) W[v] = a.in[v * a.plane + base + i];
        const double sw = M1::wave(W, q, 1);
        m = (sw > m) ? sw : m;
    }
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, m, o);
        m = (w > m) ? w : m;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; w++) m = (red[w] > m) ? red[w] : m;
        a.smax[a.wave_slot * a.ninst + k] = (unsigned long long)__double_as_longlong(m);
    }
}

// Known maxima (bit patterns) into slot a.wave_slot, and the counters reset.
__global__ void __launch_bounds__(256) batch_set_wave_kernel(BatchArgs a, const unsigned long long* S) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *a.step = a.step_init;
        *a.done = 0u;
    }
    for (int k = blockIdx.x * 256 + threadIdx.x; k < a.ninst; k += gridDim.x * 256) a.smax[a.wave_slot * a.ninst + k] = S[k];
}

BatchArgs batch_args(vg_batch* b, const double* in, double* out, double cfl, double bias, int limiter, int max_steps) {
    BatchArgs a{};
    a.in = in;
    a.out = out;
    a.plane = b->total;
    a.offset = b->d_offset;
    a.ncell = b->d_ncell;
    a.dx = b->d_dx;
    a.gam = b->d_gam;
    a.tiles = b->d_tiles;
    a.ntiles = b->ntiles;
    a.ninst = b->ninst;
    a.smax = b->d_smax;
    a.dt_out = b->d_dt;
    a.step = b->d_step;
    a.done = b->d_done;
    a.err = b->d_err;
    a.cfl = cfl;
    a.bias = bias;
    a.floor5 = std::pow(10.0, -5.0);
    a.limiter = limiter;
    a.max_steps = max_steps;
    a.wave_slot = 0;
    return a;
}

// Ring, step counter and the maxima of `state` for a run starting at step s_start; state_S (nullable) holds
// those maxima already (bit patterns, one per instance).
cudaError_t start_steps(vg_batch* b, const double* state, const unsigned long long* state_S, int s_start, double cfl,
                        double bias, int limiter, int max_steps, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(b->d_smax, 0, sizeof(unsigned long long) * 3 * b->ninst, st);
    if (e != cudaSuccess) return e;
    BatchArgs a0 = batch_args(b, state, nullptr, cfl, bias, limiter, max_steps);
    a0.wave_slot = s_start % 3;
    a0.step_init = s_start;
    if (state_S)
        batch_set_wave_kernel<<<std::max(1, std::min(b->ninst / 256 + 1, 148)), 256, 0, st>>>(a0, state_S);
    else
        batch_max_wave_kernel<<<b->ninst, 256, 0, st>>>(a0);
    return cudaGetLastError();
}

}  // namespace

cudaError_t batch_advance(vg_batch* b, const double* src, const unsigned long long* src_S, double* dst,
                          unsigned long long* dst_S, int s_start, int nsteps, double cfl, double bias, int limiter,
                          cudaStream_t st) {
    const size_t bytes = sizeof(double) * 3 * b->total;
    const size_t sbytes = sizeof(unsigned long long) * b->ninst;
    if (nsteps <= 0) {
        cudaError_t e = src == dst ? cudaSuccess : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && dst_S && dst_S != src_S) {
            if (src_S) return cudaMemcpyAsync(dst_S, src_S, sbytes, cudaMemcpyDeviceToDevice, st);
            return batch_wave_max(b, src, dst_S, st);
        }
        return e;
    }
    // src is only read; intermediate states alternate between the batch's two buffers and the last step writes
    // dst directly (dst must not be src or one of the batch's buffers)
    cudaError_t e = start_steps(b, src, src_S, s_start, cfl, bias, limiter, s_start + nsteps, st);
    const double* cur = src;
    for (int i = 0; i < nsteps && e == cudaSuccess; i++) {
        double* nxt = (i == nsteps - 1) ? dst : b->buf[i & 1];
        BatchArgs a = batch_args(b, cur, nxt, cfl, bias, limiter, s_start + nsteps);
        batch_step_kernel<<<b->grid, BP, 0, st>>>(a);
        e = cudaGetLastError();
        cur = nxt;
    }
    b->last_forward_steps += nsteps;
    // the last step accumulated the maxima of its result into slot (s_start + nsteps) % 3
    if (e == cudaSuccess && dst_S)
        e = cudaMemcpyAsync(dst_S, b->d_smax + ((s_start + nsteps) % 3) * b->ninst, sbytes, cudaMemcpyDeviceToDevice, st);
    return e;
}

cudaError_t batch_wave_max(vg_batch* b, const double* state, unsigned long long* out_S, cudaStream_t st) {
    BatchArgs a0 = batch_args(b, state, nullptr, 0.0, 0.0, 0, 0);
    // a private ring slot view: slot 0 of out_S, counters untouched by pointing them at scratch
    a0.smax = out_S;
    a0.wave_slot = 0;
    a0.step = b->d_step;
    a0.step_init = 0;
    batch_max_wave_kernel<<<b->ninst, 256, 0, st>>>(a0);
    return cudaGetLastError();
}

}  // namespace vg

using vg::BatchArgs;
using vg::Tile;

namespace {

vg_status bfail(vg_status st, const std::string& m) {
    vg::set_last_error(m);
    return st;
}

#define VB_CUDA(call)                                                                               \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return bfail(e_ == cudaErrorMemoryAllocation ? VG_ENOMEM : VG_ECUDA,  \
                                            std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

}  // namespace

extern "C" {

vg_status vg_batch_create(int ninst, const int* ncell, const double* dx, const double* gamma, const double* p_inf, int device,
                          vg_batch** out) {
    if (!out || !ncell || !dx || !gamma || ninst < 1) return bfail(VG_EINVAL, "bad vg_batch_create argument");
    *out = nullptr;
    for (int k = 0; k < ninst; k++)
        if (ncell[k] < 2 || !(dx[k] > 0.0)) return bfail(VG_EINVAL, "every instance needs >= 2 cells and dx > 0");
    VB_CUDA(cudaSetDevice(device));
    vg_batch* b = new (std::nothrow) vg_batch();
    if (!b) return bfail(VG_ENOMEM, "host allocation");
    b->ninst = ninst;
    b->device = device;
    b->ncell.assign(ncell, ncell + ninst);
    b->offset.resize(ninst);
    std::vector<Tile> tiles;
    long total = 0;
    for (int k = 0; k < ninst; k++) {
        b->offset[k] = total;
        total += ncell[k];
    }
    // tiles in decreasing instance size so the persistent grid ends on short work (longest first)
    std::vector<int> order(ninst);
    for (int k = 0; k < ninst; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return ncell[x] > ncell[y]; });
    for (int k : order)
        for (int s0 = 0; s0 < ncell[k]; s0 += vg::BP - 2) tiles.push_back({k, s0});
    b->total = total;
    b->ntiles = (int)tiles.size();
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vg::batch_step_kernel, vg::BP, 0);
    b->grid = std::max(1, std::min(b->ntiles, sms * std::max(per_sm, 1)));
    std::vector<double> gam(2 * ninst);
    for (int k = 0; k < ninst; k++) {
        gam[2 * k] = gamma[k];
        gam[2 * k + 1] = p_inf ? p_inf[k] : 0.0;
    }
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaMalloc(&b->buf[i], sizeof(double) * 3 * total);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_offset, sizeof(long) * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ncell, sizeof(int) * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_dx, sizeof(double) * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_gam, sizeof(double) * 2 * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tiles, sizeof(Tile) * tiles.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_smax, sizeof(unsigned long long) * 3 * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_dt, sizeof(double) * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_step, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_done, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_offset, b->offset.data(), sizeof(long) * ninst, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_ncell, ncell, sizeof(int) * ninst, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_dx, dx, sizeof(double) * ninst, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_gam, gam.data(), sizeof(double) * 2 * ninst, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        vg_batch_destroy(b);
        return bfail(VG_ECUDA, std::string("vg_batch_create: ") + cudaGetErrorString(e));
    }
    *out = b;
    return VG_OK;
}

vg_status vg_batch_destroy(vg_batch* b) {
    if (!b) return VG_OK;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto p : b->buf)
        if (p) cudaFree(p);
    for (auto p : b->lam)
        if (p) cudaFree(p);
    for (void* p : {(void*)b->d_offset, (void*)b->d_ncell, (void*)b->d_dx, (void*)b->d_gam, (void*)b->d_tiles,
                    (void*)b->d_smax, (void*)b->d_dt, (void*)b->d_step, (void*)b->d_done, (void*)b->d_err, (void*)b->ckpt,
                    (void*)b->d_target, (void*)b->d_atiles, (void*)b->d_tile_part, (void*)b->d_tile_first,
                    (void*)b->d_tile_count, (void*)b->d_ggam, (void*)b->ckptS, (void*)b->d_arg, (void*)b->d_loss})
        if (p) cudaFree(p);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
    return VG_OK;
}

long vg_batch_total_cells(vg_batch* b) { return b ? b->total : 0; }

vg_status vg_batch_upload(vg_batch* b, const double* planes, int is_device, void* stream) {
    if (!b || !planes) return bfail(VG_EINVAL, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const long n = b->total;
    // v, w and lambda are not carried: their check runs on host threads while rho, u and p are in flight, and a
    // failed check leaves the batch without a state
    b->has_state = false;
    bool bad = false;
    std::thread checker;
    if (!is_device)
        checker = std::thread([&]() {
            bad = vg::host::any_differs({planes + 2 * n, planes + 3 * n}, 0.0, n) ||
                  vg::host::any_differs({planes + 5 * n}, 1.0, n);
        });
    const int ref[3] = {0, 1, 4};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 3 && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(b->buf[0] + k * n, planes + ref[k] * n, sizeof(double) * n,
                            is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (checker.joinable()) checker.join();
    VB_CUDA(e);
    if (bad) return bfail(VG_EUNSUPPORTED, "batched 1D Euler needs v == w == 0 and lambda == 1");
    b->cur = 0;
    b->has_state = true;
    b->nonfinite = false;
    return VG_OK;
}

vg_status vg_batch_download(vg_batch* b, double* planes, int is_device, void* stream) {
    if (!b || !planes) return bfail(VG_EINVAL, "null argument");
    if (!b->has_state) return bfail(VG_EINVAL, "no state uploaded");
    cudaStream_t st = (cudaStream_t)stream;
    const long n = b->total;
    const int ref[3] = {0, 1, 4};
    for (int k = 0; k < 3; k++)
        VB_CUDA(cudaMemcpyAsync(planes + ref[k] * n, b->buf[b->cur] + k * n, sizeof(double) * n,
                                is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    if (!is_device) {  // the constant planes are filled while the copies run
        vg::host::fill_plane(planes + 2 * n, 0.0, n);
        vg::host::fill_plane(planes + 3 * n, 0.0, n);
        vg::host::fill_plane(planes + 5 * n, 1.0, n);
        if (b->nonfinite) {  // where a cell's state is non-finite the reference's v, w and lambda are NaN too
            VB_CUDA(cudaStreamSynchronize(st));
            vg::host::mark_nonfinite(planes, n, 6, 0x13u, 0x2cu);
        }
    } else {
        std::vector<double> z(n, 0.0), o(n, 1.0);
        VB_CUDA(cudaMemcpyAsync(planes + 2 * n, z.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
        VB_CUDA(cudaMemcpyAsync(planes + 3 * n, z.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
        VB_CUDA(cudaMemcpyAsync(planes + 5 * n, o.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
        VB_CUDA(cudaStreamSynchronize(st));
    }
    VB_CUDA(cudaStreamSynchronize(st));
    return VG_OK;
}

vg_status vg_batch_run(vg_batch* b, double cfl, int steps, double bias, int limiter, double* dt_last, void* stream) {
    if (!b || steps < 1 || !(cfl > 0.0)) return bfail(VG_EINVAL, "bad vg_batch_run argument");
    if (!b->has_state) return bfail(VG_EINVAL, "no state uploaded");
    cudaStream_t st = (cudaStream_t)stream;
    VB_CUDA(cudaSetDevice(b->device));
    // state to buffer 0 so the captured graph always starts there
    if (b->cur != 0) {
        VB_CUDA(cudaMemcpyAsync(b->buf[0], b->buf[1], sizeof(double) * 3 * b->total, cudaMemcpyDeviceToDevice, st));
        b->cur = 0;
    }
    VB_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(unsigned int), st));
    VB_CUDA(vg::start_steps(b, b->buf[0], nullptr, 0, cfl, bias, limiter, steps, st));
    // one graph per (steps, cfl, bias, limiter): the whole time loop, one persistent kernel per step
    if (!b->graph || b->graph_steps != steps || b->graph_cfl != cfl || b->graph_bias != bias || b->graph_limiter != limiter) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaGraph_t g = nullptr;
        VB_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < steps; i++) {
            BatchArgs a = vg::batch_args(b, b->buf[i & 1], b->buf[1 - (i & 1)], cfl, bias, limiter, steps);
            vg::batch_step_kernel<<<b->grid, vg::BP, 0, b->cap>>>(a);
        }
        cudaError_t e1 = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(b->cap, &g);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return bfail(VG_ECUDA, "batch graph capture failed");
        }
        cudaError_t e3 = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        VB_CUDA(e3);
        b->graph_steps = steps;
        b->graph_cfl = cfl;
        b->graph_bias = bias;
        b->graph_limiter = limiter;
    }
    VB_CUDA(cudaGraphLaunch(b->graph, st));
    b->cur = steps & 1;
    b->last_launches = 1 + steps;
    unsigned int err = 0;
    VB_CUDA(cudaMemcpyAsync(&err, b->d_err, sizeof(err), cudaMemcpyDeviceToHost, st));
    if (dt_last) VB_CUDA(cudaMemcpyAsync(dt_last, b->d_dt, sizeof(double) * b->ninst, cudaMemcpyDeviceToHost, st));
    VB_CUDA(cudaStreamSynchronize(st));
    if (err) {
        b->nonfinite = true;
        return bfail(VG_ENAN, "non-finite value, non-positive density or pressure at or below -p_inf produced");
    }
    return VG_OK;
}

long vg_batch_last_launch_count(vg_batch* b) { return b ? b->last_launches : 0; }

}  // extern "C"
