// Homogeneous HPR relaxation: a batch of independent cells, each advanced by the HPR relaxation source alone, and
// the discrete adjoint of that evolution.  No counterpart in the reference, which has neither batches nor
// derivatives; the forward step is the reference's own source step on a spatially uniform field.
//
// Forward.  One step of length h is one sub-cycle of HPRForcingSolver's RK4 (Solvers/hprforcingsolver.cpp:
// 332-357) on a uniform 1D field with zero limiter bias: there the neighbours of a cell equal each other, so every
// slope of the fractional flux predictor is exactly zero and the predictor reduces to the primitive round trip it
// performs (setConservedVariableVector on a default-constructed state, then computeConservedVariableVector).  Per
// cell and step:
//   U = cons(W);  k1 = h S(U);  for s = 1..3: U_s = U + c_s k_s (c = 1/2, 1/2, 1), round trips as the forcing
//   performs them, k_{s+1} = h S(U_s);  U' = U + (k1 + (2 k2 + (2 k3 + k4))) / 6;  W' = setcons(U')
// in the reference's association order and compiled without FMA contraction (the unit is built with -fmad=false),
// so a step equals the forcing kernel's on such a field.  Relaxation times may differ per cell.
//
// Adjoint.  The loss cotangent dL/dW(T) is pulled back through the steps in conserved variables (the round trips
// are identities of exact arithmetic and drop out), with the source's vector-Jacobian product of
// source_adjoint.cuh at each RK4 stage, then converted to dL/dW(0) and dL/dtau1, dL/dtau2 per cell.  Each cell is
// independent, so one thread owns one cell for the whole reversal, with its own checkpoints in global memory: the
// host lays out Griewank's binomial schedule as a list of operations (advance a checkpoint, reverse a step) that
// every thread executes in one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/vanguard_slic.h"
#include "source_step.cuh"
#include "vg_ops.h"

namespace vg {
namespace srcb {

struct Args {
    double* W;           // 17 x n current state (primitives)
    const double* tau;   // 2 x n relaxation times (tau1, tau2)
    long n;
    double h;
    int steps;
    double params[kParams];
};

__global__ void __launch_bounds__(BT) run_kernel(Args a) {
    const long c = blockIdx.x * (long)BT + threadIdx.x;
    if (c >= a.n) return;
    const H::P q = cell_params(a.params, a.tau, a.n, c);
    double W[NV];
    for (int v = 0; v < NV; v++) W[v] = a.W[v * a.n + c];
    advance(W, q, a.h, a.steps);
    for (int v = 0; v < NV; v++) a.W[v * a.n + c] = W[v];
}

}  // namespace srcb
}  // namespace vg

struct vg_source_batch {
    int device = 0;
    long n = 0;
    double params[VG_MAX_PARAMS] = {0};
    double* W = nullptr;      // 17 x n current state
    double* tau = nullptr;    // 2 x n
    bool has_state = false;
    double* slots = nullptr;  // checkpoint slots (allocated by the first gradient)
    int nslots = 0;
    double* lam = nullptr;    // 17 x n cotangent in, 17 x n gradient out, 2 x n tau gradient
    vg::srcb::Op* d_ops = nullptr;
    int ops_cap = 0;
    long last_fwd = 0, last_rev = 0;
};

namespace {

vg_status sfail(vg_status st, const std::string& m) {
    vg::set_last_error(m);
    return st;
}

#define VS_CUDA(call)                                                                                \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return sfail(e_ == cudaErrorMemoryAllocation ? VG_ENOMEM : VG_ECUDA,   \
                                            std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

double beta(int s, int t) {  // C(s + t, s): steps s stored states reverse with at most t advances per step
    double v = 1.0;
    for (int i = 1; i <= t; i++) v = v * (s + i) / i;
    return v;
}

// Griewank's binomial schedule as a list of operations: reverse steps [s0, s1) with W(s0) in `slot` and c free
// slots besides it; the recomputation slot is `tmp`.
struct Planner {
    std::vector<vg::srcb::Op> ops;
    std::vector<bool> used;
    int tmp = 0;
    long fwd = 0, rev = 0;
    int take() {
        for (size_t i = 1; i < used.size(); i++)
            if (!used[i]) {
                used[i] = true;
                return (int)i;
            }
        return -1;
    }
    void advance(int src, int dst, int count) {
        ops.push_back({0, src, dst, count, 0});
        fwd += count;
    }
    void reverse_step(int slot, int s) {
        ops.push_back({1, slot, 0, 0, s});
        fwd += 1;  // the step is recomputed inside the reverse operation
        rev += 1;
    }
    void reverse(int s0, int s1, int c, int slot) {
        const int n = s1 - s0;
        if (n == 1) return reverse_step(slot, s0);
        if (c == 0) {
            for (int s = s1 - 1; s > s0; s--) {
                advance(slot, tmp, s - s0);
                reverse_step(tmp, s);
            }
            return reverse_step(slot, s0);
        }
        int t = 1;
        while (beta(c + 1, t) < n) t++;
        const int right = (int)std::min<double>(n - 1, beta(c, t));
        const int m = s1 - right;
        const int ns = take();
        advance(slot, ns, m - s0);
        reverse(m, s1, c - 1, ns);
        used[ns] = false;
        reverse(s0, m, c, slot);
    }
};

}  // namespace

extern "C" {

vg_status vg_source_batch_create(int ncell, const double* params, int device, vg_source_batch** out) {
    if (!out || !params || ncell < 1) return sfail(VG_EINVAL, "bad vg_source_batch_create argument");
    *out = nullptr;
    if (params[12] != 0.0 || params[17] != 0.0)
        return sfail(VG_EUNSUPPORTED, "the source batch covers the StiffenedGas equation of state with elastic strain "
                                      "relaxation (params[12] == 0, params[17] == 0)");
    if (!(params[0] > 1.0) || !(params[2] > 0.0) || !(params[3] > 0.0) || !(params[4] > 0.0) || !(params[5] > 0.0))
        return sfail(VG_EINVAL, "need gamma > 1 and positive c_v, rho0, T0, c_s");
    VS_CUDA(cudaSetDevice(device));
    vg_source_batch* b = new (std::nothrow) vg_source_batch();
    if (!b) return sfail(VG_ENOMEM, "host allocation");
    b->device = device;
    b->n = ncell;
    std::memcpy(b->params, params, sizeof(double) * VG_MAX_PARAMS);
    b->params[vg::kInvGm1] = 1.0 / (params[0] - 1.0);
    cudaError_t e = cudaMalloc(&b->W, sizeof(double) * 17 * b->n);
    if (e == cudaSuccess) e = cudaMalloc(&b->tau, sizeof(double) * 2 * b->n);
    if (e == cudaSuccess) e = cudaMalloc(&b->lam, sizeof(double) * 36 * b->n);
    if (e != cudaSuccess) {
        vg_source_batch_destroy(b);
        return sfail(VG_ENOMEM, std::string("vg_source_batch_create: ") + cudaGetErrorString(e));
    }
    *out = b;
    return VG_OK;
}

vg_status vg_source_batch_destroy(vg_source_batch* b) {
    if (!b) return VG_OK;
    cudaFree(b->W);
    cudaFree(b->tau);
    cudaFree(b->slots);
    cudaFree(b->lam);
    cudaFree(b->d_ops);
    delete b;
    return VG_OK;
}

vg_status vg_source_batch_upload(vg_source_batch* b, const double* planes, const double* tau, int is_device,
                                 void* stream) {
    if (!b || !planes) return sfail(VG_EINVAL, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    VS_CUDA(cudaSetDevice(b->device));
    VS_CUDA(cudaMemcpyAsync(b->W, planes, sizeof(double) * 17 * b->n, kind, st));
    if (tau) {
        VS_CUDA(cudaMemcpyAsync(b->tau, tau, sizeof(double) * 2 * b->n, kind, st));
    } else {
        std::vector<double> t(2 * b->n);
        std::fill(t.begin(), t.begin() + b->n, b->params[7]);
        std::fill(t.begin() + b->n, t.end(), b->params[8]);
        VS_CUDA(cudaMemcpyAsync(b->tau, t.data(), sizeof(double) * 2 * b->n, cudaMemcpyHostToDevice, st));
    }
    VS_CUDA(cudaStreamSynchronize(st));
    b->has_state = true;
    return VG_OK;
}

vg_status vg_source_batch_download(vg_source_batch* b, double* planes, int is_device, void* stream) {
    if (!b || !planes) return sfail(VG_EINVAL, "null argument");
    if (!b->has_state) return sfail(VG_EINVAL, "no state uploaded");
    cudaStream_t st = (cudaStream_t)stream;
    VS_CUDA(cudaMemcpyAsync(planes, b->W, sizeof(double) * 17 * b->n,
                            is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    VS_CUDA(cudaStreamSynchronize(st));
    return VG_OK;
}

vg_status vg_source_batch_run(vg_source_batch* b, double h, int steps, void* stream) {
    if (!b || !(h > 0.0) || steps < 1) return sfail(VG_EINVAL, "bad vg_source_batch_run argument");
    if (!b->has_state) return sfail(VG_EINVAL, "no state uploaded");
    cudaStream_t st = (cudaStream_t)stream;
    VS_CUDA(cudaSetDevice(b->device));
    vg::srcb::Args a{};
    a.W = b->W;
    a.tau = b->tau;
    a.n = b->n;
    a.h = h;
    a.steps = steps;
    std::memcpy(a.params, b->params, sizeof(a.params));
    vg::srcb::run_kernel<<<(unsigned)((b->n + vg::srcb::BT - 1) / vg::srcb::BT), vg::srcb::BT, 0, st>>>(a);
    VS_CUDA(cudaGetLastError());
    VS_CUDA(cudaStreamSynchronize(st));
    return VG_OK;
}

vg_status vg_source_batch_gradient(vg_source_batch* b, const double* cotangent, double h, int steps, int checkpoints,
                                   double* grad_planes, double* grad_tau, int is_device, long* forward_steps,
                                   long* adjoint_steps, void* stream) {
    if (!b || !cotangent || !(h > 0.0) || steps < 1) return sfail(VG_EINVAL, "bad vg_source_batch_gradient argument");
    if (checkpoints < 1) return sfail(VG_EINVAL, "need at least one checkpoint slot (the initial state)");
    if (!b->has_state) return sfail(VG_EINVAL, "no state uploaded");
    checkpoints = std::min(checkpoints, steps);
    cudaStream_t st = (cudaStream_t)stream;
    VS_CUDA(cudaSetDevice(b->device));
    // slots 1 .. checkpoints - 1 hold checkpoints, slot `checkpoints` is the recomputation buffer (slot 0: the state)
    const int nslots = checkpoints + 1;
    if (b->nslots != nslots) {
        cudaFree(b->slots);
        b->slots = nullptr;
        b->nslots = 0;
        VS_CUDA(cudaMalloc(&b->slots, sizeof(double) * 17 * b->n * nslots));
        b->nslots = nslots;
    }
    Planner pl;
    pl.used.assign(checkpoints, false);
    pl.used[0] = true;
    pl.tmp = checkpoints;
    pl.reverse(0, steps, checkpoints - 1, 0);
    if ((int)pl.ops.size() > b->ops_cap) {
        cudaFree(b->d_ops);
        b->d_ops = nullptr;
        b->ops_cap = 0;
        VS_CUDA(cudaMalloc(&b->d_ops, sizeof(vg::srcb::Op) * pl.ops.size()));
        b->ops_cap = (int)pl.ops.size();
    }
    VS_CUDA(cudaMemcpyAsync(b->d_ops, pl.ops.data(), sizeof(vg::srcb::Op) * pl.ops.size(), cudaMemcpyHostToDevice, st));
    const long n = b->n;
    double* lamT = b->lam;
    double* gW = b->lam + 17 * n;
    double* gtau = b->lam + 34 * n;
    VS_CUDA(cudaMemcpyAsync(lamT, cotangent, sizeof(double) * 17 * n,
                            is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    vg::srcb::GradArgs a{};
    a.W0 = b->W;
    a.slots = b->slots;
    a.tau = b->tau;
    a.lamT = lamT;
    a.gW = gW;
    a.gtau = gtau;
    a.ops = b->d_ops;
    a.nops = (int)pl.ops.size();
    a.n = n;
    a.h = h;
    a.steps = steps;
    std::memcpy(a.params, b->params, sizeof(a.params));
    VS_CUDA(vg::srcb::launch_gradient(a, (unsigned)((n + vg::srcb::BT - 1) / vg::srcb::BT), st));
    const cudaMemcpyKind back = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (grad_planes) VS_CUDA(cudaMemcpyAsync(grad_planes, gW, sizeof(double) * 17 * n, back, st));
    if (grad_tau) VS_CUDA(cudaMemcpyAsync(grad_tau, gtau, sizeof(double) * 2 * n, back, st));
    VS_CUDA(cudaStreamSynchronize(st));
    b->last_fwd = pl.fwd;
    b->last_rev = pl.rev;
    if (forward_steps) *forward_steps = pl.fwd;
    if (adjoint_steps) *adjoint_steps = pl.rev;
    return VG_OK;
}

}  // extern "C"
