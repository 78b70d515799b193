// Reverse pass of the homogeneous HPR source batch (vg_source_batch_gradient): one thread per cell executes the
// host's binomial checkpoint schedule (a list of advance and reverse operations) for its cell, pulling the loss
// cotangent back through each step with the source's vector-Jacobian product (source_adjoint.cuh).  Compiled with
// FMA contraction (see source_step.cuh).
#include "source_adjoint.cuh"
#include "source_step.cuh"

namespace vg {
namespace srcb {

__device__ __forceinline__ const double* slot_ptr(const GradArgs& a, int s) {
    return s == 0 ? a.W0 : a.slots + (long)s * NV * a.n;
}

__global__ void __launch_bounds__(BT) gradient_kernel(GradArgs a) {
    const long c = blockIdx.x * (long)BT + threadIdx.x;
    if (c >= a.n) return;
    const H::P q = cell_params(a.params, a.tau, a.n, c);
    double lam[NV];          // dL/dU of the state after the step being reversed
    double lamJ[3] = {0.0, 0.0, 0.0};  // a non-thermal material's J passes through unchanged
    double gt1 = 0.0, gt2 = 0.0;
    for (int v = 0; v < NV; v++) lam[v] = 0.0;
#pragma unroll 1
    for (int o = 0; o < a.nops; o++) {
        const Op op = a.ops[o];
        double W[NV];
        const double* src = slot_ptr(a, op.src);
        for (int v = 0; v < NV; v++) W[v] = src[v * a.n + c];
        if (op.kind == 0) {
            advance(W, q, a.h, op.count);
            double* dst = a.slots + (long)op.dst * NV * a.n;
            for (int v = 0; v < NV; v++) dst[v * a.n + c] = W[v];
            continue;
        }
        // reverse step op.step from W = W(step)
        double U[NV], Un[NV], st[4][NV];
        H::cons(W, q, U);
        step_u(U, q, a.h, Un, st);
        if (op.step == a.steps - 1) {  // dL/dU(T) from dL/dW(T) through W(T) = setcons(U(T))
            double lw[NV];
            for (int v = 0; v < NV; v++) lw[v] = a.lamT[v * a.n + c];
            srcadj::setcons_vjp(Un, q, lw, lam);
            if (!q.thermal)
                for (int k = 0; k < 3; k++) lamJ[k] = lw[14 + k];
        }
        // U' = U + (k1 + 2 k2 + 2 k3 + k4) / 6, k_s = h S(stage_s), stage_{s} = U + c_s k_{s-1}
        double lk[4][NV], nu[NV];
        for (int v = 0; v < NV; v++) {
            lk[0][v] = lam[v] / 6.0;
            lk[1][v] = lam[v] / 3.0;
            lk[2][v] = lam[v] / 3.0;
            lk[3][v] = lam[v] / 6.0;
        }
        const double cs[4] = {0.0, 0.5, 0.5, 1.0};
#pragma unroll 1
        for (int s = 3; s >= 0; s--) {
            double mu[NV];
            for (int v = 0; v < NV; v++) {
                mu[v] = a.h * lk[s][v];
                nu[v] = 0.0;
            }
            srcadj::source_vjp(st[s], q, mu, nu, gt1, gt2);
            for (int v = 0; v < NV; v++) {
                lam[v] += nu[v];
                if (s > 0) lk[s - 1][v] += cs[s] * nu[v];
            }
        }
    }
    // dL/dW(0) from dL/dU(0) through U(0) = cons(W(0))
    double W0[NV], g[NV];
    for (int v = 0; v < NV; v++) W0[v] = a.W0[v * a.n + c];
    srcadj::cons_vjp(W0, q, lam, g);
    if (!q.thermal)
        for (int k = 0; k < 3; k++) g[14 + k] += lamJ[k];
    for (int v = 0; v < NV; v++) a.gW[v * a.n + c] = g[v];
    a.gtau[c] = gt1;
    a.gtau[a.n + c] = gt2;
}

cudaError_t launch_gradient(const GradArgs& a, unsigned blocks, cudaStream_t st) {
    gradient_kernel<<<blocks, BT, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace srcb
}  // namespace vg
