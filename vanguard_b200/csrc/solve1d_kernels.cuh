// Whole-run 1D SLIC loop in one thread-block cluster, for rows of up to S1D_CL * (2 * S1D_NT - 2) cells.
//
// A 1000-cell run (the Sod shock tube) is launch-latency bound: the graph-driven loop spends ~9 us per step on two
// kernel nodes whose work takes well under a microsecond.  Here a cluster of S1D_CL blocks, one per SM, runs every
// step of SecondOrderSolver::solve (Solvers/secondordersolver.cpp:288-314) without leaving the device.  Block r owns a
// contiguous segment of the row in its shared memory; per step it forms the CFL maximum of the previous update from
// every block's partial maximum (read through distributed shared memory), the time step of step_begin_kernel
// (Solvers/solvers.cpp:388-452: x0.2 for the first six steps, clamped to t_end), and then the X sweep's four stages --
// conserve, evolve edges, FORCE, update -- over its segment, reading the two halo cells a side from its neighbours'
// shared memory.  The updated state goes to the other of two shared buffers, so one cluster barrier per step orders
// every read of a step before the writes that follow it.  Every per-cell value comes from the same device functions as
// the graph-driven sweeps (slic_kernels.cuh), and the maximum of non-negative values does not depend on the order, so
// the result is bit for bit the graph-driven loop's.  Every block takes the same decisions (the same t, it and dt from
// the same maximum), so all of them reach every barrier.  A run stops at t_end, at max_steps, or after S1D_STEP_CAP
// steps (the host reports a run that did not reach its end).
#pragma once

#include <cooperative_groups.h>

#include "slic_kernels.cuh"
#include "vg_common.cuh"

namespace vg {

constexpr int S1D_CL = 8;    // blocks of the cluster (the portable maximum)
constexpr int S1D_NT = 128;  // threads per block
constexpr int S1D_KMAX = 2;  // edge-stage cells per thread (segment cells -1 .. len)
constexpr int S1D_STEP_CAP = 1 << 22;

// Cells per block for an nx-cell row, and the largest row.
__host__ __device__ constexpr int solve1d_seg(int nx) { return (nx + S1D_CL - 1) / S1D_CL; }
constexpr int solve1d_max_cells() { return S1D_CL * (S1D_KMAX * S1D_NT - 2); }
// Smallest row: every block owns at least two cells, so every halo cell lies within one ghost of the row
constexpr int solve1d_min_cells() { return 2 * S1D_CL; }

// Shared-memory doubles of one block for segments of `seg` cells: two primitive buffers, conserved vectors with two
// halo cells a side, evolved right-side edge states of cells -1 .. seg, interface fluxes at -1/2 .. seg - 1/2.
template <class M>
__host__ __device__ constexpr long solve1d_smem_doubles(int seg) {
    return 2L * M::NW * seg + (long)M::NU * (seg + 4) + (long)M::NU * (seg + 2) + (long)M::NU * (seg + 1);
}

template <class M>
__global__ void __cluster_dims__(S1D_CL, 1, 1) __launch_bounds__(S1D_NT) solve1d_kernel(SweepArgs a) {
    namespace cg = cooperative_groups;
    static_assert(!M::HAS_SOURCE, "models with a source or a per-step c_h run the graph-driven loop");
    constexpr int NU = M::NU, NW = M::NW;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ double sm[];
    __shared__ double part[2];  // this block's maximum wave speed of the state in buffer b
    __shared__ double red[S1D_NT / 32];
    const int nx = a.nx, seg = solve1d_seg(nx);
    const int rank = (int)cluster.block_rank();
    const int c0 = rank * seg;                                   // first cell of the segment
    const int len = max(0, min(seg, nx - c0));                   // cells of the segment
    double* Wb[2] = {sm, sm + (long)NW * seg};                   // [NW][seg] each
    double* Ush = sm + 2L * NW * seg;                            // [NU][seg + 4], slot = local cell + 2
    double* Esh = Ush + (long)NU * (seg + 4);                    // [NU][seg + 2], index = local cell + 1
    double* Fsh = Esh + (long)NU * (seg + 2);                    // [NU][seg + 1], index j = interface j - 1/2
    const int tid = threadIdx.x;
    const typename M::P q = M::params(a.params, 0.0);

    // the block's maximum of non-negative speeds (non-finite values are skipped, as the graph-driven reduction does)
    auto block_max = [&](double v, double* out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xffffffffu, v, o);
            v = (w > v) ? w : v;
        }
        if ((tid & 31) == 0) red[tid >> 5] = v;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < S1D_NT / 32; w++) m = (red[w] > m) ? red[w] : m;
            *out = m;
        }
    };

    double wave = 0.0;
    for (int i = tid; i < len; i += S1D_NT) {
        double W[NW];
#pragma unroll
        for (int v = 0; v < NW; v++) {
            W[v] = a.in[v * a.plane + c0 + i];
            Wb[0][(long)v * seg + i] = W[v];
        }
        const double s = M::wave(W, q, 1);
        if (s > wave) wave = s;
    }
    block_max(wave, &part[0]);
    cluster.sync();

    SweepConst k;
    k.cm = 0.5 * (1.0 + a.bias);
    k.cp = 0.5 * (1.0 - a.bias);
    k.bias = a.bias;
    k.floor5 = a.floor5;
    k.limiter = a.limiter;
    const double cfl = a.ctrl->cfl, dx = a.ctrl->dx, t_end = a.ctrl->t_end;
    const int max_steps = a.ctrl->max_steps;
    double t = a.ctrl->t, dt = 0.0;
    int it = a.ctrl->it, b = 0;

    for (;;) {
        // step_begin_kernel, taken identically by every block: S from every block's partial maximum (never NaN), lane r
        // of each warp reading block r's through distributed shared memory and the warp combining them
        double m = 0.0;
        if ((tid & 31) < S1D_CL) m = cluster.map_shared_rank(part, tid & 31)[b];
#pragma unroll
        for (int o = S1D_CL / 2; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xffffffffu, m, o);
            m = (w > m) ? w : m;
        }
        const double S = __shfl_sync(0xffffffffu, m, 0);
        if (!((t < t_end) && (it < max_steps) && (it < S1D_STEP_CAP))) break;
        dt = cfl * (dx / S);
        if (it <= 5) dt *= 0.2;
        if ((t + dt) > t_end) dt = t_end - t;
        sweep_scale(dt * 1.0, dx, k.r, k.rinv, k.half_r);

        // stage 1: conserved vectors of cells c0 - 2 .. c0 + len + 1, through the row's ghosts and the neighbours
        for (int slot = tid; slot < len + 4; slot += S1D_NT) {
            const int cell = ghost_index(c0 + slot - 2, nx, a.periodic);
            const int owner = cell / seg;
            const double* Wsrc = owner == rank ? Wb[b] : cluster.map_shared_rank(Wb[b], owner);
            double W[NW], U[NU];
#pragma unroll
            for (int v = 0; v < NW; v++) W[v] = Wsrc[(long)v * seg + (cell - owner * seg)];
            M::cons(W, q, U);
#pragma unroll
            for (int v = 0; v < NU; v++) Ush[(long)v * (seg + 4) + slot] = U[v];
        }
        __syncthreads();

        // stage 2: evolved edge states of local cells -1 .. len; the left-side one stays in registers for stage 3
        double ub[S1D_KMAX][NU];
#pragma unroll
        for (int kk = 0; kk < S1D_KMAX; kk++) {
            const int cell = -1 + tid + kk * S1D_NT;
            if (cell > len) break;
            double uL[NU], u[NU], uR[NU], ua[NU];
#pragma unroll
            for (int v = 0; v < NU; v++) {
                uL[v] = Ush[(long)v * (seg + 4) + cell + 1];
                u[v] = Ush[(long)v * (seg + 4) + cell + 2];
                uR[v] = Ush[(long)v * (seg + 4) + cell + 3];
            }
            evolve_edges<M, 0>(uL, u, uR, k, q, ub[kk], ua, cell >= 0, cell <= len - 1);
#pragma unroll
            for (int v = 0; v < NU; v++) Esh[(long)v * (seg + 2) + cell + 1] = ua[v];
        }
        __syncthreads();

        // stage 3: FORCE flux at the interface left of local cells 0 .. len
#pragma unroll
        for (int kk = 0; kk < S1D_KMAX; kk++) {
            const int cell = -1 + tid + kk * S1D_NT;
            if (cell > len) break;
            if (cell < 0) continue;
            double ua[NU], F[NU];
#pragma unroll
            for (int v = 0; v < NU; v++) ua[v] = Esh[(long)v * (seg + 2) + cell];
            force_flux<M, 0>(ua, ub[kk], k, q, F);
#pragma unroll
            for (int v = 0; v < NU; v++) Fsh[(long)v * (seg + 1) + cell] = F[v];
        }
        __syncthreads();

        // stage 4: conservative update (Solvers/firstordersolver.cpp:428-433) into the other buffer, and the
        // block's part of the next step's CFL maximum
        wave = 0.0;
        for (int i = tid; i < len; i += S1D_NT) {
            double Un[NU], W[NW];
#pragma unroll
            for (int v = 0; v < NU; v++)
                Un[v] = Ush[(long)v * (seg + 4) + i + 2] +
                        (k.r * (Fsh[(long)v * (seg + 1) + i] - Fsh[(long)v * (seg + 1) + i + 1]));
#pragma unroll
            for (int v = 0; v < NW; v++) W[v] = Wb[b][(long)v * seg + i];  // fields setcons leaves alone keep theirs
            M::setcons(Un, q, W);
#pragma unroll
            for (int v = 0; v < NW; v++) Wb[1 - b][(long)v * seg + i] = W[v];
            if (bad_state<M>(W, q)) atomicOr(a.err, ERR_STATE);
            const double s = M::wave(W, q, 1);
            if (s > wave) wave = s;
        }
        block_max(wave, &part[1 - b]);
        t += dt;
        it += 1;
        b = 1 - b;
        cluster.sync();  // the new state and maxima are complete; every read of the old buffer is done
    }
    cluster.sync();  // no block leaves while a neighbour may still read its shared memory

    for (int i = tid; i < len; i += S1D_NT)
#pragma unroll
        for (int v = 0; v < NW; v++) a.out[v * a.plane + c0 + i] = Wb[b][(long)v * seg + i];
    if (rank == 0 && tid == 0) {
        a.ctrl->t = t;
        a.ctrl->it = it;
        a.ctrl->dt = dt;
        a.ctrl->active = 0;
    }
}

}  // namespace vg
