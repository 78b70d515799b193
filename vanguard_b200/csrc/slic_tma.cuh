// TMA-staged, persistent X sweep of the PAIR_X models (the Euler mixed form).
//
// Each block walks a strided list of tiles of two grid rows x (P + 2) cells (P - 2 outputs plus a two-cell halo on
// each side).  One thread loads a tile with a single cp.async.bulk.tensor (TMA) copy of all primitive planes into
// shared memory and signals an mbarrier; while the block computes tile k from one buffer, the copy of tile k + 1
// fills the other, so global-load latency overlaps the arithmetic instead of stalling every warp at the start of
// its tile.  The per-cell arithmetic is that of sweep_x_pair_kernel (evolve_edges_pair / force_flux_pair on packed
// FP32 lanes, FP64 update and primitive recovery), so the results are the same bits.
//
// The copies carry no multicast.  Cells outside [0, nx) come back as the copy's zero fill and are replaced by the
// boundary's ghost values (ghost_index) with plain loads; rows beyond ny are computed from the fill and never
// stored.  Every mbarrier wait is bounded: a wait that runs out sets ERR_TIMEOUT, waits (bounded again) for the
// copy still in flight and returns, and the host reports VG_ETIMEOUT.  If that second wait also runs out, a copy may
// still be writing into the exited block's shared memory, so the host must treat VG_ETIMEOUT as the end of the
// context: launch nothing more on it and reset the device before reusing it.
#pragma once

#include <cstdint>

#include "slic_mixed.cuh"

namespace vg {

constexpr int kTmaWaitLimit = 1 << 20;  // try_wait polls per wait before a block gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n"
        "  .reg .pred p;\n"
        "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "  selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < kTmaWaitLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Order this thread's earlier generic-proxy accesses of shared memory before later async-proxy (TMA) writes.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// One tiled 3D copy global -> shared (no multicast); x must be a multiple of 2 for 8-byte elements.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// a.tmap: a CUtensorMap over a.in with dims {nx, ny, NW}, strides {pitch, plane} (bytes), box {P + 2, 2, NW}.
template <class M, int P, int MINB>
__global__ void __launch_bounds__(P, MINB) sweep_x_tma_kernel(SweepArgs a) {
    constexpr int NU = M::NU, NW = M::NW, S = P + 2;
    static_assert(NU == NW, "conserved and primitive planes coincide for the PAIR_X models");
    static_assert((P - 2) % 2 == 0, "tile starts must be even cell indices (16-byte TMA x alignment of FP64)");
    // Two staging buffers, each a TMA destination, so each must start on a 128-byte boundary: the per-buffer stride is
    // rounded up to 16 doubles (without it the second buffer of a 3- or 7-plane state starts 16-byte aligned only, and
    // a 7-plane copy into it faulted with a misaligned address).
    constexpr int WST = ((NW * 2 * S + 15) / 16) * 16;
    __shared__ __align__(128) double Wsm[2 * WST];  // TMA destinations; converted in place to conserved
    __shared__ float2 Es[NU][P];
    __shared__ float2 Fs[NU][P];  // interface fluxes; widened to FP64 where the update reads them
    __shared__ __align__(8) uint64_t bar[2];

    const int p = threadIdx.x;
    const int len = a.nx;
    const int ntx = (a.nx + P - 3) / (P - 2), nty = (a.ny + 1) / 2;
    const int ntiles = ntx * nty;
    constexpr uint32_t kBytes = (uint32_t)(NW * 2 * S * sizeof(double));

    if (a.ctrl && !a.ctrl->active) {
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int cell = (t % ntx) * (P - 2) - 1 + p, row0 = 2 * (t / ntx);
            if (p < 1 || p > P - 2 || cell >= len) continue;
            for (int h = 0; h < 2 && row0 + h < a.ny; h++)
                for (int v = 0; v < NW; v++) {
                    const long i = v * a.plane + (long)(row0 + h) * a.pitch + cell;
                    a.out[i] = a.in[i];
                }
        }
        return;
    }
    double ts;
    const MixedConst k = mixed_const(a, ts);
    const typename M::P q = M::params(a.params, a.ctrl ? a.ctrl->ch : a.ch_host);

    if (p == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (p == 0 && (int)blockIdx.x < ntiles) {
        const int t = blockIdx.x;
        mbar_expect_tx(&bar[0], kBytes);
        tma_load_3d(Wsm, a.tmap, &bar[0], (t % ntx) * (P - 2) - 2, 2 * (t / ntx), 0);
    }

    uint32_t phase = 0u;  // bit b: parity of the next completion of bar[b]
    int buf = 0;
    double wave = 0.0;
    bool timed_out = false;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, buf ^= 1) {
        const int tn = t + gridDim.x;
        if (p == 0 && tn < ntiles) {  // the other buffer was released by the barrier that ended the previous tile
            fence_proxy_async_smem();
            mbar_expect_tx(&bar[buf ^ 1], kBytes);
            tma_load_3d(Wsm + (buf ^ 1) * WST, a.tmap, &bar[buf ^ 1], (tn % ntx) * (P - 2) - 2, 2 * (tn / ntx), 0);
        }
        const bool arrived = mbar_wait_bounded(&bar[buf], (phase >> buf) & 1u);
        if (__syncthreads_or(!arrived)) {
            if (p == 0) atomicOr(a.err, ERR_TIMEOUT);
            // leave no copy in flight behind: the one waited for and the prefetch (bounded waits as well)
            (void)mbar_wait_bounded(&bar[buf], (phase >> buf) & 1u);
            if (tn < ntiles) (void)mbar_wait_bounded(&bar[buf ^ 1], (phase >> (buf ^ 1)) & 1u);
            timed_out = true;
            break;
        }
        phase ^= 1u << buf;

        const int tx = t % ntx;
        const int s0 = tx * (P - 2);
        const int row0 = 2 * (t / ntx);
        const int cell = s0 - 1 + p;
        double(*U)[2][S] = reinterpret_cast<double(*)[2][S]>(Wsm + buf * WST);

        // cells outside [0, nx): the boundary's ghost values (the copy filled them with zeros)
        if (s0 - 2 < 0 || s0 - 2 + S > len) {
            for (int slot = p; slot < S; slot += P) {
                const int c = s0 - 2 + slot;
                if (c >= 0 && c < len) continue;
                const int g = ghost_index(c, len, a.periodic);
                for (int h = 0; h < 2; h++) {
                    const long rb = (long)(row0 + h < a.ny ? row0 + h : row0) * a.pitch;
                    for (int v = 0; v < NW; v++) U[v][h][slot] = a.in[v * a.plane + rb + g];
                }
            }
            __syncthreads();
        }
        // primitive -> conserved in place; thread p owns slot p + 1, the edge threads the two halo ends
        auto conserve = [&](int slot) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                double W[NW], Uc[NU];
#pragma unroll
                for (int v = 0; v < NW; v++) W[v] = U[v][h][slot];
                M::cons(W, q, Uc);
#pragma unroll
                for (int v = 0; v < NU; v++) U[v][h][slot] = Uc[v];
            }
        };
        conserve(p + 1);
        if (p == 0) conserve(0);
        if (p == P - 1) conserve(P + 1);
        __syncthreads();

        f2 ub[NU];
        {
            f2 ua[NU];
            evolve_edges_pair<M, 0>([&](int i, int o) { return make_double2(U[i][0][p + o], U[i][1][p + o]); }, k, q,
                                    ub, ua);
#pragma unroll
            for (int v = 0; v < NU; v++) Es[v][p] = ua[v].v;
        }
        __syncthreads();
        if (p >= 1) {
            f2 ua[NU], F[NU];
#pragma unroll
            for (int v = 0; v < NU; v++) ua[v].v = Es[v][p - 1];
            force_flux_pair<M, 0>(ua, ub, k, q, F);
#pragma unroll
            for (int v = 0; v < NU; v++) Fs[v][p] = F[v].v;
        }
        __syncthreads();

        if (p >= 1 && p <= P - 2 && cell < len) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (row0 + h >= a.ny) continue;
                const long base = (long)(row0 + h) * a.pitch;
                double Un[NU], W[NW];
#pragma unroll
                for (int v = 0; v < NU; v++) {
                    const float fl = h == 0 ? Fs[v][p].x : Fs[v][p].y, fr = h == 0 ? Fs[v][p + 1].x : Fs[v][p + 1].y;
                    Un[v] = fma(k.r, (double)fl - (double)fr, U[v][h][p + 1]);
                }
                keep_fields<M>(a, base + cell, q, W);
                M::setcons(Un, q, W);
#pragma unroll
                for (int v = 0; v < NW; v++) a.out[v * a.plane + base + cell] = W[v];
                if (bad_state_mixed<M>(W, q)) atomicOr(a.err, ERR_STATE);
                if (a.accumulate_wave) {
                    double s = M::wave(W, q, a.dims);
                    if (s > wave) wave = s;
                }
            }
        }
        __syncthreads();  // this tile's staging buffer, Es and Fs are free for the next tile
    }
    if (timed_out) return;
    if (a.accumulate_wave) block_max_to<P>(wave, a.wave_acc);
    if (a.advance_time && blockIdx.x == 0 && threadIdx.x == 0) {
        a.ctrl->t += a.ctrl->dt;
        a.ctrl->it += 1;
    }
}

}  // namespace vg
