// Launch-configuration tables of the sweep kernels, shared by the FP64 and mixed translation units.
//
// Every model/precision instantiates the same candidate tile shapes.  The tile shape only changes which
// thread computes which cell, never the arithmetic of a cell, so all candidates produce identical results;
// the autotuner (vg_autotune in vg_api.cu) times them on the caller's grid and keeps the fastest.
#pragma once

#include <atomic>

#include <cuda_runtime.h>

#include "vg_common.cuh"

namespace vg {

using SweepFn = cudaError_t (*)(const SweepArgs&, cudaStream_t);

constexpr int kNumXCfg = 5;
constexpr int kNumYCfg = 6;

// X sweep: P cells per segment (P-2 outputs), LPB segments per block, MINB = minimum resident blocks
// per SM requested from the register allocator (1: no register cap).
template <class K, class M, int P, int LPB, int MINB>
cudaError_t launch_x(const SweepArgs& a, cudaStream_t st) {
    dim3 grid((a.nx + P - 3) / (P - 2), (a.ny + LPB - 1) / LPB);
    K::template x<M, P, LPB, MINB>(grid, P * LPB, st, a);
    return cudaGetLastError();
}

// Rows marched per Y-sweep block when segments are sized for whole waves.  A grid of a few waves leaves its last wave
// mostly empty (2048 blocks on 888 resident slots run as three waves), so the segment length is chosen from TY / 2 to
// 4 TY to minimise waves x (rows + 3), the 3 being the rows a block spends starting its march.  Whether that beats
// the shape's own TY depends on the model (measured: MHD Y sweeps 7-14 % faster, Euler's up to 5 % slower), so the
// autotuner times every shape both ways.  The results do not depend on the segmentation.
inline int y_segment_rows(int ny, int xblocks, long slots, int ty0) {
    if (slots <= 0 || ny <= 0) return ty0;
    int best = ty0;
    double best_cost = 1e300;
    for (int ty = (ty0 + 1) / 2; ty <= 4 * ty0; ty++) {
        const long blocks = (long)xblocks * ((ny + ty - 1) / ty);
        const long waves = (blocks + slots - 1) / slots;
        const double cost = (double)waves * (double)(ty + 3);
        if (cost < best_cost) {
            best_cost = cost;
            best = ty;
        }
        if (ty >= ny) break;
    }
    return best;
}

// Y sweep: TX columns per block, rows marched per thread from y_segment_rows (TY its centre), MINB as above.
template <class K, class M, int TX, int TY, int MINB>
cudaError_t launch_y(const SweepArgs& a0, cudaStream_t st) {
    if constexpr (!M::HAS_Y) {
        return cudaErrorInvalidValue;
    } else {
        static std::atomic<long> cached{0};  // resident blocks of this shape on the device (every thread stores the same)
        long slots = cached.load(std::memory_order_relaxed);
        if (slots == 0) {
            int dev = 0, sms = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            slots = (long)K::template y_resident<M, TX, TY, MINB>() * sms;
            if (slots <= 0) slots = -1;
            cached.store(slots, std::memory_order_relaxed);
        }
        if (a0.nx <= 0) return cudaSuccess;  // a call that only looks the occupancy up (before a graph capture)
        SweepArgs a = a0;
        const int xblocks = (a.nx + TX - 1) / TX;
        a.ty_rows = a.y_waves ? y_segment_rows(a.ny, xblocks, slots, TY) : TY;
        dim3 grid(xblocks, (a.ny + a.ty_rows - 1) / a.ty_rows);
        K::template y<M, TX, TY, MINB>(grid, TX, st, a);
        return cudaGetLastError();
    }
}

// X sweep staged by TMA (persistent, two rows per thread; see slic_tma.cuh) when the solver holds a tensor map over
// a.in, else the plain two-row kernel of the same shape.
template <class K, class M, int P, int MINB>
cudaError_t launch_x_tma(const SweepArgs& a, cudaStream_t st) {
    static_assert(P == kTmaTile, "the solver's tensor maps have a box of kTmaTile + 2 cells");
    if (!a.tmap) return launch_x<K, M, P, 1, MINB>(a, st);
    K::template x_tma<M, P, MINB>(st, a);
    return cudaGetLastError();
}

template <class M, class = void>
struct pair_sweeps {
    static constexpr bool value = false;
};
template <class M>
struct pair_sweeps<M, decltype((void)M::PAIR_X)> {
    static constexpr bool value = M::PAIR_X;
};

// Models with more than 9 conserved components (HPR, 17) use shorter X segments so that the three FP64
// shared-memory tiles stay inside the 48 KB static limit (kind 1); models with more than 21 (the HPR multiphysics
// model, 33) shorter still (kind 4).  The PAIR_X models (two rows per thread in the X sweep) add the TMA-staged X
// shapes for the Euler states of up to four planes (kind 2); other PAIR_X models (MHD) keep the plain two-row shapes
// (kind 3).
template <class M>
constexpr int tile_kind() {
    return (M::NU > 21) ? 4 : (M::NU > 9) ? 1 : pair_sweeps<M>::value ? (M::NW <= 4 ? 2 : 3) : 0;
}

template <class K, class M, int KIND = tile_kind<M>()>
struct SweepTable;

template <class K, class M>
struct SweepTable<K, M, 1> {
    static constexpr SweepFn x[kNumXCfg] = {
        launch_x<K, M, 64, 1, 1>, launch_x<K, M, 32, 2, 1>, launch_x<K, M, 96, 1, 1>,
        launch_x<K, M, 64, 1, 2>, launch_x<K, M, 32, 1, 1>,
    };
    static constexpr SweepFn y[kNumYCfg] = {
        launch_y<K, M, 64, 64, 1>, launch_y<K, M, 64, 32, 1>, launch_y<K, M, 32, 32, 1>,
        launch_y<K, M, 32, 64, 1>, launch_y<K, M, 128, 32, 1>, launch_y<K, M, 64, 16, 1>,
    };
};

template <class K, class M>
struct SweepTable<K, M, 4> {
    static constexpr SweepFn x[kNumXCfg] = {
        launch_x<K, M, 32, 1, 1>, launch_x<K, M, 40, 1, 1>, launch_x<K, M, 48, 1, 1>,
        launch_x<K, M, 56, 1, 1>, launch_x<K, M, 32, 1, 2>,
    };
    static constexpr SweepFn y[kNumYCfg] = {
        launch_y<K, M, 64, 64, 1>, launch_y<K, M, 64, 32, 1>, launch_y<K, M, 32, 32, 1>,
        launch_y<K, M, 32, 64, 1>, launch_y<K, M, 128, 32, 1>, launch_y<K, M, 64, 16, 1>,
    };
};

template <class K, class M>
struct SweepTable<K, M, 0> {
    static constexpr SweepFn x[kNumXCfg] = {
        launch_x<K, M, 128, 1, 1>, launch_x<K, M, 64, 2, 1>, launch_x<K, M, 192, 1, 1>,
        launch_x<K, M, 128, 1, 6>, launch_x<K, M, 128, 1, 8>,
    };
    static constexpr SweepFn y[kNumYCfg] = {
        launch_y<K, M, 64, 64, 1>, launch_y<K, M, 64, 32, 1>, launch_y<K, M, 64, 64, 12>,
        launch_y<K, M, 64, 64, 16>, launch_y<K, M, 128, 32, 5>, launch_y<K, M, 32, 64, 1>,
    };
};

template <class K, class M>
struct SweepTable<K, M, 2> {
    static constexpr SweepFn x[kNumXCfg] = {
        launch_x<K, M, 128, 1, 1>, launch_x_tma<K, M, 128, 7>, launch_x_tma<K, M, 128, 8>,
        launch_x<K, M, 128, 1, 6>, launch_x<K, M, 128, 1, 8>,
    };
    static constexpr SweepFn y[kNumYCfg] = {
        launch_y<K, M, 64, 64, 1>, launch_y<K, M, 64, 32, 1>, launch_y<K, M, 64, 64, 12>,
        launch_y<K, M, 64, 64, 16>, launch_y<K, M, 128, 32, 5>, launch_y<K, M, 32, 64, 1>,
    };
};

template <class K, class M>
struct SweepTable<K, M, 3> {
    static constexpr SweepFn x[kNumXCfg] = {
        launch_x<K, M, 128, 1, 1>, launch_x<K, M, 64, 2, 1>, launch_x<K, M, 128, 1, 4>,
        launch_x<K, M, 128, 1, 6>, launch_x<K, M, 128, 1, 8>,
    };
    static constexpr SweepFn y[kNumYCfg] = {
        launch_y<K, M, 64, 64, 1>, launch_y<K, M, 64, 32, 1>, launch_y<K, M, 64, 64, 12>,
        launch_y<K, M, 64, 64, 16>, launch_y<K, M, 128, 32, 5>, launch_y<K, M, 32, 64, 1>,
    };
};

// Names of the shapes of SweepTable<K, M, kind>.
inline const char* x_cfg_name(int i, int kind = 0) {
    static const char* n[kNumXCfg] = {"P128xL1", "P64xL2", "P192xL1", "P128xL1/min6", "P128xL1/min8"};
    static const char* nb[kNumXCfg] = {"P64xL1", "P32xL2", "P96xL1", "P64xL1/min2", "P32xL1"};
    static const char* np[kNumXCfg] = {"P128x2", "TMA P128x2/min7", "TMA P128x2/min8", "P128x2/min6", "P128x2/min8"};
    static const char* nq[kNumXCfg] = {"P128x2", "P64xL2x2", "P128x2/min4", "P128x2/min6", "P128x2/min8"};
    static const char* nw[kNumXCfg] = {"P32xL1", "P40xL1", "P48xL1", "P56xL1", "P32xL1/min2"};
    return (i >= 0 && i < kNumXCfg)
               ? (kind == 1 ? nb[i] : kind == 2 ? np[i] : kind == 3 ? nq[i] : kind == 4 ? nw[i] : n[i])
               : "?";
}
inline const char* y_cfg_name(int i, int kind = 0) {
    static const char* n[kNumYCfg] = {"TX64xTY64", "TX64xTY32", "TX64xTY64/min12", "TX64xTY64/min16",
                                      "TX128xTY32/min5", "TX32xTY64"};
    static const char* nb[kNumYCfg] = {"TX64xTY64", "TX64xTY32", "TX32xTY32", "TX32xTY64", "TX128xTY32", "TX64xTY16"};
    return (i >= 0 && i < kNumYCfg) ? ((kind == 1 || kind == 4) ? nb[i] : n[i]) : "?";
}

}  // namespace vg
