// Internal types of the ragged 1D Euler batch (batch.cu) shared with its adjoint (adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/vanguard_slic.h"
#include "vg_common.cuh"

namespace vg {

constexpr int BP = 128;  // cells per tile segment of the forward step kernel (BP - 2 outputs)

struct Tile {
    int inst;  // instance
    int s0;    // first output cell within the instance
};

struct BatchArgs {
    const double* in;
    double* out;
    long plane;                 // plane stride (total cells)
    const long* offset;         // first cell of each instance
    const int* ncell;           // cells of each instance
    const double* dx;           // cell width of each instance
    const double* gam;          // gamma, p_inf of each instance (2 per instance)
    const Tile* tiles;
    int ntiles;
    int ninst;
    unsigned long long* smax;   // 3 x ninst ring of wave-speed maxima (bit patterns)
    double* dt_out;             // dt of the current step per instance
    int* step;                  // device step counter
    unsigned int* done;         // blocks finished in this step
    unsigned int* err;
    double cfl, bias, floor5;
    int limiter;
    int max_steps;
    int wave_slot;              // slot the initial maximum kernel fills
    int step_init;              // step index the initial maximum kernel stores in *step
};

// Forward-advance nsteps steps from the state in `src` (3 planes of the batch's total cells), with step
// indices starting at s_start (the x0.2 factor applies to indices <= 5); the result is written to `dst`.
// src is left unchanged; dst must be a device buffer of the same shape other than src and the batch's buf[].
// src_S (nullable) holds the maxima |u| + c of src per instance (double bit patterns) so no pass over src is
// needed; dst_S (nullable) receives those of dst.
cudaError_t batch_advance(::vg_batch* b, const double* src, const unsigned long long* src_S, double* dst,
                          unsigned long long* dst_S, int s_start, int nsteps, double cfl, double bias, int limiter,
                          cudaStream_t st);

// out_S[k] <- max over instance k's cells of |u| + c of `state` (bit patterns); resets the batch's step counter.
cudaError_t batch_wave_max(::vg_batch* b, const double* state, unsigned long long* out_S, cudaStream_t st);

}  // namespace vg

struct vg_batch {
    int ninst = 0, device = 0;
    long total = 0;
    std::vector<int> ncell;
    std::vector<long> offset;
    double* buf[2] = {nullptr, nullptr};
    long* d_offset = nullptr;
    int* d_ncell = nullptr;
    double* d_dx = nullptr;
    double* d_gam = nullptr;
    vg::Tile* d_tiles = nullptr;
    int ntiles = 0;
    unsigned long long* d_smax = nullptr;
    double* d_dt = nullptr;
    int* d_step = nullptr;
    unsigned int* d_done = nullptr;
    unsigned int* d_err = nullptr;
    int cur = 0;
    bool has_state = false;  // a successful vg_batch_upload has filled buf[0]
    bool nonfinite = false;  // a run since the upload flagged a non-finite or unphysical state
    int grid = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    double graph_cfl = 0, graph_bias = 0;
    int graph_limiter = -1;
    long last_launches = 0;
    // adjoint workspace (allocated on first use by vg_batch_gradient)
    double* lam[2] = {nullptr, nullptr};  // dL/dW of the step being reversed and of the one before
    double* ckpt = nullptr;               // checkpoint slots + one recomputation buffer
    unsigned long long* ckptS = nullptr;  // their per-instance maxima |u| + c (double bit patterns)
    int ckpt_slots = 0;
    double* d_target = nullptr;           // target density of the loss
    vg::Tile* d_atiles = nullptr;         // adjoint tiles (contiguous per instance)
    int natiles = 0;
    int agrid = 0;
    double* d_tile_part = nullptr;        // 2 per adjoint tile: r-bar, gamma-bar partials
    int* d_tile_first = nullptr;          // first adjoint tile of each instance
    int* d_tile_count = nullptr;
    double* d_ggam = nullptr;             // gamma gradient per instance
    int* d_arg = nullptr;                 // first cell attaining S, per instance (INT_MAX between steps)
    double* d_loss = nullptr;             // per-block partial losses
    int loss_blocks = 0;
    long last_forward_steps = 0, last_adjoint_steps = 0;
};
