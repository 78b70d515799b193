// C ABI of the SLIC/FORCE solver (include/vanguard_slic.h): solver objects, state upload/download, the
// device-resident time loop replayed from captured CUDA graphs, and the per-sweep entry points.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vanguard_slic.h"
#include "host_planes.h"
#include "vg_ops.h"

using vg::Ctrl;
using vg::Ops;
using vg::SweepArgs;

static_assert(vg::kNumXCfg == VG_NUM_XCFG && vg::kNumYCfg == VG_NUM_YCFG, "the header names the tile-shape counts");

namespace {

thread_local std::string g_last_error;

vg_status fail(vg_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

vg_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? VG_ENOMEM : VG_ECUDA;
}

#define VG_CUDA(call)                                        \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
    } while (0)

int ref_nvar(int model) {
    return model == VG_MODEL_EULER ? 6 : model == VG_MODEL_MHD ? 9 : model == VG_MODEL_HPR ? 17 : model == VG_MODEL_EULER_REDUCED ? 7
           : model == VG_MODEL_EULER_MULTIPHYSICS ? 8 : model == VG_MODEL_MHD_REDUCED ? 11
           : model == VG_MODEL_MHD_INTERMEDIATE ? 12 : model == VG_MODEL_HPR_REDUCED ? 19
           : model == VG_MODEL_HPR_INTERMEDIATE ? 20 : model == VG_MODEL_HPR_MULTIPHYSICS ? 32
           : model == VG_MODEL_MHD_MULTIPHYSICS ? 16 : 0;
}

// Reference plane carried in device plane k, per variant.
const int kPlanes[vg::V_COUNT][32] = {
    {0, 1, 4},                      // V_EULER1: rho, u, p
    {0, 1, 2, 4},                   // V_EULER2: rho, u, v, p
    {0, 1, 2, 4, 5, 6, 8},          // V_MHD7:   rho, u, v, p, Bx, By, psi
    {0, 1, 2, 3, 4, 5, 6, 7, 8},    // V_MHD9
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16},  // V_HPR17
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16},  // V_HPR17S
    {0, 1, 2, 4, 5, 6},             // V_RED6: alpha1, u, v, rho1, rho2, p
    {0, 1, 2, 4, 5, 6, 7},          // V_MPH7: alpha1, u, v, rho1, p1, rho2, p2
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10},  // V_MRED11: every plane
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11},  // V_MINT12: every plane
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18},  // V_HRED19: every plane
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19},  // V_HINT20: every plane
    {0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15,
     16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31},  // V_HMPH32: every plane
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},  // V_MMPH16: every plane
};

}  // namespace

namespace vg {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace vg

namespace vg {
// Device-side fills of the planes a variant does not carry, for downloads into device memory.
__global__ void fill_plane_kernel(double* p, long n, double val) {
    const long i = blockIdx.x * 256L + threadIdx.x;
    if (i < n) p[i] = val;
}
// NaN into the `constant` planes of every cell whose `carried` planes hold a non-finite value.
__global__ void mark_nonfinite_kernel(double* planes, long n, int nref, unsigned carried, unsigned constant) {
    const long i = blockIdx.x * 256L + threadIdx.x;
    if (i >= n) return;
    bool bad = false;
    for (int r = 0; r < nref; r++)
        if (carried >> r & 1u) bad |= !isfinite(planes[(long)r * n + i]);
    if (bad)
        for (int r = 0; r < nref; r++)
            if (constant >> r & 1u) planes[(long)r * n + i] = __longlong_as_double(0x7ff8000000000000LL);
}
}  // namespace vg

struct vg_solver {
    vg_grid_desc d{};
    int dims = 2;
    int variant = -1;
    const Ops* ops = nullptr;
    long pitch = 0, plane = 0;
    int max_nw = 0;
    double* buf[2] = {nullptr, nullptr};
    double* aux = nullptr;    // source sub-cycle scratch: kAuxPlanes(max_nw) conserved planes
    int cur = 0;
    Ctrl* ctrl = nullptr;     // device
    Ctrl* hctrl = nullptr;    // pinned host mirror
    double* dout = nullptr;   // device scalar for max-wave results
    double* hout = nullptr;   // pinned host scalar
    double floor5 = 0.0;
    cudaStream_t cap = nullptr;  // private capture stream
    // graph cache: chunk of kChunk steps from buffer 0, and single steps from buffer 0 and 1
    struct GraphSet {
        bool valid = false;
        cudaGraphExec_t chunk = nullptr, single[2] = {nullptr, nullptr};
        vg_run_config cfg{};
        int variant = -1;
    } g;
    long last_launches = 0;
    int xcfg = 0, ycfg = 0;   // launch configuration of each sweep (sweep_table.cuh)
    int cfl_sep = 0;          // schedule: 0 folds the next step's CFL maximum into the last sweep, 1 a separate pass
    int yseg = 0;             // Y segments: 0 the shape's TY, 1 sized for whole waves (sweep_table.cuh)
    // TMA tensor maps over buf[0] and buf[1] for the TMA-staged X sweep (device memory; null: none)
    CUtensorMap* d_tmaps = nullptr;
    int tmap_planes = 0;
};

namespace {

constexpr int kChunk = 16;  // steps per captured chunk (even: a chunk returns to buffer 0 in 1D and 2D)

// Per-launch constants of a sweep: the ctrl slot of its length and, for a host-given dt, r / rinv / half_r.
SweepArgs prepared(const SweepArgs& a0) {
    SweepArgs a = a0;
    a.kslot = a.dt_scale == 0.5 ? 0 : 1;
    if (!a.ctrl) {
        vg::sweep_scale(a.dt_host * a.dt_scale, a.dx, a.r_host, a.rinv_host, a.half_r_host);
        a.r_host_f = (float)a.r_host;
        a.rinv_host_f = (float)a.rinv_host;
        a.half_r_host_f = (float)a.half_r_host;
    }
    return a;
}

// The tensor map over a.in for the TMA-staged X sweep, where the solver holds one for that buffer.
const void* tmap_for(const vg_solver* s, const double* in) {
    if (!s->d_tmaps || s->tmap_planes != s->ops->tma_planes) return nullptr;
    return in == s->buf[0] ? (const void*)&s->d_tmaps[0] : in == s->buf[1] ? (const void*)&s->d_tmaps[1] : nullptr;
}

cudaError_t run_sweep(const vg_solver* s, int axis, const SweepArgs& a0, cudaStream_t st) {
    SweepArgs a = prepared(a0);
    a.tmap = axis == 0 ? tmap_for(s, a.in) : nullptr;
    a.y_waves = s->yseg;
    return axis == 0 ? s->ops->x[s->xcfg](a, st) : s->ops->y[s->ycfg](a, st);
}

// Tensor maps of the TMA-staged X sweep over both state buffers: dims {nx, ny, planes}, row and plane strides in
// bytes, box {kTmaTile + 2, 2, planes} of FP64 with zero fill outside the grid.  The driver's encoder is reached
// through the runtime's entry-point query, so the library needs no link to libcuda.  On any failure the solver
// keeps no maps and the sweep shapes fall back to the plain two-row kernel.
void build_tmaps(vg_solver* s, int planes) {
    if (s->d_tmaps && s->tmap_planes == planes) return;
    s->tmap_planes = 0;
    PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&encode, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess || !encode)
        return;
    CUtensorMap maps[2];
    for (int b = 0; b < 2; b++) {
        const cuuint64_t dims[3] = {(cuuint64_t)s->d.nx, (cuuint64_t)s->d.ny, (cuuint64_t)planes};
        const cuuint64_t strides[2] = {(cuuint64_t)(s->pitch * sizeof(double)), (cuuint64_t)(s->plane * sizeof(double))};
        const cuuint32_t box[3] = {(cuuint32_t)(vg::kTmaTile + 2), 2u, (cuuint32_t)planes};
        const cuuint32_t estr[3] = {1u, 1u, 1u};
        if (encode(&maps[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, s->buf[b], dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return;
    }
    if (!s->d_tmaps && cudaMalloc(&s->d_tmaps, sizeof(maps)) != cudaSuccess) {
        s->d_tmaps = nullptr;
        return;
    }
    if (cudaMemcpy(s->d_tmaps, maps, sizeof(maps), cudaMemcpyHostToDevice) != cudaSuccess) return;
    s->tmap_planes = planes;
}

// In-process cache of tuned launch configurations keyed by variant, precision, grid and SM count;
// optionally persisted in the text file named by VG_TUNE_CACHE ("key xcfg ycfg" per line).
struct TuneEntry {
    std::string key;
    int xcfg, ycfg, sched, yseg;
};
std::vector<TuneEntry> g_tune_cache;
bool g_tune_loaded = false;

std::string tune_key(const vg_solver* s) {
    int dev = s->d.device, sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    char buf[160];
    std::snprintf(buf, sizeof(buf), "v%d_p%d_b%d_%dx%d_sm%d", s->variant, s->d.precision, s->d.boundary, s->d.nx,
                  s->d.ny, sms);
    return buf;
}

void tune_cache_load() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("VG_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char line[256], key[160];
    while (std::fgets(line, sizeof(line), f)) {
        int x, y, sc = 0, ys = 0;
        // lines without a schedule: fused; without a Y segment mode: the shape's TY
        const int got = std::sscanf(line, "%159s %d %d %d %d", key, &x, &y, &sc, &ys);
        if (got >= 3 && x >= 0 && x < vg::kNumXCfg && y >= 0 && y < vg::kNumYCfg && (sc == 0 || sc == 1) &&
            (ys == 0 || ys == 1))
            g_tune_cache.push_back({key, x, y, sc, ys});
    }
    std::fclose(f);
}

void tune_cache_store(const std::string& key, int x, int y, int sched, int yseg) {
    for (auto& e : g_tune_cache)
        if (e.key == key) {
            e.xcfg = x;
            e.ycfg = y;
            e.sched = sched;
            e.yseg = yseg;
            return;
        }
    g_tune_cache.push_back({key, x, y, sched, yseg});
    const char* path = std::getenv("VG_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d %d %d\n", key.c_str(), x, y, sched, yseg);
    std::fclose(f);
}

SweepArgs base_args(const vg_solver* s) {
    SweepArgs a{};
    a.plane = s->plane;
    a.pitch = s->pitch;
    a.nx = s->d.nx;
    a.ny = s->d.ny;
    a.periodic = s->d.boundary == VG_PERIODIC;
    a.ctrl = s->ctrl;
    a.dt_scale = 1.0;
    a.floor5 = s->floor5;
    a.dims = s->dims;
    a.wave_acc = &s->ctrl->smax_next;
    a.err = &s->ctrl->err;
    a.aux = s->aux;
    for (int i = 0; i < VG_MAX_PARAMS - 1; i++) a.params[i] = s->d.params[i];
    a.params[VG_MAX_PARAMS - 1] = 1.0 / (s->d.params[0] - 1.0);
    static_assert(vg::kParams == VG_MAX_PARAMS, "device parameter block must match VG_MAX_PARAMS");
    // the first-order loop's fixed GLM speed: MHD params[2], the MHD two-material models params[4] (both materials)
    a.ch_host = (s->d.model == VG_MODEL_MHD_REDUCED || s->d.model == VG_MODEL_MHD_INTERMEDIATE) ? s->d.params[4]
                                                                                              : s->d.params[2];
    return a;
}

// HPR relaxation source: `sub` out-of-place sub-cycles starting in buffer `from`; returns the buffer holding the
// result (Solvers/hprsecondordersolver.cpp:514-519, :532-537).
int enqueue_forcing(vg_solver* s, SweepArgs a, int sub, int from, cudaStream_t st, cudaError_t* e, int* n) {
    int b = from;
    for (int i = 0; i < sub && *e == cudaSuccess; i++) {
        a.in = s->buf[b];
        a.out = s->buf[1 - b];
        *e = s->ops->forcing(a, sub, st);
        *n += vg::kForcingLaunches;
        b = 1 - b;
    }
    return b;
}

// Enqueue one time step reading from buffer `from`; returns the number of kernels.  Every step makes an odd
// number of out-of-place passes (1 or 3 sweeps plus 2 * subcycles source passes), so it ends in buffer 1 - from.
int enqueue_step(vg_solver* s, const vg_run_config& c, int from, cudaStream_t st, cudaError_t* err) {
    SweepArgs a = base_args(s);
    a.dx = c.dx;
    a.bias = c.bias;
    a.limiter = c.limiter;
    // FirstOrderSolver's loop: FORCE sweeps, no source (its sub-cycle loop is empty), c_h as given
    const bool first = c.order == 1;
    a.ch_fixed = first;
    auto sweep = [&](int axis, const SweepArgs& sa) {
        if (!first) return run_sweep(s, axis, sa, st);
        return (axis == 0 ? s->ops->x1 : s->ops->y1)(prepared(sa), st);
    };
    int n = 0;
    cudaError_t e = s->ops->step_begin(a, st);
    n++;
    const bool stiff = !first && c.stiff_source && s->ops->relax;
    const bool reinit = c.reinit_frequency > 0 && s->ops->reinit;
    a.reinit_freq = c.reinit_frequency;
    const int sub = (!first && !stiff && s->ops->forcing && c.subcycles > 0) ? c.subcycles : 0;
    from = enqueue_forcing(s, a, sub, from, st, &e, &n);
    // stiff source: relaxation over dt/2 in place before and after the sweeps
    auto relax = [&]() {
        SweepArgs r = a;
        r.in = r.out = s->buf[from];
        r.dt_scale = 0.5;
        if (e == cudaSuccess) e = s->ops->relax(r, st);
        n++;
    };
    if (stiff) relax();
    // Without a trailing source pass the last sweep folds the next step's CFL maximum into its epilogue;
    // with one, a separate reduction runs after it.
    const int fuse_wave = sub == 0 && !stiff && !reinit && !s->cfl_sep;
    if (s->dims == 1) {
        a.in = s->buf[from];
        a.out = s->buf[1 - from];
        a.accumulate_wave = fuse_wave;
        a.advance_time = 1;
        if (e == cudaSuccess) e = sweep(0, a);
        n++;
        from = 1 - from;
    } else {
        // Solvers/secondordersolver.cpp:403-410: X(dt/2), Y(dt), X(dt/2)
        a.in = s->buf[from];
        a.out = s->buf[1 - from];
        a.dt_scale = 0.5;
        if (e == cudaSuccess) e = sweep(0, a);
        a.in = s->buf[1 - from];
        a.out = s->buf[from];
        a.dt_scale = 1.0;
        if (e == cudaSuccess) e = sweep(1, a);
        a.in = s->buf[from];
        a.out = s->buf[1 - from];
        a.dt_scale = 0.5;
        a.accumulate_wave = fuse_wave;
        a.advance_time = 1;
        if (e == cudaSuccess) e = sweep(0, a);
        n += 3;
        from = 1 - from;
    }
    a.dt_scale = 1.0;
    a.accumulate_wave = 0;
    a.advance_time = 0;
    from = enqueue_forcing(s, a, sub, from, st, &e, &n);
    if (stiff) relax();
    if (reinit) {  // in place on the step's result, before the next step's CFL maximum reads it
        SweepArgs r = a;
        r.in = r.out = s->buf[from];
        if (e == cudaSuccess) e = s->ops->reinit(r, st);
        n += s->dims == 1 ? 1 : 2;
    }
    if (!fuse_wave) {
        a.in = s->buf[from];
        if (e == cudaSuccess) e = s->ops->max_wave(a, st);
        n++;
    }
    *err = e;
    return n;
}

int kernels_per_step(const vg_solver* s, int sub, bool stiff = false, bool reinit = false) {
    int n = s->dims == 1 ? 2 : 4;                                                      // step_begin and the sweeps
    const bool forcing = !stiff && s->ops->forcing && sub > 0;
    if (forcing) n += 2 * sub * vg::kForcingLaunches;                                  // source sub-cycles
    if (stiff) n += 2;                                                                 // two relaxations
    if (reinit) n += s->dims == 1 ? 1 : 2;                                             // the reinitialisation
    if (forcing || stiff || reinit || s->cfl_sep) n += 1;                              // the separate CFL maximum
    return n;
}

void destroy_graphs(vg_solver* s) {
    if (s->g.chunk) cudaGraphExecDestroy(s->g.chunk);
    for (auto& x : s->g.single)
        if (x) cudaGraphExecDestroy(x);
    s->g = vg_solver::GraphSet{};
}

vg_status capture(vg_solver* s, const vg_run_config& c, int steps, int from, cudaGraphExec_t* out) {
    cudaGraph_t graph = nullptr;
    VG_CUDA(cudaStreamBeginCapture(s->cap, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    int b = from;
    for (int i = 0; i < steps && e == cudaSuccess; i++) {
        enqueue_step(s, c, b, s->cap, &e);
        b = 1 - b;
    }
    cudaError_t e2 = cudaStreamEndCapture(s->cap, &graph);
    if (e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(e, "kernel launch during capture");
    }
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    return VG_OK;
}

int order_of(const vg_run_config& c) { return c.order == 1 ? 1 : 2; }

bool same_cfg(const vg_run_config& a, const vg_run_config& b) {
    return a.dx == b.dx && a.bias == b.bias && a.limiter == b.limiter && a.subcycles == b.subcycles &&
           order_of(a) == order_of(b) && (a.stiff_source != 0) == (b.stiff_source != 0) &&
           a.reinit_frequency == b.reinit_frequency;
}

vg_status ensure_graphs(vg_solver* s, const vg_run_config& c) {
    if (s->g.valid && s->g.variant == s->variant && same_cfg(s->g.cfg, c)) return VG_OK;
    destroy_graphs(s);
    // the Y launchers look their occupancy up on first use: let them do it outside the capture
    if (s->dims == 2) {
        SweepArgs probe{};
        for (int i = 0; i < vg::kNumYCfg; i++) VG_CUDA(s->ops->y[i](probe, s->cap));
    }
    vg_status st;
    if ((st = capture(s, c, kChunk, 0, &s->g.chunk)) != VG_OK) return st;
    if ((st = capture(s, c, 1, 0, &s->g.single[0])) != VG_OK) return st;
    if ((st = capture(s, c, 1, 1, &s->g.single[1])) != VG_OK) return st;
    s->g.valid = true;
    s->g.cfg = c;
    s->g.variant = s->variant;
    return VG_OK;
}

// One plane between a pitched device buffer and a dense one (or any two buffers): a single linear copy when both
// are dense, a 2D copy otherwise.
cudaError_t copy_plane(double* dst, long dpitch, const double* src, long spitch, int nx, int ny, cudaMemcpyKind kind,
                       cudaStream_t st) {
    if (dpitch == nx && spitch == nx) return cudaMemcpyAsync(dst, src, sizeof(double) * nx * ny, kind, st);
    return cudaMemcpy2DAsync(dst, sizeof(double) * dpitch, src, sizeof(double) * spitch, sizeof(double) * nx, ny, kind,
                             st);
}

// The CFL maximum of the uploaded state; with_corners adds the default-constructed corner ghosts of a 2D grid.
vg_status max_wave_speed(vg_solver* s, double* out, bool with_corners, void* stream) {
    if (!s || !out) return fail(VG_EINVAL, "null argument");
    if (!s->ops) return fail(VG_EINVAL, "no state uploaded");
    cudaStream_t st = (cudaStream_t)stream;
    Ctrl* h = s->hctrl;
    std::memset(h, 0, sizeof(Ctrl));
    h->dims = with_corners ? s->dims : 0;  // the finishing kernel folds in the corner state for dims == 2 only
    VG_CUDA(cudaMemcpyAsync(s->ctrl, h, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    SweepArgs a = base_args(s);
    a.in = s->buf[s->cur];
    VG_CUDA(s->ops->max_wave(a, st));
    VG_CUDA(s->ops->max_wave_finish(a, s->dout, st));
    VG_CUDA(cudaMemcpyAsync(s->hout, s->dout, sizeof(double), cudaMemcpyDeviceToHost, st));
    VG_CUDA(cudaStreamSynchronize(st));
    *out = *s->hout;
    s->last_launches = 2;
    return VG_OK;
}
}  // namespace

extern "C" {

int vg_model_nvar(int model) { return ref_nvar(model); }

const char* vg_last_error_string(void) { return g_last_error.c_str(); }

const char* vg_status_string(vg_status st) {
    switch (st) {
        case VG_OK: return "VG_OK";
        case VG_EINVAL: return "VG_EINVAL";
        case VG_ENAN: return "VG_ENAN";
        case VG_ETIMEOUT: return "VG_ETIMEOUT";
        case VG_ECUDA: return "VG_ECUDA";
        case VG_ENOMEM: return "VG_ENOMEM";
        case VG_EUNSUPPORTED: return "VG_EUNSUPPORTED";
    }
    return "unknown vg_status";
}

vg_status vg_create(const vg_grid_desc* desc, vg_solver** out) {
    if (!desc || !out) return fail(VG_EINVAL, "null argument");
    *out = nullptr;
    if (desc->model != VG_MODEL_EULER && desc->model != VG_MODEL_MHD && desc->model != VG_MODEL_HPR &&
        desc->model != VG_MODEL_EULER_REDUCED && desc->model != VG_MODEL_EULER_MULTIPHYSICS &&
        desc->model != VG_MODEL_MHD_REDUCED && desc->model != VG_MODEL_MHD_INTERMEDIATE &&
        desc->model != VG_MODEL_HPR_REDUCED && desc->model != VG_MODEL_HPR_INTERMEDIATE &&
        desc->model != VG_MODEL_HPR_MULTIPHYSICS && desc->model != VG_MODEL_MHD_MULTIPHYSICS)
        return fail(VG_EUNSUPPORTED, "model not available in this build");
    if (desc->nx < 2 || desc->ny < 1 || (desc->ny > 1 && desc->ny < 2))
        return fail(VG_EINVAL, "grid needs at least 2 cells along every swept axis");
    if (desc->precision != VG_FP64 && desc->precision != VG_MIXED) return fail(VG_EINVAL, "bad precision");
    if (desc->boundary != VG_TRANSMISSIVE && desc->boundary != VG_PERIODIC) return fail(VG_EINVAL, "bad boundary");
    if (desc->precision == VG_MIXED && !vg::ops_mixed(vg::V_EULER2))
        return fail(VG_EUNSUPPORTED, "mixed precision not available in this build");
    if (desc->precision == VG_MIXED && desc->model == VG_MODEL_EULER_MULTIPHYSICS)
        return fail(VG_EUNSUPPORTED, "the multiphysics two-material model runs in VG_FP64 only (its trace material's "
                                     "energy is not stable under FP32 flux values)");
    if (desc->precision == VG_MIXED && (desc->model == VG_MODEL_MHD_REDUCED || desc->model == VG_MODEL_MHD_INTERMEDIATE))
        return fail(VG_EUNSUPPORTED, "the MHD two-material models run in VG_FP64 only");
    if (desc->precision == VG_MIXED && (desc->model == VG_MODEL_HPR_REDUCED || desc->model == VG_MODEL_HPR_INTERMEDIATE ||
                                        desc->model == VG_MODEL_HPR_MULTIPHYSICS))
        return fail(VG_EUNSUPPORTED, "the HPR two-material models run in VG_FP64 only");
    if ((desc->model == VG_MODEL_HPR_MULTIPHYSICS || desc->model == VG_MODEL_MHD_MULTIPHYSICS) && desc->ny != 1)
        return fail(VG_EUNSUPPORTED, "the multiphysics two-material models of HPR and MHD are 1D (ny = 1), as the "
                                     "reference's are");
    if (desc->precision == VG_MIXED && desc->model == VG_MODEL_MHD_MULTIPHYSICS)
        return fail(VG_EUNSUPPORTED, "the MHD two-material models run in VG_FP64 only");
    if (desc->model == VG_MODEL_HPR) {
        const double eos = desc->params[12];
        if (eos != 0.0 && eos != 1.0 && eos != 2.0)
            return fail(VG_EINVAL, "HPR params[12] (equation of state) must be 0 StiffenedGas, 1 ShockMieGruneisen or 2 "
                                   "GodunovRomenski");
    }
    VG_CUDA(cudaSetDevice(desc->device));
    vg_solver* s = new (std::nothrow) vg_solver();
    if (!s) return fail(VG_ENOMEM, "host allocation");
    s->d = *desc;
    s->dims = desc->ny > 1 ? 2 : 1;
    s->max_nw = desc->model == VG_MODEL_EULER ? 4 : desc->model == VG_MODEL_MHD ? 9 : desc->model == VG_MODEL_EULER_REDUCED ? 6
                : desc->model == VG_MODEL_EULER_MULTIPHYSICS ? 7 : desc->model == VG_MODEL_MHD_REDUCED ? 11
                : desc->model == VG_MODEL_MHD_INTERMEDIATE ? 12 : desc->model == VG_MODEL_HPR_REDUCED ? 19
                : desc->model == VG_MODEL_HPR_INTERMEDIATE ? 20 : desc->model == VG_MODEL_HPR_MULTIPHYSICS ? 32
                : desc->model == VG_MODEL_MHD_MULTIPHYSICS ? 16 : 17;
    s->pitch = ((long)desc->nx + 31) / 32 * 32;  // 256-byte aligned rows
    s->plane = s->pitch * desc->ny;
    s->floor5 = std::pow(10.0, -5.0);  // SlopeLimiters::computeSlopeVector's floor (Solvers/slopelimiters.cpp:232-239)
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; b++) e = cudaMalloc(&s->buf[b], sizeof(double) * s->plane * s->max_nw);
    if (e == cudaSuccess && desc->model != VG_MODEL_EULER)  // scratch of the source sub-cycles (conserved planes)
        e = cudaMalloc(&s->aux, sizeof(double) * s->plane * vg::aux_planes(s->max_nw));
    if (e == cudaSuccess) e = cudaMalloc(&s->ctrl, sizeof(Ctrl));
    if (e == cudaSuccess) e = cudaMalloc(&s->dout, sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&s->hctrl, sizeof(Ctrl));
    if (e == cudaSuccess) e = cudaMallocHost(&s->hout, sizeof(double));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemset(s->ctrl, 0, sizeof(Ctrl));
    if (e != cudaSuccess) {
        vg_destroy(s);
        return cuda_fail(e, "vg_create allocation");
    }
    *out = s;
    return VG_OK;
}

vg_status vg_destroy(vg_solver* s) {
    if (!s) return VG_OK;
    destroy_graphs(s);
    for (auto& b : s->buf)
        if (b) cudaFree(b);
    if (s->aux) cudaFree(s->aux);
    if (s->d_tmaps) cudaFree(s->d_tmaps);
    if (s->ctrl) cudaFree(s->ctrl);
    if (s->dout) cudaFree(s->dout);
    if (s->hctrl) cudaFreeHost(s->hctrl);
    if (s->hout) cudaFreeHost(s->hout);
    if (s->cap) cudaStreamDestroy(s->cap);
    delete s;
    return VG_OK;
}

vg_status vg_upload_primitive(vg_solver* s, const double* planes, int is_device, void* stream) {
    if (!s || !planes) return fail(VG_EINVAL, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const long n = (long)s->d.nx * s->d.ny;
    const int model = s->d.model;
    // Planes the compiled variants do not carry must hold their constant (0, or Euler's lambda = 1).  Where the
    // variant does not depend on them, the check runs on host threads while the carried planes are in flight;
    // where it does (1D Euler's v, MHD's w and Bz), it runs first.
    int variant;
    std::vector<const double*> zero_planes;
    const double* one_plane = nullptr;
    bool check_after = false;
    if (model == VG_MODEL_EULER) {
        if (is_device) {
            variant = vg::V_EULER2;  // device input cannot be scanned on the host: carry v, trust w and lambda
        } else if (s->dims == 2) {
            variant = vg::V_EULER2;
            zero_planes = {planes + 3 * n};
            one_plane = planes + 5 * n;
            check_after = true;
        } else {
            if (vg::host::any_differs({planes + 3 * n}, 0.0, n) || vg::host::any_differs({planes + 5 * n}, 1.0, n))
                return fail(VG_EUNSUPPORTED, "Euler state with w != 0 or lambda != 1 needs the 6-component variant");
            variant = vg::host::any_differs({planes + 2 * n}, 0.0, n) ? vg::V_EULER2 : vg::V_EULER1;
        }
    } else if (model == VG_MODEL_EULER_REDUCED || model == VG_MODEL_EULER_MULTIPHYSICS) {
        // the two-material models carry every plane but w, which must be 0
        if (!is_device) {
            zero_planes = {planes + 3 * n};
            check_after = true;
        }
        variant = model == VG_MODEL_EULER_REDUCED ? vg::V_RED6 : vg::V_MPH7;
    } else if (model == VG_MODEL_MHD_REDUCED) {
        variant = vg::V_MRED11;
    } else if (model == VG_MODEL_MHD_INTERMEDIATE) {
        variant = vg::V_MINT12;
    } else if (model == VG_MODEL_HPR_REDUCED) {
        variant = vg::V_HRED19;
    } else if (model == VG_MODEL_HPR_INTERMEDIATE) {
        variant = vg::V_HINT20;
    } else if (model == VG_MODEL_HPR_MULTIPHYSICS) {
        variant = vg::V_HMPH32;
    } else if (model == VG_MODEL_MHD_MULTIPHYSICS) {
        variant = vg::V_MMPH16;
    } else if (model == VG_MODEL_HPR) {
        // a solid equation of state or plasticity selects the instantiation that carries them
        variant = (s->d.params[12] != 0.0 || s->d.params[17] != 0.0) ? vg::V_HPR17S : vg::V_HPR17;
    } else {
        const bool reduced = !is_device && !vg::host::any_differs({planes + 3 * n, planes + 7 * n}, 0.0, n);
        variant = reduced ? vg::V_MHD7 : vg::V_MHD9;
    }
    const Ops* ops = s->d.precision == VG_MIXED ? vg::ops_mixed(variant) : vg::ops_fp64(variant);
    if (!ops) return fail(VG_EUNSUPPORTED, "no kernel variant for this state");
    // the device state is replaced from here on: until this call succeeds the solver holds none
    s->ops = nullptr;
    s->variant = variant;
    s->cur = 0;
    if (ops->tma_planes > 0) build_tmaps(s, ops->tma_planes);
    bool bad = false;
    std::thread checker;
    if (check_after)
        checker = std::thread([&]() {
            bad = vg::host::any_differs(zero_planes, 0.0, n) || (one_plane && vg::host::any_differs({one_plane}, 1.0, n));
        });
    const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < ops->nw && e == cudaSuccess; k++)
        e = copy_plane(s->buf[0] + k * s->plane, s->pitch, planes + (long)kPlanes[variant][k] * n, s->d.nx, s->d.nx,
                       s->d.ny, kind, st);
    // HPRReducedStateVector::setPrimitiveVariableVector (HPR/Multiphysics/hprreducedstatevector.cpp:78-104) and
    // HPRIntermediateStateVector's (hprintermediatestatevector.cpp:82-110) take J only when either material is
    // thermal; otherwise the cells keep the default J = 0, which nothing reads
    if (e == cudaSuccess && (variant == vg::V_HRED19 || variant == vg::V_HINT20) && s->d.params[11] == 0.0 &&
        s->d.params[31] == 0.0)
        e = cudaMemsetAsync(s->buf[0] + (variant == vg::V_HRED19 ? 14 : 13) * s->plane, 0, sizeof(double) * 3 * s->plane,
                            st);
    // HPRMultiphysicsStateVector::setPrimitiveVariableVector (hprmultiphysicsstatevector.cpp:98-139) takes each
    // material's J only when that material is thermal
    for (int k = 0; k < 2 && variant == vg::V_HMPH32; k++)
        if (e == cudaSuccess && s->d.params[20 * k + 11] == 0.0)
            e = cudaMemsetAsync(s->buf[0] + (15 + 14 * k) * s->plane, 0, sizeof(double) * 3 * s->plane, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(&s->ctrl->err, 0, sizeof(unsigned), st);  // a fresh state: no error yet
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (checker.joinable()) checker.join();
    if (e != cudaSuccess) return cuda_fail(e, "vg_upload_primitive");
    if (bad) {
        if (model == VG_MODEL_EULER)
            return fail(VG_EUNSUPPORTED, "Euler state with w != 0 or lambda != 1 needs the 6-component variant");
        return fail(VG_EUNSUPPORTED, "two-material state with w != 0");
    }
    s->ops = ops;
    return VG_OK;
}

vg_status vg_download_primitive(vg_solver* s, double* planes, int is_device, void* stream) {
    if (!s || !planes) return fail(VG_EINVAL, "null argument");
    if (!s->ops) return fail(VG_EINVAL, "no state uploaded");
    cudaStream_t st = (cudaStream_t)stream;
    const long n = (long)s->d.nx * s->d.ny;
    const int nref = ref_nvar(s->d.model);
    unsigned carried = 0, constant = 0;
    const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    // the error word of the runs and sweeps since the upload: set when a cell became non-finite (or unphysical)
    VG_CUDA(cudaMemcpyAsync(&s->hctrl->err, &s->ctrl->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    for (int k = 0; k < s->ops->nw; k++) {
        int r = kPlanes[s->variant][k];
        carried |= 1u << r;
        VG_CUDA(copy_plane(planes + (long)r * n, s->d.nx, s->buf[s->cur] + k * s->plane, s->pitch, s->d.nx, s->d.ny,
                           kind, st));
    }
    // planes that are not carried hold their constant value (0, or lambda = 1): filled while the copies run
    for (int r = 0; r < nref; r++) {
        if (carried >> r & 1u) continue;
        constant |= 1u << r;
        const double val = (s->d.model == VG_MODEL_EULER && r == 5) ? 1.0 : 0.0;
        if (is_device) {
            vg::fill_plane_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(planes + (long)r * n, n, val);
            VG_CUDA(cudaGetLastError());
        } else {
            vg::host::fill_plane(planes + (long)r * n, val, n);
        }
    }
    VG_CUDA(cudaStreamSynchronize(st));
    // HPRMultiphysicsStateVector::computePrimitiveVariableVector (hprmultiphysicsstatevector.cpp:204-249) returns a
    // cold material's J as 0; the device state keeps the J that the reinitialisation mixes in, as the reference's
    // cells do
    if (s->variant == vg::V_HMPH32) {
        for (int k = 0; k < 2; k++) {
            if (s->d.params[20 * k + 11] != 0.0) continue;
            for (int r = 15 + 14 * k; r < 18 + 14 * k; r++) {
                if (is_device) {
                    vg::fill_plane_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(planes + (long)r * n, n, 0.0);
                    VG_CUDA(cudaGetLastError());
                } else {
                    vg::host::fill_plane(planes + (long)r * n, 0.0, n);
                }
            }
        }
        VG_CUDA(cudaStreamSynchronize(st));
    }
    // The reference recovers every primitive of a cell from its conserved vector (setConservedVariableVector), so
    // once a cell's state is non-finite its w = (rho w) / rho and lambda = (rho lambda) / rho (MHD: w, Bz) are NaN
    // as well; the constants above hold only where the carried state is finite.
    if (constant && s->hctrl->err) {
        if (is_device) {
            vg::mark_nonfinite_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(planes, n, nref, carried, constant);
            VG_CUDA(cudaGetLastError());
            VG_CUDA(cudaStreamSynchronize(st));
        } else {
            vg::host::mark_nonfinite(planes, n, nref, carried, constant);
        }
    }
    return VG_OK;
}

vg_status vg_run(vg_solver* s, const vg_run_config* cfg, int* steps_taken, double* t_reached, void* stream) {
    if (!s || !cfg) return fail(VG_EINVAL, "null argument");
    if (!s->ops) return fail(VG_EINVAL, "no state uploaded");
    if (!(cfg->dx > 0.0) || !(cfg->cfl > 0.0)) return fail(VG_EINVAL, "dx and cfl must be positive");
    if (cfg->max_steps <= 0 && !(cfg->t_end > 0.0)) return fail(VG_EINVAL, "need t_end > 0 or max_steps > 0");
    if (cfg->subcycles < 0) return fail(VG_EINVAL, "subcycles must be >= 0");
    // HPRSecondOrderSolver::solve of the HPR multiphysics model takes subcyclingIterations and runs an empty loop
    // (Solvers/hprsecondordersolver.cpp:368-373, :378-383); MHDSecondOrderSolver::solve of the MHD multiphysics model
    // takes subcyclingIterations and reinitialisationFrequency and uses neither (Solvers/mhdsecondordersolver.cpp:
    // 362-385): accepted and ignored, as there
    const bool multiphysics = s->d.model == VG_MODEL_HPR_MULTIPHYSICS || s->d.model == VG_MODEL_MHD_MULTIPHYSICS;
    if (cfg->subcycles > 0 && !s->ops->forcing && !multiphysics)
        return fail(VG_EUNSUPPORTED, "source sub-cycling needs a model with a source (HPR relaxation, MHD GLM damping)");
    if (cfg->order != 0 && cfg->order != 1 && cfg->order != 2) return fail(VG_EINVAL, "order must be 1 or 2");
    if (cfg->order == 1 && !s->ops->x1) return fail(VG_EUNSUPPORTED, "this kernel form has no first-order loop");
    if (cfg->stiff_source && cfg->order != 1 && !s->ops->relax)
        return fail(VG_EUNSUPPORTED, "the stiff source relaxation exists for the HPR model only");
    if (cfg->reinit_frequency < 0) return fail(VG_EINVAL, "reinit_frequency must be >= 0");
    if (cfg->reinit_frequency > 0 && (!s->ops->reinit || cfg->order == 1) && s->d.model != VG_MODEL_MHD_MULTIPHYSICS)
        return fail(VG_EUNSUPPORTED, "volume-fraction reinitialisation belongs to the reduced two-material model's "
                                     "second-order loop");
    if (cfg->stiff_source && cfg->order != 1 && s->d.params[17] != 0.0)
        return fail(VG_EUNSUPPORTED, "the stiff source relaxation integrates the elastic strain relaxation only; plastic "
                                     "materials run the RK4 source sub-cycles");
    cudaStream_t st = (cudaStream_t)stream;
    VG_CUDA(cudaSetDevice(s->d.device));

    // A plain second-order run of a small 1D row runs in one launch (solve1d_kernels.cuh): the whole loop on the
    // chip, in a cluster of blocks that share the row through distributed shared memory
    const bool plain = cfg->order != 1 && !(cfg->stiff_source && s->ops->relax) && !(cfg->subcycles > 0 && s->ops->forcing) &&
                       !(cfg->reinit_frequency > 0 && s->ops->reinit);
    if (plain && s->ops->solve1d && s->dims == 1 && s->d.nx >= s->ops->solve1d_min && s->d.nx <= s->ops->solve1d_max) {
        Ctrl* h = s->hctrl;
        std::memset(h, 0, sizeof(Ctrl));
        h->t_end = cfg->t_end > 0.0 ? cfg->t_end : 1.0e300;
        h->cfl = cfg->cfl;
        h->dx = cfg->dx;
        h->max_steps = cfg->max_steps > 0 ? cfg->max_steps : INT_MAX;
        h->active = 1;
        h->dims = 1;
        VG_CUDA(cudaMemcpyAsync(s->ctrl, h, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
        SweepArgs a = base_args(s);
        a.in = a.out = s->buf[s->cur];
        a.dx = cfg->dx;
        a.bias = cfg->bias;
        a.limiter = cfg->limiter;
        VG_CUDA(s->ops->solve1d(a, st));
        VG_CUDA(cudaMemcpyAsync(h, s->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
        VG_CUDA(cudaStreamSynchronize(st));
        s->last_launches = 1;
        if (steps_taken) *steps_taken = h->it;
        if (t_reached) *t_reached = h->t;
        if (h->err) return fail(VG_ENAN, "non-finite value, non-positive density or pressure at or below -p_inf produced");
        if (h->t < h->t_end && h->it < h->max_steps)
            return fail(VG_EINVAL, "the time step stopped advancing: the one-launch 1D loop ended at its step cap");
        return VG_OK;
    }

    // Normalise so that the state starts in buffer 0 (graphs are captured from buffer 0).
    if (s->cur != 0) {
        VG_CUDA(cudaMemcpyAsync(s->buf[0], s->buf[1], sizeof(double) * s->plane * s->ops->nw, cudaMemcpyDeviceToDevice, st));
        s->cur = 0;
    }
    vg_status vs = ensure_graphs(s, *cfg);
    if (vs != VG_OK) return vs;

    Ctrl* h = s->hctrl;
    std::memset(h, 0, sizeof(Ctrl));
    h->t_end = cfg->t_end > 0.0 ? cfg->t_end : 1.0e300;
    h->cfl = cfg->cfl;
    h->dx = cfg->dx;
    h->max_steps = cfg->max_steps > 0 ? cfg->max_steps : INT_MAX;
    h->active = 1;
    h->dims = s->dims;
    VG_CUDA(cudaMemcpyAsync(s->ctrl, h, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    SweepArgs a = base_args(s);
    a.in = s->buf[0];
    a.dx = cfg->dx;
    VG_CUDA(s->ops->max_wave(a, st));
    long launches = 1;

    long launched_steps = 0;
    if (cfg->max_steps > 0 && !(cfg->t_end > 0.0)) {
        // step-count run: exactly max_steps steps
        long k = cfg->max_steps;
        for (; k >= kChunk; k -= kChunk) {
            VG_CUDA(cudaGraphLaunch(s->g.chunk, st));
            launched_steps += kChunk;
        }
        int b = 0;
        for (; k > 0; k--) {
            VG_CUDA(cudaGraphLaunch(s->g.single[b], st));
            b = 1 - b;
            launched_steps++;
        }
    } else {
        // time-driven run: chunks until the device reports the end (steps past it are copies)
        for (;;) {
            VG_CUDA(cudaGraphLaunch(s->g.chunk, st));
            launched_steps += kChunk;
            VG_CUDA(cudaMemcpyAsync(h, s->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
            VG_CUDA(cudaStreamSynchronize(st));
            if (!(h->t < h->t_end) || h->it >= h->max_steps) break;
        }
    }
    const bool stiff = cfg->order != 1 && cfg->stiff_source && s->ops->relax;
    launches += launched_steps * kernels_per_step(s, cfg->order == 1 || stiff ? 0 : cfg->subcycles, stiff,
                                                  cfg->order != 1 && cfg->reinit_frequency > 0 && s->ops->reinit);
    // every step is an odd number of sweeps in 2D (3) and 1 in 1D: the state ends in buffer (steps & 1)
    s->cur = (int)(launched_steps & 1);
    VG_CUDA(cudaMemcpyAsync(h, s->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    VG_CUDA(cudaStreamSynchronize(st));
    s->last_launches = launches;
    if (steps_taken) *steps_taken = h->it;
    if (t_reached) *t_reached = h->t;
    if (h->err & vg::ERR_TIMEOUT) return fail(VG_ETIMEOUT, "a bounded wait of the TMA-staged sweep gave up");
    if (h->err) return fail(VG_ENAN, "non-finite value, non-positive density or pressure at or below -p_inf produced");
    return VG_OK;
}

vg_status vg_solve(vg_solver* s, const double* planes_in, double* planes_out, const vg_run_config* cfg, int* steps_taken,
                   double* t_reached, void* stream) {
    vg_status st = vg_upload_primitive(s, planes_in, 0, stream);
    if (st != VG_OK) return st;
    vg_status rs = vg_run(s, cfg, steps_taken, t_reached, stream);
    if (rs != VG_OK && rs != VG_ENAN) return rs;
    st = vg_download_primitive(s, planes_out, 0, stream);
    return st != VG_OK ? st : rs;
}

vg_status vg_sweep(vg_solver* s, int axis, double dx, double dt, double bias, int limiter, void* stream) {
    if (!s) return fail(VG_EINVAL, "null solver");
    if (!s->ops) return fail(VG_EINVAL, "no state uploaded");
    if (axis != 0 && axis != 1) return fail(VG_EINVAL, "axis must be 0 or 1");
    if (axis == 1 && s->dims == 1) return fail(VG_EINVAL, "Y sweep on a 1D grid");
    if (!(dx > 0.0) || !(dt > 0.0)) return fail(VG_EINVAL, "dx and dt must be positive");
    cudaStream_t st = (cudaStream_t)stream;
    SweepArgs a = base_args(s);
    a.ctrl = nullptr;
    a.dt_host = dt;
    a.dx = dx;
    a.bias = bias;
    a.limiter = limiter;
    a.in = s->buf[s->cur];
    a.out = s->buf[1 - s->cur];
    VG_CUDA(run_sweep(s, axis, a, st));
    s->cur = 1 - s->cur;
    s->last_launches = 1;
    return VG_OK;
}

vg_status vg_max_wave_speed(vg_solver* s, double* out, void* stream) { return max_wave_speed(s, out, true, stream); }

vg_status vg_max_wave_speed_cells(vg_solver* s, double* out, void* stream) {
    return max_wave_speed(s, out, false, stream);
}

vg_status vg_state_device(vg_solver* s, double** plane0, long* plane_stride, long* row_stride, int* nplanes) {
    if (!s) return fail(VG_EINVAL, "null solver");
    if (plane0) *plane0 = s->buf[s->cur];
    if (plane_stride) *plane_stride = s->plane;
    if (row_stride) *row_stride = s->pitch;
    if (nplanes) *nplanes = s->ops ? s->ops->nw : 0;
    return VG_OK;
}

long vg_last_launch_count(vg_solver* s) { return s ? s->last_launches : 0; }

vg_status vg_set_launch_config(vg_solver* s, int xcfg, int ycfg) {
    if (!s) return fail(VG_EINVAL, "null solver");
    if (xcfg < 0 || xcfg >= vg::kNumXCfg || ycfg < 0 || ycfg >= vg::kNumYCfg)
        return fail(VG_EINVAL, "launch configuration index out of range");
    if (s->xcfg != xcfg || s->ycfg != ycfg) destroy_graphs(s);
    s->xcfg = xcfg;
    s->ycfg = ycfg;
    return VG_OK;
}

vg_status vg_get_launch_config(vg_solver* s, int* xcfg, int* ycfg, const char** xname, const char** yname) {
    if (!s) return fail(VG_EINVAL, "null solver");
    if (xcfg) *xcfg = s->xcfg;
    if (ycfg) *ycfg = s->ycfg;
    const int kind = s->ops ? s->ops->tile_kind : 0;
    if (xname) *xname = vg::x_cfg_name(s->xcfg, kind);
    if (yname) *yname = vg::y_cfg_name(s->ycfg, kind);
    return VG_OK;
}

vg_status vg_autotune(vg_solver* s, const vg_run_config* cfg, int reps, float* times_ms, void* stream) {
    if (!s || !cfg) return fail(VG_EINVAL, "null argument");
    if (!s->ops) return fail(VG_EINVAL, "no state uploaded");
    if (!(cfg->dx > 0.0)) return fail(VG_EINVAL, "dx must be positive");
    if (reps < 1) reps = 3;
    tune_cache_load();
    std::string key = tune_key(s);
    if (!times_ms) {
        for (auto& e : g_tune_cache)
            if (e.key == key) {
                vg_status vs = vg_set_launch_config(s, e.xcfg, e.ycfg);
                if (vs == VG_OK && s->yseg != e.yseg) {
                    destroy_graphs(s);
                    s->yseg = e.yseg;
                }
                return vs != VG_OK ? vs : vg_set_schedule(s, e.sched);
            }
    }
    cudaStream_t st = (cudaStream_t)stream;
    // Time every candidate on the uploaded state: out-of-place sweeps into the spare buffer, with the
    // time step the current state would take (so the limiter and flux paths are the ones a run takes).
    double smax = 0.0;
    vg_status vs = vg_max_wave_speed(s, &smax, stream);
    if (vs != VG_OK) return vs;
    double dt = cfg->cfl * (cfg->dx / (smax > 0.0 ? smax : 1.0));
    SweepArgs a = base_args(s);
    a.ctrl = nullptr;
    a.dt_host = dt;
    a.dx = cfg->dx;
    a.bias = cfg->bias;
    a.limiter = cfg->limiter;
    a.in = s->buf[s->cur];
    a.out = s->buf[1 - s->cur];
    a = prepared(a);
    cudaEvent_t e0, e1;
    VG_CUDA(cudaEventCreate(&e0));
    VG_CUDA(cudaEventCreate(&e1));
    float best[2] = {1e30f, 1e30f};
    int pick[2] = {0, 0}, pick_yseg = 0;
    for (int axis = 0; axis < s->dims; axis++) {
        int n = axis == 0 ? vg::kNumXCfg : vg::kNumYCfg;
        // each Y shape is timed with its own segment length and with segments sized for whole waves
        for (int c = 0; c < n * (axis == 0 ? 1 : 2); c++) {
            const int shape = c % n;
            const vg::SweepFn fn = axis == 0 ? s->ops->x[shape] : s->ops->y[shape];
            a.tmap = axis == 0 ? tmap_for(s, a.in) : nullptr;
            a.y_waves = axis == 1 && c >= n;
            cudaError_t e = fn(a, st);  // warm-up (module load, caches)
            if (e != cudaSuccess) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return cuda_fail(e, "autotune launch");
            }
            VG_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < reps; r++) fn(a, st);
            VG_CUDA(cudaEventRecord(e1, st));
            VG_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            VG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms /= reps;
            float& slot_ms = times_ms ? times_ms[axis * vg::kNumXCfg + shape] : ms;
            if (times_ms && (c < n || ms < slot_ms)) slot_ms = ms;  // a shape's time: the better of its two modes
            if (ms < best[axis]) {
                best[axis] = ms;
                pick[axis] = shape;
                if (axis == 1) pick_yseg = c >= n;
            }
        }
    }
    a.y_waves = 0;
    // Schedule: where the next step's CFL maximum is taken.  Folded into the last X sweep's epilogue it costs no
    // extra pass over the state but adds the wave speed's registers to the sweep; a separate reduction reads the
    // state once more.  Both give the same bits (the maximum of the same values); time the step's tail each way
    // with the chosen X shape.
    int sched = 0;
    {
        const vg::SweepFn xfn = s->ops->x[pick[0]];
        a.tmap = tmap_for(s, a.in);
        float t2[2] = {0.0f, 0.0f};
        for (int sc = 0; sc < 2; sc++) {
            SweepArgs b = a;
            b.accumulate_wave = sc == 0;
            SweepArgs m = base_args(s);
            m.in = a.out;
            auto tail = [&]() {
                cudaError_t e = xfn(b, st);
                if (sc == 1 && e == cudaSuccess) e = s->ops->max_wave(m, st);
                return e;
            };
            cudaError_t e = tail();  // warm-up
            if (e != cudaSuccess) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return cuda_fail(e, "autotune launch");
            }
            VG_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < reps; r++) tail();
            VG_CUDA(cudaEventRecord(e1, st));
            VG_CUDA(cudaEventSynchronize(e1));
            VG_CUDA(cudaEventElapsedTime(&t2[sc], e0, e1));
            t2[sc] /= reps;
            if (times_ms) times_ms[vg::kNumXCfg + vg::kNumYCfg + sc] = t2[sc];
        }
        sched = t2[1] < t2[0] ? 1 : 0;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    VG_CUDA(cudaGetLastError());
    tune_cache_store(key, pick[0], pick[1], sched, pick_yseg);
    vg_status vs2 = vg_set_launch_config(s, pick[0], pick[1]);
    if (vs2 == VG_OK && s->yseg != pick_yseg) {
        destroy_graphs(s);
        s->yseg = pick_yseg;
    }
    return vs2 != VG_OK ? vs2 : vg_set_schedule(s, sched);
}

vg_status vg_set_schedule(vg_solver* s, int cfl_separate) {
    if (!s) return fail(VG_EINVAL, "null solver");
    if (cfl_separate != 0 && cfl_separate != 1) return fail(VG_EINVAL, "cfl_separate must be 0 or 1");
    if (s->cfl_sep != cfl_separate) destroy_graphs(s);
    s->cfl_sep = cfl_separate;
    return VG_OK;
}

vg_status vg_get_schedule(vg_solver* s, int* cfl_separate) {
    if (!s || !cfl_separate) return fail(VG_EINVAL, "null argument");
    *cfl_separate = s->cfl_sep;
    return VG_OK;
}

}  // extern "C"
