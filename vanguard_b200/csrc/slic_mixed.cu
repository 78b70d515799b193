// Mixed FP32/FP64 SLIC kernels (VG_MIXED).  Compiled with FMA contraction on.
#include "physics_mixed.cuh"
#include "slic_kernels.cuh"
#include "slic_mixed.cuh"
#include "slic_tma.cuh"
#include "first_order_mixed.cuh"
#include "sweep_table.cuh"
#include "vg_ops.h"

namespace vg {
namespace {

constexpr int MW_NT = 256;

struct MixedKernels {
    template <class M, int P, int LPB, int MINB>
    static void x(dim3 grid, int nt, cudaStream_t st, const SweepArgs& a) {
        if constexpr (M::PAIR_X) {
            dim3 g(grid.x, (a.ny + 2 * LPB - 1) / (2 * LPB));
            sweep_x_pair_kernel<M, P, LPB, MINB><<<g, nt, 0, st>>>(a);
        } else {
            sweep_x_mixed_kernel<M, P, LPB, MINB><<<grid, nt, 0, st>>>(a);
        }
    }
    // persistent: as many blocks as fit on the device at once, or one per tile
    template <class M, int P, int MINB>
    static void x_tma(cudaStream_t st, const SweepArgs& a) {
        static int resident = 0;
        if (resident == 0) {
            int per_sm = 0, sms = 0, dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_x_tma_kernel<M, P, MINB>, P, 0);
            resident = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
        }
        const long tiles = (long)((a.nx + P - 3) / (P - 2)) * ((a.ny + 1) / 2);
        const int grid = (int)(tiles < resident ? tiles : resident);
        sweep_x_tma_kernel<M, P, MINB><<<grid, P, 0, st>>>(a);
    }
    template <class M, int TX, int TY, int MINB>
    static int y_resident() {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, sweep_y_mixed_kernel<M, TX, TY, MINB>, TX, 0);
        return b;
    }
    template <class M, int TX, int TY, int MINB>
    static void y(dim3 grid, int nt, cudaStream_t st, const SweepArgs& a) {
        sweep_y_mixed_kernel<M, TX, TY, MINB><<<grid, nt, 0, st>>>(a);
    }
};

template <class M>
cudaError_t max_wave_impl(const SweepArgs& a, cudaStream_t st) {
    long n = (long)a.nx * a.ny;
    int blocks = (int)((n + MW_NT - 1) / MW_NT);
    if (blocks > 148 * 8) blocks = 148 * 8;
    max_wave_kernel<M, MW_NT><<<blocks, MW_NT, 0, st>>>(a.in, a.plane, a.pitch, a.nx, a.ny, a.ctrl, a);
    return cudaGetLastError();
}

template <class M>
cudaError_t step_begin_impl(const SweepArgs& a, cudaStream_t st) {
    step_begin_kernel<M><<<1, 32, 0, st>>>(a.ctrl, a);
    return cudaGetLastError();
}

template <class M>
cudaError_t finish_impl(const SweepArgs& a, double* out, cudaStream_t st) {
    max_wave_finish_kernel<M><<<1, 32, 0, st>>>(a.ctrl, a, out);
    return cudaGetLastError();
}

template <class M>
cudaError_t force1_x(const SweepArgs& a, cudaStream_t st) {
    constexpr int P = 128;
    force1_x_mixed_kernel<M, P><<<dim3((a.nx + P - 1) / P, a.ny), P, 0, st>>>(a);
    return cudaGetLastError();
}

template <class M>
cudaError_t force1_y(const SweepArgs& a, cudaStream_t st) {
    if constexpr (!M::HAS_Y) {
        return cudaErrorInvalidValue;
    } else {
        constexpr int TX = 64, TY = 64;
        force1_y_mixed_kernel<M, TX, TY><<<dim3((a.nx + TX - 1) / TX, (a.ny + TY - 1) / TY), TX, 0, st>>>(a);
        return cudaGetLastError();
    }
}

using ForcingFn = cudaError_t (*)(const SweepArgs&, int, cudaStream_t);

// The source sub-cycles keep FP64: the exact forcing kernels of each model
template <class M>
constexpr Ops make_ops(ForcingFn forcing = nullptr, SweepFn relax = nullptr, SweepFn reinit = nullptr) {
    return Ops{M::NW, SweepTable<MixedKernels, M>::x, SweepTable<MixedKernels, M>::y, &max_wave_impl<M>,
               &step_begin_impl<M>, &finish_impl<M>, forcing, tile_kind<M>(), &force1_x<M>, &force1_y<M>, relax,
               tile_kind<M>() == 2 ? M::NW : 0, reinit};
}

const Ops kOps[V_COUNT] = {
    make_ops<EulerF32<1>>(),
    make_ops<EulerF32<2>>(),
    make_ops<MHDF32>(&mhd7_forcing_fp64),
    make_ops<MHDMixed<true>>(&mhd9_forcing_fp64),
    make_ops<HPRF32>(&hpr_forcing_fp64, &hpr_relax_fp64),
    make_ops<HPRSolidMixed>(&hpr_solid_forcing_fp64, &hpr_solid_relax_fp64),
    make_ops<ReducedMixed>(nullptr, nullptr, &reduced_reinit_fp64),
    Ops{},  // V_MPH7: no mixed form (see ops_mixed)
    Ops{},  // V_MRED11: no mixed form
    Ops{},  // V_MINT12: no mixed form
    Ops{},  // V_HRED19: no mixed form
    Ops{},  // V_HINT20: no mixed form
    Ops{},  // V_HMPH32: no mixed form
    Ops{},  // V_MMPH16: no mixed form
};

}  // namespace

// The multiphysics two-material model has no mixed form: its trace material (volume fraction clamped at 0.001)
// recovers its energy from the ratio of two tiny conserved components, which FP32 flux values perturb enough to
// give negative pressures where FP64 does not.
const Ops* ops_mixed(int variant) {
    return (variant >= 0 && variant < V_COUNT && kOps[variant].nw > 0) ? &kOps[variant] : nullptr;
}

}  // namespace vg
