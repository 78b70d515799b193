// The exact-FP64 form's table of kernel sets, one entry per model variant.  The kernels themselves are instantiated
// in the slic_fp64_*.cu units (every one compiled with -fmad=false), a few models per unit.
#include "vg_ops.h"

namespace vg {

Ops fp64_ops_euler1();
Ops fp64_ops_euler2();
Ops fp64_ops_mhd7();
Ops fp64_ops_mhd9();
Ops fp64_ops_hpr17();
Ops fp64_ops_hpr17s();
Ops fp64_ops_red6();
Ops fp64_ops_mph7();
Ops fp64_ops_mred11();
Ops fp64_ops_mint12();
Ops fp64_ops_hred19();
Ops fp64_ops_hint20();
Ops fp64_ops_hmph32();
Ops fp64_ops_mmph16();

const Ops* ops_fp64(int variant) {
    static const Ops table[V_COUNT] = {
        fp64_ops_euler1(), fp64_ops_euler2(), fp64_ops_mhd7(),  fp64_ops_mhd9(),   fp64_ops_hpr17(),  fp64_ops_hpr17s(),
        fp64_ops_red6(),   fp64_ops_mph7(),   fp64_ops_mred11(), fp64_ops_mint12(), fp64_ops_hred19(), fp64_ops_hint20(),
        fp64_ops_hmph32(), fp64_ops_mmph16(),
    };
    return (variant >= 0 && variant < V_COUNT) ? &table[variant] : nullptr;
}

}  // namespace vg
