// Mixed FP32/FP64 SLIC kernels.
#include "vg_ops.h"

namespace vg {

const Ops* ops_mixed(int /*variant*/) { return nullptr; }

}  // namespace vg
