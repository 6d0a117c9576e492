// passes_nh.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 448.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(448)
}  // namespace pd
