// passes_na.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 16, 24, 32, 40.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(16)
PD_PASSES_INST(24)
PD_PASSES_INST(32)
PD_PASSES_INST(40)
}  // namespace pd
