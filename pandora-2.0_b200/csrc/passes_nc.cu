// passes_nc.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 80, 96, 112.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(80)
PD_PASSES_INST(96)
PD_PASSES_INST(112)
}  // namespace pd
