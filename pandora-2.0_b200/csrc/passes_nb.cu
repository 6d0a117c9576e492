// passes_nb.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 48, 56, 64.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(48)
PD_PASSES_INST(56)
PD_PASSES_INST(64)
}  // namespace pd
