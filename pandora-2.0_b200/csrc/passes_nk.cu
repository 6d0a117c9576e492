// passes_nk.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 896, 1024.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(896)
PD_PASSES_INST(1024)
}  // namespace pd
