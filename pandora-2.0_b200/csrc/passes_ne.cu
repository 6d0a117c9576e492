// passes_ne.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 192, 224.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(192)
PD_PASSES_INST(224)
}  // namespace pd
