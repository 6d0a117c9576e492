// passes_ng.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 320, 384.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(320)
PD_PASSES_INST(384)
}  // namespace pd
