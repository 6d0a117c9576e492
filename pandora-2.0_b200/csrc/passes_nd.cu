// passes_nd.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 128, 160.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(128)
PD_PASSES_INST(160)
}  // namespace pd
