// passes_ni.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 512.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(512)
}  // namespace pd
