// passes_nf.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 256.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(256)
}  // namespace pd
