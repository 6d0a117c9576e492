// passes_nj.cu -- the pass launchers (and through them the kernels) of the transform
// lengths 640, 768.
#include "passes_n.cuh"

namespace pd {
PD_PASSES_INST(640)
PD_PASSES_INST(768)
}  // namespace pd
