// Fused step kernels with __half populations in both lattices (see step_kernels.cuh).
#include "step_kernels.cuh"

namespace xac {
template void launch_coupled_step<__half, __half>(const StepLaunch&);
}  // namespace xac
