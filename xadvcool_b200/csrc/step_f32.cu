// Fused step kernels with float population storage in both lattices (see step_kernels.cuh).
#include "step_kernels.cuh"

namespace xac {
template void launch_coupled_step<float, float>(const StepLaunch&);
}  // namespace xac
