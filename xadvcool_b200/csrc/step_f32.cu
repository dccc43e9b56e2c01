// Fused step kernels with float population storage (see step_kernels.cuh).
#include "step_kernels.cuh"

namespace xac {
template void launch_coupled_step<float>(const StepLaunch&);
}  // namespace xac
