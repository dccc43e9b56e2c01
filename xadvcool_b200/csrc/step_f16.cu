// Fused step kernels with __half population storage (see step_kernels.cuh).
#include "step_kernels.cuh"

namespace xac {
template void launch_coupled_step<__half>(const StepLaunch&);
}  // namespace xac
