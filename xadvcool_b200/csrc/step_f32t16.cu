// Fused step kernels with float fluid populations and __half thermal populations (see step_kernels.cuh).
#include "step_kernels.cuh"

namespace xac {
template void launch_coupled_step<float, __half>(const StepLaunch&);
}  // namespace xac
