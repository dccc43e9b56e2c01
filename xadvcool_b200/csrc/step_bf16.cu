// Fused step kernels with __nv_bfloat16 population storage (see step_kernels.cuh).
#include "step_kernels.cuh"

namespace xac {
template void launch_coupled_step<__nv_bfloat16>(const StepLaunch&);
}  // namespace xac
