// stage_fast64.cu -- stage kernels of the PolFast64 precision policy (one
// translation unit per policy, so they compile in parallel): double storage
// and arithmetic with the fast forms' factored algebra and refined double
// reciprocals.  Built with fused multiply-adds allowed.
#include "stage_dispatch.cuh"

namespace mpcf {

cudaError_t launch_stage_fast64(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st)
{
    return StageDispatch<PolFast64, false>::launch(ty, persist, tma, A, grid, st);
}

StageKernelInfo stage_info_fast64(int ty, bool persist, bool sums, bool tma)
{
    return StageDispatch<PolFast64, false>::info(ty, persist, sums, tma);
}

} // namespace mpcf
