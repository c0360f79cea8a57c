// stage_fp64_w3.cu -- the FP64 stage kernel with the reference's compile-time
// WENO3 reconstruction (PolFP64W3), built like stage_fp64.cu.
#include "stage_dispatch.cuh"

namespace mpcf {

cudaError_t launch_stage_fp64_w3(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st)
{
    return StageDispatch<PolFP64W3, false>::launch(ty, persist, tma, A, grid, st);
}

StageKernelInfo stage_info_fp64_w3(int ty, bool persist, bool sums, bool tma)
{
    return StageDispatch<PolFP64W3, false>::info(ty, persist, sums, tma);
}

} // namespace mpcf
