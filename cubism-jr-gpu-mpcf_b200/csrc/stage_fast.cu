// stage_fast.cu -- stage kernels of the fast FP32, mixed and FP64 policies.
// Built with fused multiply-adds allowed; the fast FP32 policies also use
// approximate division and square root (-prec-div=false -prec-sqrt=false),
// which leaves the double-precision operations of PolFP64 and of the mixed
// pressure recovery untouched.
#include "mpcf_stage.cuh"
#include "mpcf_launch.h"
#include "stage_dispatch.cuh"

namespace mpcf {

cudaError_t launch_stage_fast(int pol, int ty, bool persist, const StageArgs& A, int grid, cudaStream_t st)
{
    switch (pol)
    {
        case 1: return StageDispatch<PolFast32, false>::launch(ty, persist, A, grid, st);
        case 2: return StageDispatch<PolMixed, false>::launch(ty, persist, A, grid, st);
        case 3: return StageDispatch<PolFP64, false>::launch(ty, persist, A, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

StageKernelInfo stage_info_fast(int pol, int ty, bool persist, bool sums)
{
    switch (pol)
    {
        case 1: return StageDispatch<PolFast32, false>::info(ty, persist, sums);
        case 2: return StageDispatch<PolMixed, false>::info(ty, persist, sums);
        case 3: return StageDispatch<PolFP64, false>::info(ty, persist, sums);
        default: { StageKernelInfo I = {nullptr, 0}; return I; }
    }
}

} // namespace mpcf
