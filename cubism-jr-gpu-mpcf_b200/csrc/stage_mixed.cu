// stage_mixed.cu -- stage kernels of the PolMixed precision policy (one
// translation unit per policy, so they compile in parallel).  Built with
// fused multiply-adds allowed; the single-precision policies also use
// approximate division and square root (-prec-div=false -prec-sqrt=false),
// which leaves double-precision operations untouched.
#include "stage_dispatch.cuh"

namespace mpcf {

cudaError_t launch_stage_mixed(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st)
{
    return StageDispatch<PolMixed, false>::launch(ty, persist, tma, A, grid, st);
}

StageKernelInfo stage_info_mixed(int ty, bool persist, bool sums, bool tma)
{
    return StageDispatch<PolMixed, false>::info(ty, persist, sums, tma);
}

} // namespace mpcf
