// stage_ref_w3.cu -- the bit-exact FP32 stage kernel with the reference's
// compile-time WENO3 reconstruction (PolRef32W3).  Compiled like
// stage_ref.cu: no contraction, IEEE division and square root, no flushing.
#include "stage_dispatch.cuh"

#if defined(__CUDA_ARCH__) && !defined(MPCF_NO_FMAD)
#error "stage_ref_w3.cu must be built with --fmad=false -DMPCF_NO_FMAD"
#endif

namespace mpcf {

cudaError_t launch_stage_ref_w3(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st)
{
    return StageDispatch<PolRef32W3, true>::launch(ty, persist, tma, A, grid, st);
}

StageKernelInfo stage_info_ref_w3(int ty, bool persist, bool sums, bool tma)
{
    return StageDispatch<PolRef32W3, true>::info(ty, persist, sums, tma);
}

} // namespace mpcf
