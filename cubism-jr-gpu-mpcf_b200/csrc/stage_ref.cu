// stage_ref.cu -- the bit-exact FP32 stage kernel (PolRef32).
//
// This translation unit MUST be compiled with --fmad=false (no contraction
// of multiplies and adds into FMA), -prec-div=true, -prec-sqrt=true and
// -ftz=false: every floating-point operation then rounds like the literal
// C semantics of the reference source, so the results are bit-identical to
// the CPU restatement.  The build refuses to compile it otherwise.
#include "stage_dispatch.cuh"

#if defined(__CUDA_ARCH__) && !defined(MPCF_NO_FMAD)
#error "stage_ref.cu must be built with --fmad=false -DMPCF_NO_FMAD"
#endif

namespace mpcf {

cudaError_t launch_stage_ref(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st)
{
    return StageDispatch<PolRef32, true>::launch(ty, persist, tma, A, grid, st);
}

StageKernelInfo stage_info_ref(int ty, bool persist, bool sums, bool tma)
{
    return StageDispatch<PolRef32, true>::info(ty, persist, sums, tma);
}

} // namespace mpcf
