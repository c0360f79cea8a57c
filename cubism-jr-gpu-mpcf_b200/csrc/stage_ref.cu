// stage_ref.cu -- the bit-exact FP32 stage kernel (PolRef32).
//
// This translation unit MUST be compiled with --fmad=false (no contraction
// of multiplies and adds into FMA), -prec-div=true, -prec-sqrt=true and
// -ftz=false: every floating-point operation then rounds like the literal
// C semantics of the reference source, so the results are bit-identical to
// the CPU restatement.  The build refuses to compile it otherwise.
#include "mpcf_stage.cuh"
#include "mpcf_launch.h"

#if defined(__CUDA_ARCH__) && !defined(MPCF_NO_FMAD)
#error "stage_ref.cu must be built with --fmad=false -DMPCF_NO_FMAD"
#endif

namespace mpcf {

template <int TY, bool P>
static const void* fn() { return (const void*)stage_kernel<PolRef32, TY, P>; }

template <int TY, bool P>
static cudaError_t launch_one(const StageArgs& A, int grid, cudaStream_t st)
{
    stage_kernel<PolRef32, TY, P><<<grid, kTX * TY, stage_smem_bytes<float, TY>(), st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_stage_ref(int ty, bool persist, const StageArgs& A, int grid, cudaStream_t st)
{
    switch (ty)
    {
        case 2:  return persist ? launch_one<2, true>(A, grid, st)  : launch_one<2, false>(A, grid, st);
        case 4:  return persist ? launch_one<4, true>(A, grid, st)  : launch_one<4, false>(A, grid, st);
        case 8:  return persist ? launch_one<8, true>(A, grid, st)  : launch_one<8, false>(A, grid, st);
        case 16: return persist ? launch_one<16, true>(A, grid, st) : launch_one<16, false>(A, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

StageKernelInfo stage_info_ref(int ty, bool persist)
{
    StageKernelInfo I = {nullptr, 0};
    switch (ty)
    {
        case 2:  I.fn = persist ? fn<2, true>()  : fn<2, false>();  I.smem = stage_smem_bytes<float, 2>();  break;
        case 4:  I.fn = persist ? fn<4, true>()  : fn<4, false>();  I.smem = stage_smem_bytes<float, 4>();  break;
        case 8:  I.fn = persist ? fn<8, true>()  : fn<8, false>();  I.smem = stage_smem_bytes<float, 8>();  break;
        case 16: I.fn = persist ? fn<16, true>() : fn<16, false>(); I.smem = stage_smem_bytes<float, 16>(); break;
        default: break;
    }
    return I;
}

} // namespace mpcf
