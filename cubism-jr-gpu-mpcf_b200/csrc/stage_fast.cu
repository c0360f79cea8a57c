// stage_fast.cu -- stage kernels of the fast FP32, mixed and FP64 policies.
// Built with fused multiply-adds allowed; the fast FP32 policies also use
// approximate division and square root (-prec-div=false -prec-sqrt=false),
// which leaves the double-precision operations of PolFP64 and of the mixed
// pressure recovery untouched.
#include "mpcf_stage.cuh"
#include "mpcf_launch.h"

namespace mpcf {

template <class Pol, int TY, bool P>
static const void* fn() { return (const void*)stage_kernel<Pol, TY, P>; }

template <class Pol, int TY, bool P>
static cudaError_t launch_one(const StageArgs& A, int grid, cudaStream_t st)
{
    stage_kernel<Pol, TY, P><<<grid, kTX * TY, stage_smem_bytes<typename Pol::T, TY>(), st>>>(A);
    return cudaGetLastError();
}

template <class Pol>
static cudaError_t launch_pol(int ty, bool persist, const StageArgs& A, int grid, cudaStream_t st)
{
    switch (ty)
    {
        case 2:  return persist ? launch_one<Pol, 2, true>(A, grid, st)  : launch_one<Pol, 2, false>(A, grid, st);
        case 4:  return persist ? launch_one<Pol, 4, true>(A, grid, st)  : launch_one<Pol, 4, false>(A, grid, st);
        case 8:  return persist ? launch_one<Pol, 8, true>(A, grid, st)  : launch_one<Pol, 8, false>(A, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

template <class Pol>
static StageKernelInfo info_pol(int ty, bool persist)
{
    typedef typename Pol::T T;
    StageKernelInfo I = {nullptr, 0};
    switch (ty)
    {
        case 2: I.fn = persist ? fn<Pol, 2, true>() : fn<Pol, 2, false>(); I.smem = stage_smem_bytes<T, 2>(); break;
        case 4: I.fn = persist ? fn<Pol, 4, true>() : fn<Pol, 4, false>(); I.smem = stage_smem_bytes<T, 4>(); break;
        case 8: I.fn = persist ? fn<Pol, 8, true>() : fn<Pol, 8, false>(); I.smem = stage_smem_bytes<T, 8>(); break;
        default: break;
    }
    return I;
}

cudaError_t launch_stage_fast(int pol, int ty, bool persist, const StageArgs& A, int grid, cudaStream_t st)
{
    switch (pol)
    {
        case 1: return launch_pol<PolFast32>(ty, persist, A, grid, st);
        case 2: return launch_pol<PolMixed>(ty, persist, A, grid, st);
        case 3: return launch_pol<PolFP64>(ty, persist, A, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

StageKernelInfo stage_info_fast(int pol, int ty, bool persist)
{
    switch (pol)
    {
        case 1: return info_pol<PolFast32>(ty, persist);
        case 2: return info_pol<PolMixed>(ty, persist);
        case 3: return info_pol<PolFP64>(ty, persist);
        default: { StageKernelInfo I = {nullptr, 0}; return I; }
    }
}

} // namespace mpcf
