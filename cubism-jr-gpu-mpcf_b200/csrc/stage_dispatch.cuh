// stage_dispatch.cuh -- maps a runtime launch configuration (tile height,
// persistent or not, conservation sums or not) onto the stage_kernel
// template instances of one precision policy.
#pragma once

#include "mpcf_stage.cuh"
#include "mpcf_launch.h"

namespace mpcf {

template <class Pol, bool kWithTY16>
struct StageDispatch
{
    typedef typename Pol::T T;

    template <int TY, bool P, bool S>
    static cudaError_t go(const StageArgs& A, int grid, cudaStream_t st)
    {
        stage_kernel<Pol, TY, P, S><<<grid, kTX * TY, stage_smem_bytes<T, TY>(), st>>>(A);
        return cudaGetLastError();
    }

    template <int TY>
    static cudaError_t go_ty(bool persist, const StageArgs& A, int grid, cudaStream_t st)
    {
        const bool sums = A.tile_sums != nullptr;
        if (persist) return sums ? go<TY, true, true>(A, grid, st) : go<TY, true, false>(A, grid, st);
        return sums ? go<TY, false, true>(A, grid, st) : go<TY, false, false>(A, grid, st);
    }

    template <int TY>
    static StageKernelInfo info_ty(bool persist, bool sums)
    {
        StageKernelInfo I;
        I.smem = stage_smem_bytes<T, TY>();
        if (persist) I.fn = sums ? (const void*)stage_kernel<Pol, TY, true, true> : (const void*)stage_kernel<Pol, TY, true, false>;
        else         I.fn = sums ? (const void*)stage_kernel<Pol, TY, false, true> : (const void*)stage_kernel<Pol, TY, false, false>;
        return I;
    }

    static cudaError_t launch(int ty, bool persist, const StageArgs& A, int grid, cudaStream_t st)
    {
        switch (ty)
        {
            case 2: return go_ty<2>(persist, A, grid, st);
            case 4: return go_ty<4>(persist, A, grid, st);
            case 8: return go_ty<8>(persist, A, grid, st);
            case 16: if (kWithTY16) return go_ty<kWithTY16 ? 16 : 8>(persist, A, grid, st);
            default: return cudaErrorInvalidValue;
        }
    }

    static StageKernelInfo info(int ty, bool persist, bool sums)
    {
        switch (ty)
        {
            case 2: return info_ty<2>(persist, sums);
            case 4: return info_ty<4>(persist, sums);
            case 8: return info_ty<8>(persist, sums);
            case 16: if (kWithTY16) return info_ty<kWithTY16 ? 16 : 8>(persist, sums);
            default: { StageKernelInfo I = {nullptr, 0}; return I; }
        }
    }
};

} // namespace mpcf
