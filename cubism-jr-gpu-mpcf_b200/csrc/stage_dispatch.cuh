// stage_dispatch.cuh -- maps a runtime launch configuration (tile height,
// persistent or not, conservation sums or not, bulk-tensor-copy staging or
// not) onto the stage_kernel template instances of one precision policy.
#pragma once

#include "mpcf_stage.cuh"
#include "mpcf_launch.h"

namespace mpcf {

template <class Pol, bool kWithTY15>
struct StageDispatch
{
    typedef typename Pol::T T;

    template <int TY, bool P, bool S, bool M>
    static cudaError_t go(const StageArgs& A, int grid, cudaStream_t st)
    {
        stage_kernel<Pol, TY, P, S, M><<<grid, stage_threads<TY>(), stage_smem_bytes<Pol, TY, M>(), st>>>(A);
        return cudaGetLastError();
    }

    template <int TY, bool M>
    static cudaError_t go_ty(bool persist, const StageArgs& A, int grid, cudaStream_t st)
    {
        const bool sums = A.tile_sums != nullptr;
        if (persist) return sums ? go<TY, true, true, M>(A, grid, st) : go<TY, true, false, M>(A, grid, st);
        return sums ? go<TY, false, true, M>(A, grid, st) : go<TY, false, false, M>(A, grid, st);
    }

    template <int TY, bool M>
    static StageKernelInfo info_ty(bool persist, bool sums)
    {
        StageKernelInfo I;
        I.smem = stage_smem_bytes<Pol, TY, M>();
        if (persist) I.fn = sums ? (const void*)stage_kernel<Pol, TY, true, true, M> : (const void*)stage_kernel<Pol, TY, true, false, M>;
        else         I.fn = sums ? (const void*)stage_kernel<Pol, TY, false, true, M> : (const void*)stage_kernel<Pol, TY, false, false, M>;
        return I;
    }

    static cudaError_t launch(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st)
    {
        switch (ty)
        {
            case 3: return tma ? go_ty<3, true>(persist, A, grid, st) : go_ty<3, false>(persist, A, grid, st);
            case 7: return tma ? go_ty<7, true>(persist, A, grid, st) : go_ty<7, false>(persist, A, grid, st);
            case 8: return tma ? go_ty<8, true>(persist, A, grid, st) : go_ty<8, false>(persist, A, grid, st);
            case 15:
                if (kWithTY15)
                    return tma ? go_ty<kWithTY15 ? 15 : 7, true>(persist, A, grid, st)
                               : go_ty<kWithTY15 ? 15 : 7, false>(persist, A, grid, st);
                return cudaErrorInvalidValue;
            default: return cudaErrorInvalidValue;
        }
    }

    static StageKernelInfo info(int ty, bool persist, bool sums, bool tma)
    {
        switch (ty)
        {
            case 3: return tma ? info_ty<3, true>(persist, sums) : info_ty<3, false>(persist, sums);
            case 7: return tma ? info_ty<7, true>(persist, sums) : info_ty<7, false>(persist, sums);
            case 8: return tma ? info_ty<8, true>(persist, sums) : info_ty<8, false>(persist, sums);
            case 15:
                if (kWithTY15)
                    return tma ? info_ty<kWithTY15 ? 15 : 7, true>(persist, sums) : info_ty<kWithTY15 ? 15 : 7, false>(persist, sums);
                { StageKernelInfo I = {nullptr, 0}; return I; }
            default: { StageKernelInfo I = {nullptr, 0}; return I; }
        }
    }
};

} // namespace mpcf
