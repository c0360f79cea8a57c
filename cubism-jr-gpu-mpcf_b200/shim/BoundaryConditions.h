// BoundaryConditions.h -- the reference's boundary-condition interface
// (source/BoundaryConditions.h:19-109) on the B200 path.
//
// In the reference, applyBC_absorbing / applyBC_reflecting fill the host
// halo buffers of a GPUlab (3 ghost layers per face) from the host state,
// and the halos travel over PCIe with every stage.  On the B200 path the
// ghost layers are synthesised inside the stage kernel from the same rules
// (absorbing: zeroth-order extrapolation; reflecting: mirror with the
// normal momentum negated), so these calls record the face condition on
// the lab that owns the halo.  GPUlab subclasses that override _apply_bc
// with these calls (every GPUlab* case of the reference) run unchanged.
#pragma once

#include "Types.h"

class GPUlab;

namespace mpcf_shim
{
    // implemented in GPUlab.cpp
    void record_bc(const RealPtrVec_t* halo, int dir, int side, int type);
}

template <typename TGrid>
class BoundaryConditions
{
protected:
    const RealPtrVec_t& pdata;
    const uint_t startZ, deltaZ;

public:
    BoundaryConditions(const RealPtrVec_t& data, const uint_t first_slice_iz = 0, const uint_t n_slices = TGrid::sizeZ)
        : pdata(data), startZ(first_slice_iz), deltaZ(n_slices) {}

    template <int dir, int side, index_map map>
    void applyBC_absorbing(RealPtrVec_t& halo) { mpcf_shim::record_bc(&halo, dir, side, 0); }

    template <int dir, int side, index_map map>
    void applyBC_reflecting(RealPtrVec_t& halo) { mpcf_shim::record_bc(&halo, dir, side, 1); }
};
