// Convection_CUDA.h -- convection facade (source/Convection_CUDA.h:14-25).
#pragma once

#include "Types.h"

class Convection_CUDA
{
public:
    const Real a, dtinvh;   // LSRK3 "a" factor and dt/h

    Convection_CUDA(const Real a, const Real dtinvh);

    // register <- a*register - dtinvh*div F(U) for the whole block; the state
    // is left as it is (the update is Update_CUDA's)
    void compute(const uint_t nslices, const uint_t global_iz);
};
