// Update_CUDA.h -- update facade (source/Update_CUDA.h:13-27).
#pragma once

#include "Types.h"

class Update_CUDA
{
protected:
    Real m_b;

public:
    Update_CUDA(const Real b = 1) : m_b(b) {}

    // U <- U + b*register for the whole block
    void compute(const int nslices);
};
