// MaxSpeedOfSound_CUDA.h -- sound-speed facade (source/MaxSpeedOfSound_CUDA.h:13-17).
#pragma once

#include "Types.h"

class MaxSpeedOfSound_CUDA
{
public:
    // maximum speed of sound of the whole block; the result is available
    // from GPU::last_max_sos() (the reference leaves it in mapped memory that
    // GPUlab::max_sos reads, GPUlab.cpp:691-697)
    void compute(const uint_t nslices);
};
