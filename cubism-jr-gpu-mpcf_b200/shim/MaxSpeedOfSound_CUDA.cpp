// MaxSpeedOfSound_CUDA.cpp -- warp-shuffle / block / atomic maximum of the
// speed of sound on the device (the reference's _maxSOS,
// GPUkernels.cu:1182-1222, launched by MaxSpeedOfSound_CUDA.cpp:13-18).
#include "MaxSpeedOfSound_CUDA.h"
#include "GPU.h"
#include "../../include/mpcf_b200.h"

void MaxSpeedOfSound_CUDA::compute(const uint_t /*nslices*/)
{
    mpcf_solver* s = GPU::current_solver();
    if (!s) GPU::check(MPCF_ERR_STATE, "MaxSpeedOfSound_CUDA: no GPUlab");
    double v = 0;
    GPU::check(mpcf_max_sos(s, &v), "MaxSpeedOfSound_CUDA");
    GPU::set_last_max_sos((float)v);
}
