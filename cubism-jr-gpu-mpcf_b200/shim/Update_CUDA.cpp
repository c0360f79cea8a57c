// Update_CUDA.cpp -- U <- b*R + U (the reference's _update,
// GPUkernels.cu:1142-1179, launched by Update_CUDA.cpp:12-17).
#include "Update_CUDA.h"
#include "GPU.h"
#include "../../include/mpcf_b200.h"

void Update_CUDA::compute(const int /*nslices*/)
{
    mpcf_solver* s = GPU::current_solver();
    if (!s) GPU::check(MPCF_ERR_STATE, "Update_CUDA: no GPUlab");
    GPU::check(mpcf_update(s, (double)m_b), "Update_CUDA");
}
