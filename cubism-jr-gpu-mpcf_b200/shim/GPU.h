// GPU.h -- the host-visible GPU seam of the reference (source/GPU/GPU.h:38-85)
// on top of libmpcf_b200.  The reference kept its device buffers as
// process-wide singletons behind these free functions; here the device
// state belongs to a solver (include/mpcf_b200.h) and the seam holds the
// solver of the most recently constructed GPUlab, which the kernel facades
// (Convection_CUDA, Update_CUDA, MaxSpeedOfSound_CUDA) act on.
//
// The reference's per-chunk transfer and per-direction kernel wrappers
// (h2d_3DArray, xflux, yflux, zflux, divergence, bind_textures, ...) have no
// counterpart: the state is device resident and one fused kernel evaluates
// all three directions, the divergence and the update.
#pragma once

#include "Types.h"

struct mpcf_solver;

namespace GPU
{
    enum streamID { S1, S2 };

    void syncGPU();
    void syncStream(streamID s);
    void tell_memUsage_GPU();
    void tell_GPU();

    // solver the facades act on (set by the GPUlab constructor)
    mpcf_solver* current_solver();
    void set_current_solver(mpcf_solver* s);
    // result of the last MaxSpeedOfSound_CUDA::compute
    float last_max_sos();
    void set_last_max_sos(float v);
    // aborts with the library's message on a failed call (the reference's
    // failure behaviour: message on stderr, exit(1))
    void check(int rc, const char* what);
}
