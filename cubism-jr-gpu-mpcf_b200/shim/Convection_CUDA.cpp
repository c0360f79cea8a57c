// Convection_CUDA.cpp -- the convection facade on the fused stage kernel:
// a stage with b = 0 computes the register (a*R - dtinvh*L(U)) and leaves
// U_next = U + 0*R = U, so Convection_CUDA followed by Update_CUDA is
// bit-identical to one fused stage (Convection_CUDA.cpp:15-23 of the
// reference launches _xflux.._divergence; the update is a separate kernel).
#include "Convection_CUDA.h"
#include "GPU.h"
#include "../../include/mpcf_b200.h"

Convection_CUDA::Convection_CUDA(const Real a_, const Real dtinvh_) : a(a_), dtinvh(dtinvh_) {}

void Convection_CUDA::compute(const uint_t /*nslices*/, const uint_t /*global_iz*/)
{
    mpcf_solver* s = GPU::current_solver();
    if (!s) GPU::check(MPCF_ERR_STATE, "Convection_CUDA: no GPUlab");
    const double d = (double)dtinvh;
    GPU::check(mpcf_stage(s, (double)a, 0.0, &d), "Convection_CUDA");
}
