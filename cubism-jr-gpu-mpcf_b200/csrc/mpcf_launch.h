// mpcf_launch.h -- internal launch interface between the host runtime and
// the kernel translation units (not part of the public C ABI).
#pragma once

#include <cuda_runtime.h>
#include "mpcf_types.h"

// records the calling thread's last error message (mpcf_last_error) and
// returns `code`; defined in mpcf_api.cu
int mpcf_fail_external(int code, const char* fmt, ...);

namespace mpcf {

struct StageKernelInfo
{
    const void* fn;     // kernel entry (for occupancy queries / attributes)
    size_t smem;        // dynamic shared memory per CTA
};

// precision policy ids: 0 FP32 reference rounding, 1 fast FP32, 2 mixed, 3 FP64,
// 4 fast FP64
cudaError_t launch_stage_ref(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st);
cudaError_t launch_stage_fast32(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st);
cudaError_t launch_stage_mixed(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st);
cudaError_t launch_stage_fp64(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st);
cudaError_t launch_stage_fast64(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st);
// the reference's compile-time WENO3 build of the reference-rounding forms
cudaError_t launch_stage_ref_w3(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st);
cudaError_t launch_stage_fp64_w3(int ty, bool persist, bool tma, const StageArgs& A, int grid, cudaStream_t st);
StageKernelInfo stage_info_ref(int ty, bool persist, bool sums, bool tma);
StageKernelInfo stage_info_fast32(int ty, bool persist, bool sums, bool tma);
StageKernelInfo stage_info_mixed(int ty, bool persist, bool sums, bool tma);
StageKernelInfo stage_info_fp64(int ty, bool persist, bool sums, bool tma);
StageKernelInfo stage_info_fast64(int ty, bool persist, bool sums, bool tma);
StageKernelInfo stage_info_ref_w3(int ty, bool persist, bool sums, bool tma);
StageKernelInfo stage_info_fp64_w3(int ty, bool persist, bool sums, bool tma);

// mpcf_aux.cu
cudaError_t launch_sos(int pol, const SosArgs& A, cudaStream_t st);
cudaError_t launch_dt(int pol, const DtArgs& A, cudaStream_t st);
cudaError_t launch_sum_tiles(const DomDev* doms, int ndom, const double* tile_sums, double* out, cudaStream_t st);
// Interleaved output arrays of the reference's dump (kind 0, 9 channels) and
// save (kind 1, 7 channels) for slabs [z0, z1), and the restart direction.
cudaError_t launch_pack(int is_double, int kind, const DomDev* dom, int parity, int z0, int z1, void* out, cudaStream_t st);
cudaError_t launch_unpack_save(int is_double, const DomDev* dom, int parity, int z0, int z1, const void* in, cudaStream_t st);

// SteadyState, Sod and 2DSBI initial conditions (mpcf_aux.cu).
cudaError_t launch_ic_steady(int is_double, const DomDev* dom, int parity, const SteadyParams& P, cudaStream_t st);
cudaError_t launch_ic_sod(int is_double, const DomDev* dom, int parity, const SodParams& P, cudaStream_t st);
cudaError_t launch_ic_sbi(int is_double, const DomDev* dom, int nx, int ny, int nz, int parity, const SbiParams& P,
                          const double* bubbles, int nbubbles, cudaStream_t st);

// Shock-induced cloud-collapse IC (mpcf_aux.cu); post4 receives the
// post-shock rho1, u1, p1 and the shock Mach number in the state's precision.
cudaError_t launch_sic_cloud(int is_double, const DomDev* dom, int nx, int ny, int nz, int parity,
                             const SicParams& P, const double* shapes, int nshapes, cudaStream_t st);
void sic_post_shock(int is_double, const SicParams& P, double post4[4]);

cudaError_t launch_ic_cloud(int is_double, const DomDev* dom, int parity, const IcParams& P,
                            const double* bubbles, int nbubbles, cudaStream_t st);
cudaError_t launch_fill_ghosts(int is_double, const DomDev* dom, int parity,
                               void* gx, void* gy, void* gz, cudaStream_t st);
cudaError_t launch_zero(void* p, size_t bytes, cudaStream_t st);
// ghost planes of linked slabs: links = nlinks (lower, upper) pairs on the
// device, max_plane = the largest nx*ny among the linked domains
cudaError_t launch_halo(int esz, const DomDev* doms, const int* links, int nlinks, long long max_plane,
                        int parity, cudaStream_t st);
// ghost planes of one slot of a windowed run: from the neighbouring slots'
// planes (lo / hi) or, where they are null, the domain's z boundary condition
cudaError_t launch_window_ghosts(int esz, void* dst, const void* lo, const void* hi, long long fs, long long plane,
                                 int nz, int bc_lo, int bc_hi, cudaStream_t st);
cudaError_t launch_update(int is_double, const DomDev* doms, int ndom, int parity, double b, cudaStream_t st);
cudaError_t launch_fma_probe(int blocks, int iters, float* out, cudaStream_t st);
cudaError_t launch_sum_state(const DomDev* doms, int ndom, int parity, int nchunks, int chunk, int is_double,
                             double* chunk_sums, double* out, cudaStream_t st);

} // namespace mpcf
