/*
 * ref_devmath.cpp -- runs the reference's own device math on the host.
 * TEST INFRASTRUCTURE ONLY: built by `make -C oracle ref` into oracle/_ref/
 * (git-ignored) from the reference header source/GPU/GPUonly.cuh, included
 * from where it lies; used by tests/ to pin the oracle function by function.
 *
 * GPUonly.cuh holds the reference's WENO5, clipping, stencil reads, Einfeldt,
 * HLLC and extra-term functions as `__device__ inline` code.  They are plain
 * arithmetic, so with `__device__` defined away they compile as host C++.
 * Two CUDA 12 removals are stood in for here, without touching the
 * reference source:
 *   - the legacy texture-reference template `texture<T,3,mode>` and `tex3D`
 *     (GPUonly.cuh:87-93): a host struct bound to a host array, fetched
 *     with the reference's sampler settings (unnormalised coordinates, point
 *     filtering, clamp addressing; GPUkernels.cu:1388-1400);
 *   - the device overloads min(float,float)/max(float,float) used by
 *     _hllc_rho (GPUonly.cuh:881-882), which map to fminf/fmaxf.
 * Compiled with -ffp-contract=off like the oracle, so both evaluate the
 * same expressions with the same rounding.
 */
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>

#define __device__

static inline float min(const float a, const float b) { return fminf(a, b); }
static inline float max(const float a, const float b) { return fmaxf(a, b); }

template <class T, int dim, enum cudaTextureReadMode mode>
struct texture
{
    const T* data;
    int nx, ny, nz;
};

template <class T>
static inline T tex3D(const texture<T, 3, cudaReadModeElementType>& t, const float x, const float y, const float z)
{
    /* point sampling of unnormalised coordinates: texel floor(c), clamped */
    long ix = (long)floorf(x), iy = (long)floorf(y), iz = (long)floorf(z);
    ix = ix < 0 ? 0 : (ix >= t.nx ? t.nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= t.ny ? t.ny - 1 : iy);
    iz = iz < 0 ? 0 : (iz >= t.nz ? t.nz - 1 : iz);
    return t.data[ix + (long)t.nx * (iy + (long)t.ny * iz)];
}

#include "GPU/GPUonly.cuh"

/* globals GPUonly.cuh declares extern (defined in GPUhousehold.cu) */
RealPtrVec_t d_tmp, d_rhs, d_xgl, d_xgr, d_ygl, d_ygr, d_xflux, d_yflux, d_zflux;
std::vector<cudaArray_t> d_GPUin;
Real *d_Gm, *d_Gp, *d_Pm, *d_Pp, *d_hllc_vel, *d_sumG, *d_sumP, *d_divU;
int *d_maxSOS;
cudaStream_t stream1, stream2;
cudaEvent_t h2d_tmp_completed, divergence_completed, update_completed;

extern "C" {

int ref_devmath_dims(int* d) { d[0] = NodeBlock::sizeX; d[1] = NodeBlock::sizeY; d[2] = NodeBlock::sizeZ; return 0; }

float ref_weno_pluss(float b, float c, float d, float e, float f) { return _weno_pluss(b, c, d, e, f); }
float ref_weno_minus(float a, float b, float c, float d, float e) { return _weno_minus(a, b, c, d, e); }
float ref_weno_pluss_clipped(float b, float c, float d, float e, float f) { return _weno_pluss_clipped(b, c, d, e, f); }
float ref_weno_minus_clipped(float a, float b, float c, float d, float e) { return _weno_minus_clipped(a, b, c, d, e); }

void ref_char_vel_einfeldt(float rm, float rp, float vm, float vp, float pm, float pp,
                           float Gm, float Gp, float Pm, float Pp, float* out2)
{
    float a, b;
    _char_vel_einfeldt(rm, rp, vm, vp, pm, pp, Gm, Gp, Pm, Pp, a, b);
    out2[0] = a; out2[1] = b;
}
float ref_char_vel_star(float rm, float rp, float vm, float vp, float pm, float pp, float sm, float sp)
{ return _char_vel_star(rm, rp, vm, vp, pm, pp, sm, sp); }
float ref_hllc_rho(float rm, float rp, float vm, float vp, float sm, float sp, float ss)
{ return _hllc_rho(rm, rp, vm, vp, sm, sp, ss); }
float ref_hllc_vel(float rm, float rp, float vm, float vp, float vdm, float vdp, float sm, float sp, float ss)
{ return _hllc_vel(rm, rp, vm, vp, vdm, vdp, sm, sp, ss); }
float ref_hllc_pvel(float rm, float rp, float vm, float vp, float pm, float pp, float sm, float sp, float ss)
{ return _hllc_pvel(rm, rp, vm, vp, pm, pp, sm, sp, ss); }
float ref_hllc_e(float rm, float rp, float vdm, float vdp, float v1m, float v1p, float v2m, float v2p,
                 float pm, float pp, float Gm, float Gp, float Pm, float Pp, float sm, float sp, float ss)
{ return _hllc_e(rm, rp, vdm, vdp, v1m, v1p, v2m, v2p, pm, pp, Gm, Gp, Pm, Pp, sm, sp, ss); }
float ref_extraterm_hllc_vel(float um, float up, float Gm, float Gp, float Pm, float Pp, float sm, float sp, float ss)
{ return _extraterm_hllc_vel(um, up, Gm, Gp, Pm, Pp, sm, sp, ss); }

/* The stencil of face (ix,iy) in slice iz of a single chunk: `in` is the
 * chunk input (NX x NY x (nslices+6), z-ghost slices included, as uploaded
 * by GPUlab::process_all, GPUlab.cpp:742-761), gl/gr the compact x or y
 * ghost buffers (GHOSTMAPX / GHOSTMAPY).  dir 0/1/2 -> _read_stencil_X/Y/Z
 * (GPUonly.cuh:305-593), global_iz = 0 (GPUlab.cpp:244). */
void ref_read_stencil(int dir, const float* in, int nslices, const float* gl, const float* gr,
                      unsigned ix, unsigned iy, unsigned iz, float* out6)
{
    texture<float, 3, cudaReadModeElementType> t;
    t.data = in; t.nx = NodeBlock::sizeX; t.ny = NodeBlock::sizeY; t.nz = nslices + 6;
    Stencil s;
    if (dir == 0) _read_stencil_X(s, t, gl, gr, ix, iy, iz, 0);
    else if (dir == 1) _read_stencil_Y(s, t, gl, gr, ix, iy, iz, 0);
    else _read_stencil_Z(s, t, ix, iy, iz);
    out6[0] = s.im3; out6[1] = s.im2; out6[2] = s.im1; out6[3] = s.i; out6[4] = s.ip1; out6[5] = s.ip2;
}

} /* extern "C" */
