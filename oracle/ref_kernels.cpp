/*
 * ref_kernels.cpp -- runs the reference's own stage kernels on the host.
 * TEST INFRASTRUCTURE ONLY: built by `make -C oracle ref` into oracle/_ref/
 * (git-ignored).  The build takes source/GPU/GPUkernels.cu from where it
 * lies, up to the _maxSOS kernel (which reduces through shared memory and
 * is pinned separately), into oracle/_ref/gpukernels_body.inc and includes
 * it here; nothing of it is kept in the repository.
 *
 * The kernels _xflux, _xextraterm_hllc, _yflux, _yextraterm_hllc, _zflux,
 * _zextraterm_hllc, _divergence and _update (GPUkernels.cu:35-1179) use no
 * shared memory and no barriers: every thread computes its (ix, iy) column
 * of faces or cells on its own.  So they run here as host functions, one
 * call per thread of the reference's launch grid (`launch` below), with
 * the CUDA index built-ins as thread-local host variables and the texture
 * stand-in of ref_devmath.cpp.  A stage is the single-chunk
 * GPUlab::process_all (GPUlab.cpp:703-793, nslices = NZ, global_iz = 0):
 * the seven kernels in the order of GPU::xflux/yflux/zflux/divergence/update
 * with their grids (GPUkernels.cu:1227-1334), then the register is the rhs
 * and the state is the updated tmp.  Built with -ffp-contract=off like the
 * oracle, so the tests compare the oracle's restated flux assembly, extra
 * terms, divergence and update with the reference's own code bit for bit.
 */
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#define __device__
#define __global__

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

/* the CUDA index built-ins of the thread being run */
static thread_local dim3 blockIdx, threadIdx;
static thread_local dim3 blockDim, gridDim;

#include "gpukernels_body.inc"

/* globals GPUonly.cuh declares extern (defined in GPUhousehold.cu) */
RealPtrVec_t d_tmp, d_rhs, d_xgl, d_xgr, d_ygl, d_ygr, d_xflux, d_yflux, d_zflux;
std::vector<cudaArray_t> d_GPUin;
Real *d_Gm, *d_Gp, *d_Pm, *d_Pp, *d_hllc_vel, *d_sumG, *d_sumP, *d_divU;
int *d_maxSOS;
cudaStream_t stream1, stream2;
cudaEvent_t h2d_tmp_completed, divergence_completed, update_completed;

/* Every thread of a (grid.x, grid.y) x (block.x) launch, rows of blocks in
 * parallel (the kernels' threads are independent). */
template <class F>
static void launch(const dim3 grid, const dim3 block, F f)
{
    #pragma omp parallel for schedule(static)
    for (int by = 0; by < (int)grid.y; ++by)
    {
        gridDim = grid;
        blockDim = block;
        for (unsigned bx = 0; bx < grid.x; ++bx)
            for (unsigned tx = 0; tx < block.x; ++tx)
            {
                blockIdx = dim3(bx, (unsigned)by, 0);
                threadIdx = dim3(tx, 0, 0);
                f();
            }
    }
}

static RealPtrVec_t fields(std::vector<Real>& store, const size_t n)
{
    store.assign(7 * n, 0);
    RealPtrVec_t v(7);
    for (int q = 0; q < 7; ++q) v[q] = store.data() + q * n;
    return v;
}

extern "C" {

int ref_kernels_dims(int* d) { d[0] = NodeBlock::sizeX; d[1] = NodeBlock::sizeY; d[2] = NodeBlock::sizeZ; return _NTHREADS_; }

/* One stage of the block.  U (in/out): the 7 fields; R (in/out): the
 * register; gx, gy, gz: the ghost layers in the layout of the oracle's
 * oracle_fill_ghosts_f32 ([side][field][...], the reference's halo layouts,
 * z ghosts as 3 planes per side).  On return U holds b*rhs + U and R the rhs
 * = a*R - dtinvh*L(U), as GPUlab::process_all leaves pdata and ptmp. */
void ref_kernels_stage(float* const* U, float* const* R, const float* gx, const float* gy, const float* gz,
                       float a, float b, float dtinvh)
{
    const uint_t nx = NodeBlock::sizeX, ny = NodeBlock::sizeY, nz = NodeBlock::sizeZ;
    const size_t N = (size_t)nx * ny * nz, plane = (size_t)nx * ny;
    const size_t sx = (size_t)3 * ny * nz, sy = (size_t)nx * 3 * nz, sz = plane * 3;

    /* chunk input of each field: z-left ghosts, the block, z-right ghosts
     * (GPUlab.cpp:742-761), read through the textures */
    std::vector<Real> in(7 * (N + 2 * sz));
    texture<float, 3, cudaReadModeElementType>* tex[7] = {&texR, &texU, &texV, &texW, &texE, &texG, &texP};
    for (int q = 0; q < 7; ++q)
    {
        Real* c = in.data() + q * (N + 2 * sz);
        memcpy(c, gz + (0 * 7 + q) * sz, sizeof(Real) * sz);
        memcpy(c + sz, U[q], sizeof(Real) * N);
        memcpy(c + sz + N, gz + (1 * 7 + q) * sz, sizeof(Real) * sz);
        tex[q]->data = c; tex[q]->nx = (int)nx; tex[q]->ny = (int)ny; tex[q]->nz = (int)nz + 6;
    }
    std::vector<Real> s_xgl, s_xgr, s_ygl, s_ygr, s_xf, s_yf, s_zf, s_rhs, s_tmp;
    RealPtrVec_t xgl = fields(s_xgl, sx), xgr = fields(s_xgr, sx), ygl = fields(s_ygl, sy), ygr = fields(s_ygr, sy);
    for (int q = 0; q < 7; ++q)
    {
        memcpy(xgl[q], gx + (0 * 7 + q) * sx, sizeof(Real) * sx);
        memcpy(xgr[q], gx + (1 * 7 + q) * sx, sizeof(Real) * sx);
        memcpy(ygl[q], gy + (0 * 7 + q) * sy, sizeof(Real) * sy);
        memcpy(ygr[q], gy + (1 * 7 + q) * sy, sizeof(Real) * sy);
    }
    RealPtrVec_t xf = fields(s_xf, (size_t)(nx + 1) * ny * nz);
    RealPtrVec_t yf = fields(s_yf, (size_t)nx * (ny + 1) * nz);
    RealPtrVec_t zf = fields(s_zf, plane * (nz + 1));
    RealPtrVec_t rhs = fields(s_rhs, N);
    RealPtrVec_t tmp = fields(s_tmp, N);
    for (int q = 0; q < 7; ++q) memcpy(tmp[q], R[q], sizeof(Real) * N);
    /* face and cell scratch, sized for the largest face count */
    const size_t nf = std::max((size_t)(nx + 1) * ny * nz, std::max((size_t)nx * (ny + 1) * nz, plane * (nz + 1)));
    std::vector<Real> Gm(nf), Gp(nf), Pm(nf), Pp(nf), vel(nf), sumG(N), sumP(N), divU(N);

    devPtrSet XGL(xgl), XGR(xgr), YGL(ygl), YGR(ygr), XF(xf), YF(yf), ZF(zf), RHS(rhs), TMP(tmp);
    const uint_t ns = nz;
    const dim3 blocks(_NTHREADS_, 1, 1);
    const dim3 gx_faces((nx + 1 + _NTHREADS_ - 1) / _NTHREADS_, ny, 1);
    const dim3 g_cells((nx + _NTHREADS_ - 1) / _NTHREADS_, ny, 1);
    const dim3 gy_faces((nx + _NTHREADS_ - 1) / _NTHREADS_, ny + 1, 1);

    launch(gx_faces, blocks, [&] { _xflux(ns, 0, XGL, XGR, XF, vel.data(), Gm.data(), Gp.data(), Pm.data(), Pp.data()); });
    launch(g_cells, blocks, [&] { _xextraterm_hllc(ns, Gm.data(), Gp.data(), Pm.data(), Pp.data(), vel.data(), sumG.data(), sumP.data(), divU.data()); });
    launch(gy_faces, blocks, [&] { _yflux(ns, 0, YGL, YGR, YF, vel.data(), Gm.data(), Gp.data(), Pm.data(), Pp.data()); });
    launch(g_cells, blocks, [&] { _yextraterm_hllc(ns, Gm.data(), Gp.data(), Pm.data(), Pp.data(), vel.data(), sumG.data(), sumP.data(), divU.data()); });
    launch(g_cells, blocks, [&] { _zflux(ns, ZF, vel.data(), Gm.data(), Gp.data(), Pm.data(), Pp.data()); });
    launch(g_cells, blocks, [&] { _zextraterm_hllc(ns, Gm.data(), Gp.data(), Pm.data(), Pp.data(), vel.data(), sumG.data(), sumP.data(), divU.data()); });
    launch(g_cells, blocks, [&] { _divergence(ns, XF, YF, ZF, RHS, a, dtinvh, TMP, sumG.data(), sumP.data(), divU.data()); });
    launch(g_cells, blocks, [&] { _update(ns, b, TMP, RHS); });

    for (int q = 0; q < 7; ++q)
    {
        memcpy(U[q], tmp[q], sizeof(Real) * N);
        memcpy(R[q], rhs[q], sizeof(Real) * N);
    }
}

} /* extern "C" */
