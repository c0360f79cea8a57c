/*
 * ref_harness.cpp -- C entry points around pieces of the reference that
 * compile from their own sources.  TEST INFRASTRUCTURE ONLY: built by
 * `make -C oracle ref` into oracle/_ref/ (git-ignored) with the reference
 * tree on the include path; used by tests/ to pin the oracle, and by
 * bench.py's CPU-baseline leg.  Nothing from the reference is copied here;
 * the reference headers are included from where they lie.
 *
 *   REF_HARNESS_SOS: MaxSpeedOfSound_CPP::compute (source/MaxSpeedOfSound.cpp:18-55),
 *                    compiled for a 65536-cell block and applied chunk by chunk.
 *   REF_HARNESS_BC:  BoundaryConditions<NodeBlock>::applyBC_absorbing /
 *                    applyBC_reflecting (source/BoundaryConditions.h:60-109)
 *                    for the compile-time block size.
 *   REF_HARNESS_DUMP: the output streamers myTensorialStreamer and
 *                    mySaveStreamer (source/Types.h:192-277) filling the
 *                    interleaved array DumpHDF5_MPI / ReadHDF5_MPI move
 *                    (source/IO/HDF5Dumper_MPI.h:104-121, 243-253).
 */
#include <vector>
#include <cstring>
#include <algorithm>

#ifdef REF_HARNESS_SOS
#include "MaxSpeedOfSound.h"

extern "C" float ref_max_sos_cpp(long long n, float** U)
{
    const long long CH = (long long)_BLOCKSIZEX_ * _BLOCKSIZEY_ * _BLOCKSIZEZ_;
    MaxSpeedOfSound_CPP k;
    float sos = 0;
    std::vector<float> pad[7];
    for (long long off = 0; off < n; off += CH)
    {
        RealPtrVec_t src(7);
        const long long len = std::min(CH, n - off);
        for (int q = 0; q < 7; ++q)
        {
            if (len == CH) src[q] = U[q] + off;
            else
            {
                /* pad a short last chunk with copies of its first cell: the
                 * maximum is unchanged */
                pad[q].assign(CH, U[q][off]);
                std::memcpy(pad[q].data(), U[q] + off, sizeof(float) * len);
                src[q] = pad[q].data();
            }
        }
        const float s = k.compute(src);
        sos = std::max(sos, s);
    }
    return sos;
}
#endif

#ifdef REF_HARNESS_BC
#include "BoundaryConditions.h"

extern "C" int ref_bc_dims(int* d) { d[0] = _BLOCKSIZEX_; d[1] = _BLOCKSIZEY_; d[2] = _BLOCKSIZEZ_; return 0; }

/* Fills the six halos like GPUlab*::_apply_bc does on one rank (all faces
 * SKIN).  Output layout matches oracle_fill_ghosts_f32: [side][q][...]. */
extern "C" int ref_fill_ghosts(const int* bc, float** U, float* gx_all, float* gy_all, float* gz_all)
{
    const int NX = _BLOCKSIZEX_, NY = _BLOCKSIZEY_, NZ = _BLOCKSIZEZ_;
    const size_t sx = (size_t)3 * NY * NZ, sy = (size_t)NX * 3 * NZ, sz = (size_t)NX * NY * 3;
    RealPtrVec_t data(7);
    for (int q = 0; q < 7; ++q) data[q] = U[q];
    RealPtrVec_t hx[2], hy[2], hz[2];
    for (int s = 0; s < 2; ++s)
    {
        hx[s].resize(7); hy[s].resize(7); hz[s].resize(7);
        for (int q = 0; q < 7; ++q)
        {
            hx[s][q] = gx_all + (s * 7 + q) * sx;
            hy[s][q] = gy_all + (s * 7 + q) * sy;
            hz[s][q] = gz_all + (s * 7 + q) * sz;
        }
    }
    BoundaryConditions<NodeBlock> b(data);
    if (bc[0]) b.applyBC_reflecting<0,0,ghostmap::X>(hx[0]); else b.applyBC_absorbing<0,0,ghostmap::X>(hx[0]);
    if (bc[1]) b.applyBC_reflecting<0,1,ghostmap::X>(hx[1]); else b.applyBC_absorbing<0,1,ghostmap::X>(hx[1]);
    if (bc[2]) b.applyBC_reflecting<1,0,ghostmap::Y>(hy[0]); else b.applyBC_absorbing<1,0,ghostmap::Y>(hy[0]);
    if (bc[3]) b.applyBC_reflecting<1,1,ghostmap::Y>(hy[1]); else b.applyBC_absorbing<1,1,ghostmap::Y>(hy[1]);
    if (bc[4]) b.applyBC_reflecting<2,0,ghostmap::Z>(hz[0]); else b.applyBC_absorbing<2,0,ghostmap::Z>(hz[0]);
    if (bc[5]) b.applyBC_reflecting<2,1,ghostmap::Z>(hz[1]); else b.applyBC_absorbing<2,1,ghostmap::Z>(hz[1]);
    return 0;
}
#endif

#ifdef REF_HARNESS_DUMP
#include "Types.h"

extern "C" int ref_dump_dims(int* d) { d[0] = _BLOCKSIZEX_; d[1] = _BLOCKSIZEY_; d[2] = _BLOCKSIZEZ_; return 0; }

/* out[NCH*(ix + NX*(iy + NY*iz)) + c] = channel c of the streamer at (ix,iy,iz):
 * kind 0 = myTensorialStreamer (9 channels), 1 = mySaveStreamer (7) */
extern "C" int ref_pack(int kind, float** U, float* out)
{
    std::vector<Real*> ptr(U, U + 7);
    const int NX = _BLOCKSIZEX_, NY = _BLOCKSIZEY_, NZ = _BLOCKSIZEZ_;
    for (int iz = 0; iz < NZ; ++iz)
        for (int iy = 0; iy < NY; ++iy)
            for (int ix = 0; ix < NX; ++ix)
            {
                if (kind == 0)
                {
                    myTensorialStreamer st(ptr);
                    Real o[myTensorialStreamer::NCHANNELS];
                    st.operate(ix, iy, iz, o);
                    std::memcpy(out + myTensorialStreamer::NCHANNELS * (ix + NX * (iy + NY * iz)), o, sizeof(o));
                }
                else
                {
                    mySaveStreamer st(ptr);
                    Real o[mySaveStreamer::NCHANNELS];
                    st.operate(ix, iy, iz, o);
                    std::memcpy(out + mySaveStreamer::NCHANNELS * (ix + NX * (iy + NY * iz)), o, sizeof(o));
                }
            }
    return 0;
}

/* the restart direction: mySaveStreamer::operate(input, ix, iy, iz) */
extern "C" int ref_unpack_save(const float* in, float** U)
{
    std::vector<Real*> ptr(U, U + 7);
    mySaveStreamer st(ptr);
    const int NX = _BLOCKSIZEX_, NY = _BLOCKSIZEY_, NZ = _BLOCKSIZEZ_;
    for (int iz = 0; iz < NZ; ++iz)
        for (int iy = 0; iy < NY; ++iy)
            for (int ix = 0; ix < NX; ++ix)
            {
                Real v[mySaveStreamer::NCHANNELS];
                std::memcpy(v, in + mySaveStreamer::NCHANNELS * (ix + NX * (iy + NY * iz)), sizeof(v));
                st.operate(v, ix, iy, iz);
            }
    return 0;
}
#endif
