// NodeBlock.h -- host block storage with the reference's interface
// (source/NodeBlock.h:22-119): compile-time block size _BLOCKSIZEX/Y/Z_,
// 7 SoA fields `data` (rho, rho u, rho v, rho w, E, G, P) plus the LSRK3
// register `tmp`, cell (ix,iy,iz) at ix + sizeX*(iy + sizeY*iz), spacing
// h = maxextent / max(sizeX, sizeY, sizeZ).  Code written against the
// reference block compiles against this one unchanged.
#pragma once

#include <cstdlib>
#include <cassert>
#include <cmath>
#include <vector>
#include <algorithm>

#ifdef _FLOAT_PRECISION_
typedef float Real;
#else
typedef double Real;
#endif

class NodeBlock
{
public:
    enum PRIM { R = 0, U, V, W, E, G, P, NPRIMITIVES = 7 };

    static const int NVAR = NPRIMITIVES;
    static const int sizeX = _BLOCKSIZEX_;
    static const int sizeY = _BLOCKSIZEY_;
    static const int sizeZ = _BLOCKSIZEZ_;

protected:
    double origin[3];
    double extent[3];
    double h;
    std::vector<Real*> data;
    std::vector<Real*> tmp;

private:
    void _alloc()
    {
        const size_t n = (size_t)sizeX * sizeY * sizeZ;
        for (int v = 0; v < NVAR; ++v)
        {
            // 64-byte alignment: pinned-copy friendly and vector friendly
            void* p = nullptr;
            void* q = nullptr;
            if (posix_memalign(&p, 64, sizeof(Real) * n) || posix_memalign(&q, 64, sizeof(Real) * n)) std::abort();
            data[v] = (Real*)p;
            tmp[v] = (Real*)q;
        }
    }

public:
    NodeBlock(const double maxextent = 1.0) : data(NVAR, nullptr), tmp(NVAR, nullptr)
    {
        h = maxextent / std::max(sizeX, std::max(sizeY, sizeZ));
        origin[0] = origin[1] = origin[2] = 0.0;
        extent[0] = h * sizeX;
        extent[1] = h * sizeY;
        extent[2] = h * sizeZ;
        _alloc();
    }

    virtual ~NodeBlock()
    {
        for (int v = 0; v < NVAR; ++v) { free(data[v]); free(tmp[v]); }
    }

    void clear_data() { for (int v = 0; v < NVAR; ++v) std::fill(data[v], data[v] + (size_t)sizeX * sizeY * sizeZ, (Real)0); }
    void clear_tmp()  { for (int v = 0; v < NVAR; ++v) std::fill(tmp[v], tmp[v] + (size_t)sizeX * sizeY * sizeZ, (Real)0); }
    void clear() { clear_data(); clear_tmp(); }

    double h_gridpoint() const { return h; }
    void get_pos(const unsigned ix, const unsigned iy, const unsigned iz, double pos[3]) const
    {
        pos[0] = origin[0] + h * (ix + 0.5);
        pos[1] = origin[1] + h * (iy + 0.5);
        pos[2] = origin[2] + h * (iz + 0.5);
    }
    void get_origin(double O[3]) const { O[0] = origin[0]; O[1] = origin[1]; O[2] = origin[2]; }
    void get_extent(double Ex[3]) const { Ex[0] = extent[0]; Ex[1] = extent[1]; Ex[2] = extent[2]; }

    const std::vector<Real*>& pdata() const { return data; }
    const std::vector<Real*>& ptmp() const { return tmp; }
    std::vector<Real*>& pdata() { return data; }
    std::vector<Real*>& ptmp() { return tmp; }

    Real& operator()(const unsigned ix, const unsigned iy, const unsigned iz, const PRIM p)
    {
        assert(ix < (unsigned)sizeX && iy < (unsigned)sizeY && iz < (unsigned)sizeZ);
        return data[p][ix + (size_t)sizeX * (iy + (size_t)sizeY * iz)];
    }
};
