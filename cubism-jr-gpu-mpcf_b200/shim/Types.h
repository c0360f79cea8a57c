// Types.h -- the type and index-map vocabulary of the reference's host code
// (source/Types.h:17-69), so code written against it compiles unchanged.
// The index maps are the data-layout contract of the reference's halo
// buffers: ID3 (x fastest), GHOSTMAPX [z][y][3], GHOSTMAPY [z][3][x].
#pragma once

#include <cstdio>
#include <cassert>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <cmath>

#include "NodeBlock.h"

typedef std::vector<Real*> RealPtrVec_t;
typedef unsigned int uint_t;

enum Coord { X = 0, Y, Z };

#define ID3(ix,iy,iz,NX,NY) ((ix) + (NX) * ((iy) + (NY) * (iz)))
#define GHOSTMAPX(ix,iy,iz) ((ix) + 3 * ((iy) + NodeBlock::sizeY * (iz)))
#define GHOSTMAPY(ix,iy,iz) ((ix) + NodeBlock::sizeX * ((iy) + 3 * (iz)))

typedef uint_t (*index_map)(const int, const int, const int);

struct ghostmap
{
    static inline uint_t X(const int ix, const int iy, const int iz) { return GHOSTMAPX(ix, iy, iz); }
    static inline uint_t Y(const int ix, const int iy, const int iz) { return GHOSTMAPY(ix, iy, iz); }
    static inline uint_t Z(const int ix, const int iy, const int iz) { return ID3(ix, iy, iz, NodeBlock::sizeX, NodeBlock::sizeY); }
};

struct flesh2ghost
{
    static inline uint_t X_L(const int ix, const int iy, const int iz) { return ghostmap::X(ix, iy, iz); }
    static inline uint_t X_R(const int ix, const int iy, const int iz) { return ghostmap::X(ix - NodeBlock::sizeX + 3, iy, iz); }
    static inline uint_t Y_L(const int ix, const int iy, const int iz) { return ghostmap::Y(ix, iy, iz); }
    static inline uint_t Y_R(const int ix, const int iy, const int iz) { return ghostmap::Y(ix, iy - NodeBlock::sizeY + 3, iz); }
};

// Interface-smoothing helpers of the case set-ups (source/Types.h:84-100):
// a sharp step (1 where phi <= 0) and a cosine ramp of half-width EPSILON.
class SimTools
{
public:
    static double EPSILON;

    static Real heaviside(const Real phi) { return phi > 0 ? 0 : 1; }

    static Real heaviside_smooth(const Real phi)
    {
        const Real alpha = M_PI * std::min(1., std::max(0., 0.5 * (phi + EPSILON) / EPSILON));
        return 0.5 + 0.5 * std::cos(alpha);
    }

    // State {rho, u, p} behind a normal shock of Mach number `mach` running
    // into the stiffened-gas state pre_shock (Rankine-Hugoniot relations, in
    // the mixed Real/double arithmetic of source/Types.h:100-109, which the
    // cases' results depend on).
    static void getPostShockRatio(const Real pre_shock[3], const Real mach, const Real gamma, const Real pc, Real postShock[3])
    {
        const Real m2 = std::pow(mach, (Real)2.);
        const double mpost = std::sqrt((m2 * (gamma - 1.) + 2.) / (2. * gamma * m2 - (gamma - 1.)));
        postShock[0] = (gamma + 1.) * m2 / ((gamma - 1.) * m2 + 2.) * pre_shock[0];
        postShock[2] = 1. / (gamma + 1.) * (2. * gamma * m2 - (gamma - 1.)) * pre_shock[2];
        const double u_pre  = mach * std::sqrt(gamma * (pc + pre_shock[2]) / pre_shock[0]);
        const double u_post = mpost * std::sqrt(gamma * (pc + postShock[2]) / postShock[0]);
        postShock[1] = u_pre - u_post;
    }

    // Mirror check of a grid in its "minor" direction dims[1]: every field of
    // a cell equals that of the cell mirrored across the grid's mid-plane in
    // dims[1] (asserted to tol); prints the largest difference.  dims =
    // {principal, minor, third}; NULL means {x, y, z}.
    template <typename TGrid>
    static void symmetry_check(TGrid& grid, const int verbosity, const Real tol = 1.0e-6, uint_t dims[3] = NULL)
    {
        uint_t d[3] = {0, 1, 2};
        if (dims) { d[0] = dims[0]; d[1] = dims[1]; d[2] = dims[2]; }
        const int n[3] = {TGrid::sizeX, TGrid::sizeY, TGrid::sizeZ};
        Real linf = 0;
        int a[3], b[3];
        for (a[d[2]] = 0; a[d[2]] < n[d[2]]; ++a[d[2]])
            for (a[d[1]] = 0; a[d[1]] < n[d[1]] / 2; ++a[d[1]])
                for (a[d[0]] = 0; a[d[0]] < n[d[0]]; ++a[d[0]])
                {
                    b[d[0]] = a[d[0]];
                    b[d[1]] = n[d[1]] - 1 - a[d[1]];
                    b[d[2]] = a[d[2]];
                    Real m = 0;
                    for (int q = 0; q < 7; ++q)
                    {
                        const typename TGrid::PRIM f = (typename TGrid::PRIM)q;
                        const Real diff = std::abs(grid(a[0], a[1], a[2], f) - grid(b[0], b[1], b[2], f));
                        assert(diff < tol);
                        m = std::max(m, diff);
                    }
                    if (verbosity == 3) printf("Symmetry Check: (%d,%d,%d)<->(%d,%d,%d) => Linf = %f\n", a[0], a[1], a[2], b[0], b[1], b[2], m);
                    linf = std::max(linf, m);
                }
        printf("Global Linf = %f\n", linf);
    }
};

// ---------------------------------------------------------------------------
// Output streamers of the dump and the save (source/Types.h:157-277): the
// channels one cell contributes to the interleaved output array.  The
// library's mpcf_pack fills the same arrays on the GPU.
// ---------------------------------------------------------------------------
struct myTensorialStreamer
{
    static const int NCHANNELS = 9;
    const Real *r, *u, *v, *w, *e, *G, *P;
    myTensorialStreamer(const std::vector<Real*>& p) : r(p[0]), u(p[1]), v(p[2]), w(p[3]), e(p[4]), G(p[5]), P(p[6]) {}
    // rho, velocity, pressure, G, P and two zero channels
    void operate(const int ix, const int iy, const int iz, Real out[NCHANNELS]) const
    {
        const int c = ID3(ix, iy, iz, NodeBlock::sizeX, NodeBlock::sizeY);
        out[0] = r[c];
        out[1] = u[c] / r[c];
        out[2] = v[c] / r[c];
        out[3] = w[c] / r[c];
        out[4] = (e[c] - 0.5 * (u[c] * u[c] + v[c] * v[c] + w[c] * w[c]) / r[c] - P[c]) / G[c];
        out[5] = G[c];
        out[6] = P[c];
        out[7] = 0.;
        out[8] = 0.;
    }
    static const char* getAttributeName() { return "Tensor"; }
};

struct myScalarStreamer
{
    static const int NCHANNELS = 1;
    const Real* r;
    myScalarStreamer(const std::vector<Real*>& p) : r(p[0]) {}
    void operate(const int ix, const int iy, const int iz, Real out[NCHANNELS]) const
    {
        out[0] = r[ID3(ix, iy, iz, NodeBlock::sizeX, NodeBlock::sizeY)];
    }
    static const char* getAttributeName() { return "Scalar"; }
};

struct mySaveStreamer
{
    static const int NCHANNELS = NodeBlock::NVAR;
    Real* f[7];
    mySaveStreamer(const std::vector<Real*>& p) { for (int q = 0; q < 7; ++q) f[q] = p[q]; }
    // the conserved fields of one cell, out and back in (restart)
    void operate(const int ix, const int iy, const int iz, Real out[NCHANNELS]) const
    {
        const int c = ID3(ix, iy, iz, NodeBlock::sizeX, NodeBlock::sizeY);
        for (int q = 0; q < 7; ++q) out[q] = f[q][c];
    }
    void operate(const Real in[NCHANNELS], const int ix, const int iy, const int iz) const
    {
        const int c = ID3(ix, iy, iz, NodeBlock::sizeX, NodeBlock::sizeY);
        for (int q = 0; q < 7; ++q) f[q][c] = in[q];
    }
    static const char* getAttributeName() { return "Save Data"; }
};

class Simulation
{
protected:
    virtual void _setup() {}
public:
    virtual void run() = 0;
    virtual ~Simulation() {}
};
