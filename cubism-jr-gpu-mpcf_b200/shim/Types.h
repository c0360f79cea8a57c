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
};

class Simulation
{
protected:
    virtual void _setup() {}
public:
    virtual void run() = 0;
    virtual ~Simulation() {}
};
