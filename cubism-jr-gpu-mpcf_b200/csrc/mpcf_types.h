// mpcf_types.h -- plain structures shared by the host runtime and the
// kernels of libmpcf_b200 (no CUDA types in here beyond what a .cu sees).
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace mpcf {

// Boundary condition codes per face (x-left, x-right, y-left, y-right,
// z-left, z-right).  Absorbing = zeroth-order extrapolation, reflecting =
// mirror with the normal momentum negated (BoundaryConditions.h:60-109).
// Halo (z faces only) = the 3 ghost planes are stored state, filled from a
// neighbouring slab of the same global domain (GridMPI.h:65-106 and the
// halo exchange of GPUlab.cpp:622-644).
enum { BC_ABSORBING = 0, BC_REFLECTING = 1, BC_HALO = 2 };
constexpr int kHaloPlanes = 3;

// Bits of the device error word.
enum {
    ERRBIT_NONPHYSICAL = 1u << 0,   // rho <= 0, E <= 0, G <= 0 or non-finite after an update
    ERRBIT_SOS_NONFINITE = 1u << 1, // max sound speed not finite or not positive
    ERRBIT_TMA_TIMEOUT = 1u << 2,   // a bulk tensor copy did not complete within the wait limit
    ERRBIT_BOUNDS = 1u << 3,        // bounds-checking build: an index left its buffer (clamped)
    ERRBIT_TMA_INFLIGHT = 1u << 4,  // after a give-up, a CTA's bounded wait for its own copies ran out too
};

// One domain as the kernels see it.  All 7 fields of a buffer live in one
// allocation with a field stride `fs` (elements, a multiple of 64), cell
// (ix,iy,iz) at ix + nx*(iy + ny*iz) inside a field (Types.h:31).  With
// halo faces the state buffers hold zlo planes below plane 0 and zhi above
// plane nz-1 (U[b] points at plane 0, iz runs over -zlo .. nz-1+zhi); the
// register has no ghost planes.
struct DomDev
{
    void*  U[2];        // ping-pong state buffers (T*), 7 fields each
    void*  R;           // low-storage RK register (T*), 7 fields
    long long fs;       // field stride in elements
    int    nx, ny, nz;
    int    bc[6];
    int    tiles_x, tiles_y, tiles_z;
    int    tile_begin;  // first global tile id of this domain
    int    sos_chunk_begin;   // first global sound-speed chunk of this domain
    int    sos_chunks;
    int    tma_ok;      // 1: tensor maps of this domain are valid (rows of 16-byte multiples)
    int    zlo, zhi;    // stored ghost planes below z = 0 / above z = nz-1 (0 or 3, halo faces)
    int    org[3];      // cell (0,0,0) is cell org of a global grid of gdim cells (initial conditions)
    int    gdim[3];
    // the extended domain the stage kernel sees: planes -zlo .. nz-1+zhi as
    // 0 .. nzx-1 (Ux/Rx = U/R shifted back by zlo planes; the register is
    // only ever read at the domain's own planes)
    void*  Ux[2];
    void*  Rx;
    int    nzx;
    int    group;       // domains of one group (z-slabs of a global domain) share one dt
    double h;
};

// Arguments of one stage launch (all domains of a solver).
struct StageArgs
{
    const DomDev* doms;
    int    ndom;
    int    ntiles;      // end of the launch's tile range (all tiles: the total over all domains)
    int    tile0;       // first tile of the launch's range (0: from the first tile)
    int    dz;          // z-chunk depth of a tile
    int    parity;      // read U[parity], write U[parity^1]
    double a, b;        // LSRK3 stage coefficients
    const void* dtinvh; // T[ndom], dt/h per domain
    unsigned* counter;  // persistent-launch work counter (zeroed before launch)
    unsigned* err;      // device error word
    double* tile_sums;  // [ntiles][5] FP64 partial conservation sums, or null
    const void* tmaps;  // per domain 4 CUtensorMap (128 B each): [buffer 0, 1] x [halo box, interior box]
    void* sos_bits;     // per domain maximum sound speed of the new state (bits), or null
    unsigned test_flags; // TEST_* below; 0 outside the failure-detection tests
};

// Failure-detection tests: with TEST_DROP_LAST_COPY a non-persistent stage
// kernel arms the mbarrier of the last bulk copy of each chunk but does not
// issue the copy, so the CTA's final bounded wait runs out (ERRBIT_TMA_TIMEOUT)
// with no copy in flight.  TEST_DROP_MID_COPY drops the chunk's first copy
// after the prologue instead: the wait runs out one slab in, the CTA issues
// no further copy and waits for the one still pending before it exits.
// Persistent instances ignore both.  With any flag set, counter[1] counts the
// bulk copies issued.
enum { TEST_DROP_LAST_COPY = 1u, TEST_DROP_MID_COPY = 2u };

struct SosArgs
{
    const DomDev* doms;
    int    ndom;
    int    nchunks;     // chunks of this launch (all domains: the total)
    int    chunk;       // cells per chunk
    int    chunk0;      // first chunk of the launch (block b takes chunk chunk0 + b)
    int    parity;
    void*  sos_bits;    // per domain: unsigned (float bits) or unsigned long long (double bits)
};

struct DtArgs
{
    const DomDev* doms;
    int    ndom;
    double cfl, dt_max;
    void*  sos_bits;
    void*  dtinvh;      // T[ndom]
    double* dt;         // [ndom]
    double* time;       // [ndom], accumulated
    unsigned* err;
    int    grouped;     // some domains share a group (linked slabs): dt from the group's maximum
};

// Bubble-cloud initial condition (liquid with gas bubbles, tanh-smoothed
// indicator).  Material parameters gamma and pc give G = 1/(gamma-1) and
// P = gamma*pc/(gamma-1).
struct IcParams
{
    double rho_l, p_l, gamma_l, pc_l;
    double rho_g, p_g, gamma_g, pc_g;
    double noise;       // velocity noise amplitude (uniform in [-noise, noise])
    double width;       // interface width in cells (tanh smoothing over width*h)
    unsigned long long seed;
};

// Parameters of the reference's shock-induced cloud-collapse case
// (Sim_SICCloudMPI.cpp:52-81), in the order of its command-line options.
struct SicParams
{
    double rho0, u0, p0;        // pre-shock liquid
    double rhoB, uB, pB;        // bubble gas
    double pressure_ratio;      // p1/p0 across the shock
    double shock_n[3];          // shock normal (normalised by the set-up)
    double shock_s[3];          // a point on the shock plane
    double g1, g2, pc1, pc2;    // liquid / gas gamma and pc
    double eps;                 // interface half-width (SimTools::EPSILON; 0: sharp)
};

// Options of the reference's SteadyState, Sod and 2DSBI cases
// (Sim_SteadyStateMPI.cpp:103-109, Sim_SodMPI.cpp:27-57, Sim_2DSBIMPI.cpp:
// 15-58,83-96); axes are 0 = x, 1 = y, 2 = z.
struct SteadyParams { double rho, u, v, w, p, g, pc; };
struct SodParams
{
    double x0, rho1, rho2, u1, u2, p1, p2, g1, g2, pc1, pc2;
    int reverse, axis;
};
struct SbiParams
{
    double x0, mach, rho, rhobubble, u, p, pbubble, g1, g2, pc1, pc2;
    int reverse, mollfactor, axis0, axis1;
};

} // namespace mpcf
