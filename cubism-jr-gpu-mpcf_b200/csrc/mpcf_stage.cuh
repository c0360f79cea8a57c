// mpcf_stage.cuh -- the fused LSRK3 stage kernel.
//
// One launch advances every cell of every domain through one low-storage
// RK stage: ghost synthesis from the boundary conditions, WENO5/HLLC face
// fluxes in x, y and z, the non-conservative G/P extra terms, the flux
// divergence with the register update, and the state update.  It replaces
// the reference chain
//   _apply_bc (host) -> _xflux/_xextraterm_hllc -> _yflux/_yextraterm_hllc
//   -> _zflux/_zextraterm_hllc -> _divergence -> _update
// (BoundaryConditions.h:60-109, GPUkernels.cu:35-1179) and its per-stage
// PCIe streaming (GPUlab.cpp:202-372,703-793); all state stays in HBM.
//
// Work decomposition.  A tile is 32 x TY columns in x-y and a z-chunk of
// depth dz.  Warp w < TY owns row w, one thread per column; for TY = 2^n - 1
// a further warp (the helper) owns no column.  The CTA marches up the chunk
// one slab at a time:
//   * a 6-slab ring of primitives (rho,u,v,w,p,G,P) of the tile's own
//     columns lives in shared memory (z-stencil of the z faces);
//   * slab k with its 3-cell x/y halo is staged in `cur` (x/y stencils);
//   * reconstruction is per cell: the three WENO5 smoothness indicators of
//     a cell serve both its edge values (the minus side of the face right
//     of it and the plus side of the face left of it), in every direction;
//   * z: every column thread reconstructs its cell k, evaluates the z face
//     k-1/2 from the carried upper edge of cell k-1, and finalises cell
//     k-1: rhs = a*R - dtinvh*div(F) (with the G/P extra terms),
//     R <- rhs, U_next <- b*rhs + U;
//   * x, y: every column thread writes its cell's edge values into the face
//     slots in shared memory; the helper warp reconstructs the ghost cells
//     around the tile (rows -1 and TY, columns -1 and 32; without a helper
//     warps 0..2 take one job each, or every warp a share of their planes
//     in the reference-rounding forms); after a barrier each face is
//     evaluated in place in its slot, the x face left of every cell and the
//     y face below it by the cell's thread, the faces above and right of
//     the tile by the helper (warps 3 and 4 without one);
//   * after a second barrier every cell gathers its x/y flux differences,
//     carried to its finalisation in the next slab.
// Each cell is converted to primitives once per stage (the reference
// converts the six stencil cells again at every face).  The state is
// ping-ponged (read U[parity], write U[parity^1]) so neighbouring tiles
// always see the old state.
//
// Loads.  Without TMA every thread loads its cells with ordinary global
// loads (the generic path, any domain shape).  With TMA (domains whose rows
// are multiples of 16 bytes), one elected thread issues two bulk tensor
// copies per slab into shared memory -- the 40 x (TY+6) halo box of the next
// slab and the 32 x TY interior of the slab three ahead -- which land while
// the current slab's faces are evaluated; out-of-domain cells of the staged
// box are mapped to their mirror / clamp source inside the box.  Waits on
// the copies are bounded: a copy that does not complete sets an error bit,
// the CTA stops waiting for copies and carries on (its data are then stale,
// never out of bounds), so a failed copy cannot stall the launch.
//
// DRAM traffic per cell-stage: read U (7 T) + read R (7 T) + write R and
// U_next (14 T) = 112 B in FP32.  Halo and ring re-reads hit L2.
#pragma once

#include "mpcf_math.cuh"
#include "mpcf_types.h"

namespace mpcf {

constexpr int kTX = 32;

__host__ __device__ constexpr size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Shared-memory layout of one CTA.  The T region is addressed in elements.
// Every primitive plane q (rho, u, v, w, p, G, P) has the same pitch kPP and
// holds both stencil sources, so a stencil of any direction is
// addr[j] + q*kPP with kPP a compile-time constant:
//   plane q:  ring [6 slots][TY][32]      z-ring of the tile's own columns
//             cur  [TY+6][38]             slab k with 3-cell x/y halos
// Face slots, pitch kFP = (TY+1)*32, 14 planes each:
//   fx   [14][TY][33]                     x faces of slab k
//   fy   [14][TY+1][32]                   y faces of slab k
// Before a face is evaluated, planes 0..6 of its slot hold its minus side
// and planes 7..13 its plus side (the reconstructed edge values of the two
// cells it separates); the evaluation overwrites planes 0..11 in place with
// its results (7 fluxes, G-, G+, P-, P+, the extra-term velocity).
// then, in bytes: the FP64 reduction scratch [TY][5], the tile broadcast,
// two mbarriers and, with TMA, the two staging buffers (128-byte aligned):
//   A     [7][TY+6][40]                   halo box, x from x0-4, y from y0-3
//   B     [7][TY][32]                     interior of a slab
template <class T, int TY, bool TMA>
struct StageLayout
{
    static constexpr int kNF     = 14;                     // planes of a face slot
    static constexpr int kCurW   = kTX + 6;                // cur row width
    static constexpr int kRing   = TY * kTX;               // one ring slot of a plane
    static constexpr int kCurOff = 6 * kRing;              // cur inside a plane
    static constexpr int kPP     = kCurOff + (TY + 6) * kCurW;
    static constexpr int kFP     = (TY + 1) * kTX;         // >= TY * 33 for TY <= 32
    static constexpr int kFx     = 7 * kPP;
    static constexpr int kFy     = kFx + kNF * kFP;
    static constexpr int kEnd    = kFy + kNF * kFP;
    static constexpr int kAW     = kTX + 8;                // staged halo box width
    static constexpr int kAH     = TY + 6;                 // staged halo box height
    static constexpr size_t kRedBytes  = align_up(kEnd * sizeof(T), 16);
    static constexpr size_t kTileBytes = kRedBytes + sizeof(double) * TY * 5;
    static constexpr size_t kMbarBytes = align_up(kTileBytes + 16, 16);
    static constexpr size_t kABytes    = sizeof(T) * 7 * kAH * kAW;
    static constexpr size_t kBBytes    = sizeof(T) * 7 * TY * kTX;
    static constexpr size_t kStageA    = align_up(kMbarBytes + 16, 128);
    static constexpr size_t kStageB    = align_up(kStageA + kABytes, 128);
    // + 128: the kernel rounds the dynamic shared-memory base up to 128 B
    static constexpr size_t kBytes     = (TMA ? kStageB + kBBytes : kMbarBytes + 16) + 128;
    static_assert(kFP >= TY * (kTX + 1), "x-face plane");
};

// Boundary-condition map of one coordinate: absorbing clamps to the edge
// cell, reflecting mirrors (-1-i on the left, 2n-1-i on the right) and
// flips the sign of the normal momentum (BoundaryConditions.h:60-109).
// Halo faces never reach it: the stage sees a slab with its stored ghost
// planes as one extended domain.
__device__ __forceinline__ int bc_map(int i, const int n, const int lo, const int hi, bool& flip)
{
    if (i < 0)       { flip = (lo == BC_REFLECTING); i = flip ? -1 - i : 0; }
    else if (i >= n) { flip = (hi == BC_REFLECTING); i = flip ? 2 * n - 1 - i : n - 1; }
    else             { flip = false; }
    return min(max(i, 0), n - 1);
}

struct DomRegs
{
    int nx, ny, nz;
    int bc0, bc1, bc2, bc3, bc4, bc5;
    long long fs;
};

// Bounds-checking build (MPCF_CHECK_BOUNDS, libmpcf_b200_check.so): every
// computed shared-memory and global index of the stage kernel is checked
// against its region; one outside sets ERRBIT_BOUNDS and is clamped into the
// region, so no access leaves its buffer (the results are then void).
// Without the flag the checks compile to nothing.
#ifdef MPCF_CHECK_BOUNDS
template <class I> __device__ __forceinline__ I in_bounds(const I i, const I lo, const I hi, bool& oob)
{
    if (i < lo || i >= hi) { oob = true; return lo; }
    return i;
}
#define MPCF_IN(i, lo, hi) in_bounds<decltype(i)>((i), (decltype(i))(lo), (decltype(i))(hi), oob)
#else
#define MPCF_IN(i, lo, hi) (i)
#endif

// Load the conserved state of (ix,iy,iz) (any integers: out-of-domain cells
// are synthesised from the boundary conditions) and convert to primitives.
template <class Pol>
__device__ __forceinline__ void load_prim(const DomRegs& D, const typename Pol::T* __restrict__ U,
                                          int ix, int iy, int iz, typename Pol::T q[7], bool& oob)
{
    (void)oob;
    typedef typename Pol::T T;
    bool fx, fy, fz;
    ix = bc_map(ix, D.nx, D.bc0, D.bc1, fx);
    iy = bc_map(iy, D.ny, D.bc2, D.bc3, fy);
    iz = bc_map(iz, D.nz, D.bc4, D.bc5, fz);
    const long long idx = MPCF_IN((long long)ix + (long long)D.nx * ((long long)iy + (long long)D.ny * iz),
                                  0, (long long)D.nx * D.ny * D.nz);
    T c[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) c[k] = __ldg(U + k * D.fs + idx);
    if (fx) c[1] = -c[1];
    if (fy) c[2] = -c[2];
    if (fz) c[3] = -c[3];
    to_primitive<Pol>(c, q);
}

template <class T>
__device__ __forceinline__ bool physical(const T r, const T e, const T G, const T P)
{
    // also false for NaN.  P is only required to be finite: it is 0 in pure
    // gas, and the update leaves round-off there (about -1e-17 in every
    // precision on a bubble cloud).  A state without a real sound speed
    // (p + pc <= 0) is flagged by the sound speed (ERRBIT_SOS).
    return (r > (T)0) && (e > (T)0) && (G > (T)0) && (e < (T)INFINITY) && (r < (T)INFINITY) &&
           (P < (T)INFINITY) && (P > -(T)INFINITY);
}

// ---------------------------------------------------------------------------
// Bulk tensor copies (TMA) and mbarriers, hand-written PTX for sm_100a.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

// Bounded wait for the phase with parity `parity`; false after the limit:
// 2^18 polls, about 1.3 s on the B200 (a copy completes in microseconds).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (int i = 0; i < (1 << 18); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Prefetch the 128-byte line holding `p` into L1 (no register written).
__device__ __forceinline__ void prefetch_l1(const void* p)
{
    asm volatile("prefetch.global.L1 [%0];" :: "l"(p));
}

// Generic-proxy accesses of this thread before async-proxy (bulk copy)
// accesses that follow: orders shared-memory reuse of a staging buffer.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 4-D tile copy global -> shared, completion counted on `bar` (no multicast).
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* tmap, int c0, int c1, int c2, int c3, uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5}], [%6];"
                 :: "r"(dst), "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar) : "memory");
}

// Register budget: at least kMinWarpsPerSM resident warps per SM.  The
// face pipeline has 14 independent reconstructions, so the compiler would
// otherwise trade occupancy for unbounded instruction-level parallelism.
// FP64 values take two registers, so its budget is half the warps.
#ifndef MPCF_MIN_WARPS_PER_SM
#define MPCF_MIN_WARPS_PER_SM 16
#endif
// Tile heights of the form 2^n - 1 (3, 7, 15) carry a helper warp that
// takes the tile's extra jobs (ghost rows and columns, the faces above and
// right of the tile); other heights (8) give them to warps 0..4, one each
// (the reference-rounding forms spread the ghost reconstructions over all
// warps), which suits domains whose y extents are multiples of 8.
template <int TY> struct TileShape
{
    static constexpr bool kHelper = ((TY + 1) & TY) == 0;
    static constexpr int kWarps = kHelper ? TY + 1 : TY;
};

template <class T, int TY> struct MinBlocks
{
    static constexpr int w = sizeof(T) == 8 ? MPCF_MIN_WARPS_PER_SM / 2 : MPCF_MIN_WARPS_PER_SM;
    static constexpr int v = (w / TileShape<TY>::kWarps) > 0 ? (w / TileShape<TY>::kWarps) : 1;
};

// Threads of one CTA: TY column warps and, with a helper, the helper warp.
template <int TY> __host__ __device__ constexpr int stage_threads() { return kTX * TileShape<TY>::kWarps; }

// Ghost job g of a tile (0: row -1, 1: row TY, 2: columns -1 and 32) for
// lane tx: the centre of the stencil in the cur slab, its step, and the face
// slot that takes the edge value (dR: a minus slot, from the right / upper
// edge; dL: a plus slot, from the left / lower edge).  Columns -1 and 32
// take lanes 0..TY-1 and 16..15+TY; false for the idle lanes.
template <class L, int TY>
__device__ __forceinline__ bool ghost_job(const int g, const int tx, int& base, int& step, int& dR, int& dL)
{
    if (g == 0)      { base = L::kCurOff + 2 * L::kCurW + tx + 3;        step = L::kCurW; dR = L::kFy + tx; }
    else if (g == 1) { base = L::kCurOff + (TY + 3) * L::kCurW + tx + 3; step = L::kCurW; dL = L::kFy + TY * kTX + tx; }
    else if (tx < TY)                  { base = L::kCurOff + (tx + 3) * L::kCurW + 2;        step = 1; dR = L::kFx + tx * (kTX + 1); }
    else if (tx >= 16 && tx < 16 + TY) { base = L::kCurOff + (tx - 13) * L::kCurW + kTX + 3; step = 1; dL = L::kFx + (tx - 16) * (kTX + 1) + kTX; }
    else return false;
    return true;
}

template <class Pol, int TY, bool PERSIST, bool SUMS, bool TMA>
__global__ void __launch_bounds__(stage_threads<TY>(), MinBlocks<typename Pol::T, TY>::v)
stage_kernel(const StageArgs A)
{
    typedef typename Pol::T T;
    typedef StageLayout<T, TY, TMA> L;
#ifdef MPCF_CHECK_BOUNDS
    // slot 0 of a face plane, x or y faces
    auto face_slot = [](const int d) { return (d >= L::kFx && d < L::kFx + L::kFP) || (d >= L::kFy && d < L::kFy + L::kFP); };
#endif
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    // 128-byte aligned base (bulk tensor copies need it for their targets)
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);
    T* sm = reinterpret_cast<T*>(smem_raw);
    double* red = reinterpret_cast<double*>(smem_raw + L::kRedBytes);
    int* tile_bc = reinterpret_cast<int*>(smem_raw + L::kTileBytes);
    const uint32_t barA = smem_u32(smem_raw + L::kMbarBytes);
    const uint32_t barB = barA + 8;
    T* stA = reinterpret_cast<T*>(smem_raw + L::kStageA);
    T* stB = reinterpret_cast<T*>(smem_raw + L::kStageB);

    const int tx = threadIdx.x & (kTX - 1);
    const int ty = threadIdx.x >> 5;
    const T a = (T)A.a;
    const T b = (T)A.b;
    const T factor6 = (T)1.0f / (T)6.0f;   // GPUkernels.cu:1103
    bool ok = true;
    bool oob = false;                      // bounds-checking build: an index left its buffer
    uint32_t phA = 0, phB = 0;             // mbarrier phase parities
    __shared__ T sos_w[TileShape<TY>::kWarps];   // per-warp maxima of the fused sound speed
    // A thread whose bounded wait runs out sets tma_late and waits for no
    // further copy.  Thread 0 issues every copy; once it has given up it
    // issues none, and before the CTA takes another tile or exits it waits
    // (bounded again) for its copies that no wait of its own has seen
    // complete: pendA/pendB, with the parity of that copy's phase.
    bool tma_late = false;
    bool pendA = false, pendB = false;
    uint32_t parA = 0, parB = 0;
    bool tma_inflight = false;             // a drain wait ran out as well
    // thread 0: one bulk copy into stage buffer `st` (barrier `bar`), with
    // its phase recorded as pending (and counted in failure-detection tests)
    auto issue = [&](const char* tmap, const bool isA, const int c0, const int c1, const int c2)
    {
        if (isA) { mbar_expect_tx(barA, (uint32_t)L::kABytes); tma_load_4d(smem_u32(stA), tmap, c0, c1, c2, 0, barA); pendA = true; parA = phA; }
        else     { mbar_expect_tx(barB, (uint32_t)L::kBBytes); tma_load_4d(smem_u32(stB), tmap + 128, c0, c1, c2, 0, barB); pendB = true; parB = phB; }
        if (A.test_flags) atomicAdd(A.counter + 1, 1u);
    };
    // bounded wait of this thread on `bar` for phase `ph`; thread 0 clears
    // the copy's pending mark when it sees it complete
    auto wait_copy = [&](const bool isA)
    {
        if (tma_late) return;
        if (!mbar_wait(isA ? barA : barB, isA ? phA : phB)) { tma_late = true; return; }
        if (threadIdx.x == 0) { if (isA) pendA = false; else pendB = false; }
    };

    if (TMA)
    {
        if (threadIdx.x == 0) { mbar_init(barA, 1); mbar_init(barB, 1); mbar_init_fence(); }
        __syncthreads();
    }

    // tiles tile0 .. ntiles-1: from the work counter, or one per CTA
    int t;
    if (PERSIST)
    {
        if (threadIdx.x == 0) *tile_bc = A.tile0 + (int)atomicAdd(A.counter, 1u);
        __syncthreads();
        t = *tile_bc;
    }
    else t = A.tile0 + blockIdx.x;

    while (t < A.ntiles)
    {
        // ---- decode tile -> domain, tile coordinates
        int d = 0;
        while (d + 1 < A.ndom && A.doms[d + 1].tile_begin <= t) ++d;
        const DomDev& DD = A.doms[d];
        // A slab with halo faces is seen as its extended domain, stored
        // ghost planes included (planes -zlo .. nz-1+zhi become 0 ..
        // nz+zlo+zhi-1); only its own planes zlo .. zlo+nz-1 are advanced, so
        // no stencil ever reaches past the stored planes on a halo side.
        DomRegs D;
        D.nx = DD.nx; D.ny = DD.ny; D.nz = DD.nzx;
        D.bc0 = DD.bc[0]; D.bc1 = DD.bc[1]; D.bc2 = DD.bc[2];
        D.bc3 = DD.bc[3]; D.bc4 = DD.bc[4]; D.bc5 = DD.bc[5];
        D.fs = DD.fs;
        const T* __restrict__ U    = (const T*)DD.Ux[A.parity];
        T* __restrict__       Un   = (T*)DD.Ux[A.parity ^ 1];
        T* __restrict__       R    = (T*)DD.Rx;
        const T dtinvh = ((const T*)A.dtinvh)[d];
        const bool use_tma = TMA && DD.tma_ok;
        // tensor maps of the buffer read in this stage: halo box, interior box
        const char* tm = (const char*)A.tmaps + ((size_t)d * 4 + (size_t)A.parity * 2) * 128;

        const int lt = t - DD.tile_begin;
        const int bx = lt % DD.tiles_x;
        const int by = (lt / DD.tiles_x) % DD.tiles_y;
        const int bz = lt / (DD.tiles_x * DD.tiles_y);
        const int x0 = bx * kTX, y0 = by * TY;
        const int z0 = DD.zlo + bz * A.dz;
        const int z1 = min(z0 + A.dz, DD.zlo + DD.nz);
        const int gx = x0 + tx, gy = y0 + ty;
        const bool row = ty < TY;          // a column thread (not the helper)
        const bool valid = row && (gx < D.nx) && (gy < D.ny);
        const int own = ty * kTX + tx;     // own column inside a ring slot
        // the tile's columns are all inside the domain: its ring holds the
        // exact primitives of every cur interior cell
        const bool full = (x0 + kTX <= D.nx) && (y0 + TY <= D.ny);
        // the staged halo box needs no boundary mapping in x and y
        const bool inner = (x0 >= 4) && (x0 + kTX + 4 <= D.nx) && (y0 >= 3) && (y0 + TY + 3 <= D.ny);

        // ---- prologue: slabs z0-3 .. z0+1 of the own column into the ring
        for (int sl = z0 - 3; row && sl <= z0 + 1; ++sl)
        {
            T q[7];
            load_prim<Pol>(D, U, gx, gy, sl, q, oob);
            const int slot = (sl + 6) % 6;
            const int ri = MPCF_IN(slot * L::kRing + own, 0, L::kCurOff);
#pragma unroll
            for (int m = 0; m < 7; ++m) sm[m * L::kPP + ri] = q[m];
        }
        if (use_tma && threadIdx.x == 0 && !tma_late)
        {
            // first copies: halo box of slab z0 and interior of slab z0+2
            bool fz;
            fence_proxy_async();
            issue(tm, true, x0 - 4, y0 - 3, bc_map(z0, D.nz, D.bc4, D.bc5, fz));
            issue(tm, false, x0, y0, bc_map(z0 + 2, D.nz, D.bc4, D.bc5, fz));
        }

        T Sp[7];                 // x/y part of the flux bracket of cell k-1
        T sG = 0, sP = 0, dU = 0;
        T zfp[12];               // z face (k-1)-1/2
        T Rzp[7];                // per-cell z: right edge of cell k-1 (minus side of face k-1/2)
#pragma unroll
        for (int m = 0; m < 7; ++m) Sp[m] = 0;
#pragma unroll
        for (int m = 0; m < 12; ++m) zfp[m] = 0;
        double cs[5] = {0, 0, 0, 0, 0};
        T smax = 0;              // fused sound speed of the new state (last stage)
        bool sbad = false;

        for (int k = z0; k <= z1; ++k)
        {
            // (A) leading slab k+2 of the own column
            if (row)
            {
                const int slot = (k + 2 + 6) % 6;
                T q[7];
                if (use_tma)
                {
                    wait_copy(false);
                    phB ^= 1;
                    bool fx = false, fy = false, fz;
                    int mx = tx, my = ty;
                    if (!full)
                    {
                        mx = min(max(bc_map(gx, D.nx, D.bc0, D.bc1, fx) - x0, 0), kTX - 1);
                        my = min(max(bc_map(gy, D.ny, D.bc2, D.bc3, fy) - y0, 0), TY - 1);
                    }
                    bc_map(k + 2, D.nz, D.bc4, D.bc5, fz);
                    T c[7];
                    const int bi = MPCF_IN(my * kTX + mx, 0, TY * kTX);
#pragma unroll
                    for (int m = 0; m < 7; ++m) c[m] = stB[m * TY * kTX + bi];
                    if (fx) c[1] = -c[1];
                    if (fy) c[2] = -c[2];
                    if (fz) c[3] = -c[3];
                    to_primitive<Pol>(c, q);
                }
                else load_prim<Pol>(D, U, gx, gy, k + 2, q, oob);
                const int ri = MPCF_IN(slot * L::kRing + own, 0, L::kCurOff);
#pragma unroll
                for (int m = 0; m < 7; ++m) sm[m * L::kPP + ri] = q[m];
            }
            // (B) slab k with halos into cur (slab k < nz: no z mapping)
            if (k < z1)
            {
                const int slot = k % 6;
                if (use_tma && !full)
                {
                    // tile reaching past the domain: convert the whole staged
                    // box, mapping out-of-domain cells to their sources
                    wait_copy(true);
                    phA ^= 1;
                    for (int i = threadIdx.x; i < (TY + 6) * L::kCurW; i += stage_threads<TY>())
                    {
                        const int ly = i / L::kCurW - 3, lx = i % L::kCurW - 3;
                        bool fx, fy;
                        const int mx = min(max(bc_map(x0 + lx, D.nx, D.bc0, D.bc1, fx) - x0 + 4, 0), L::kAW - 1);
                        const int my = min(max(bc_map(y0 + ly, D.ny, D.bc2, D.bc3, fy) - y0 + 3, 0), L::kAH - 1);
                        T c[7], q[7];
                        const int ai = MPCF_IN(my * L::kAW + mx, 0, L::kAH * L::kAW);
#pragma unroll
                        for (int m = 0; m < 7; ++m) c[m] = stA[m * L::kAH * L::kAW + ai];
                        if (fx) c[1] = -c[1];
                        if (fy) c[2] = -c[2];
                        to_primitive<Pol>(c, q);
                        const int ci = MPCF_IN(L::kCurOff + (ly + 3) * L::kCurW + lx + 3, L::kCurOff, L::kPP);
#pragma unroll
                        for (int m = 0; m < 7; ++m) sm[m * L::kPP + ci] = q[m];
                    }
                }
                else
                {
                    // interior from the ring, then the 6*32 + 6*TY halo cells
                    // the x/y stencils read (the corners are never read)
                    if (row)
                    {
                        const int ci = MPCF_IN(L::kCurOff + (ty + 3) * L::kCurW + tx + 3, L::kCurOff, L::kPP);
                        const int ri = MPCF_IN(slot * L::kRing + own, 0, L::kCurOff);
#pragma unroll
                        for (int m = 0; m < 7; ++m)
                            sm[m * L::kPP + ci] = sm[m * L::kPP + ri];
                    }
                    if (use_tma)
                    {
                        wait_copy(true);
                        phA ^= 1;
                    }
                    for (int i = threadIdx.x; i < 6 * kTX + 6 * TY; i += stage_threads<TY>())
                    {
                        int lx, ly;
                        if (i < 6 * kTX)
                        {
                            const int r = i >> 5;
                            lx = i & (kTX - 1);
                            ly = r < 3 ? r - 3 : TY + r - 3;
                        }
                        else
                        {
                            const int j = i - 6 * kTX;
                            const int c = j % 6;
                            ly = j / 6;
                            lx = c < 3 ? c - 3 : kTX + c - 3;
                        }
                        T q[7];
                        if (use_tma)
                        {
                            bool fx = false, fy = false;
                            int mx = lx + 4, my = ly + 3;
                            if (!inner)
                            {
                                mx = min(max(bc_map(x0 + lx, D.nx, D.bc0, D.bc1, fx) - x0 + 4, 0), L::kAW - 1);
                                my = min(max(bc_map(y0 + ly, D.ny, D.bc2, D.bc3, fy) - y0 + 3, 0), L::kAH - 1);
                            }
                            T c[7];
                            const int ai = MPCF_IN(my * L::kAW + mx, 0, L::kAH * L::kAW);
#pragma unroll
                            for (int m = 0; m < 7; ++m) c[m] = stA[m * L::kAH * L::kAW + ai];
                            if (fx) c[1] = -c[1];
                            if (fy) c[2] = -c[2];
                            to_primitive<Pol>(c, q);
                        }
                        else load_prim<Pol>(D, U, x0 + lx, y0 + ly, k, q, oob);
                        const int ci = MPCF_IN(L::kCurOff + (ly + 3) * L::kCurW + lx + 3, L::kCurOff, L::kPP);
#pragma unroll
                        for (int m = 0; m < 7; ++m) sm[m * L::kPP + ci] = q[m];
                    }
                }
            }
            __syncthreads();
            // the staging buffers are free again: copy the next slab's data
            // while this slab's faces are evaluated
            if (use_tma && threadIdx.x == 0 && !tma_late)
            {
                bool fz;
                fence_proxy_async();
                if (k + 1 <= z1)
                {
                    // the failure-detection tests arm the barrier of a copy
                    // without issuing it: the chunk's last copy, or its
                    // first copy after the prologue (then later waits find
                    // the CTA given up, and no further copy is issued)
                    const bool drop = !PERSIST && (((A.test_flags & TEST_DROP_LAST_COPY) && k + 1 == z1) ||
                                                   ((A.test_flags & TEST_DROP_MID_COPY) && k == z0));
                    if (drop) mbar_expect_tx(barB, (uint32_t)L::kBBytes);
                    else      issue(tm, false, x0, y0, bc_map(k + 3, D.nz, D.bc4, D.bc5, fz));
                }
                if (k + 1 < z1) issue(tm, true, x0 - 4, y0 - 3, bc_map(k + 1, D.nz, D.bc4, D.bc5, fz));
            }

            // R and U of cell k-1 are first prefetched into L1, so that its
            // finalisation after the z face finds them.
            const bool fin = (k > z0) && valid;
#ifdef MPCF_CHECK_BOUNDS
            // cell k-1 of the own column: inside the domain's own planes
            const long long idx = fin ? MPCF_IN((long long)gx + (long long)D.nx * ((long long)gy + (long long)D.ny * (k - 1)),
                                                (long long)DD.zlo * DD.nx * DD.ny, (long long)(DD.zlo + DD.nz) * DD.nx * DD.ny)
                                      : 0;
#else
            const long long idx = (long long)gx + (long long)D.nx * ((long long)gy + (long long)D.ny * (k - 1));
#endif
            if (fin)
            {
#pragma unroll
                for (int m = 0; m < 7; ++m) { prefetch_l1(R + m * D.fs + idx); prefetch_l1(U + m * D.fs + idx); }
            }
            // (E) finalisation of cell k-1 of the own column from the z face
            // k-1/2: rhs = a*R - dtinvh*div(F) (with the G/P extra terms),
            // R <- rhs, U_next <- b*rhs + U.  It reads only this thread's
            // registers and global memory.
            auto finalize = [&](const FaceOut<T>& zf)
            {
                T Rold[7], Uold[7];
#pragma unroll
                for (int m = 0; m < 7; ++m) { Rold[m] = R[m * D.fs + idx]; Uold[m] = __ldg(U + m * D.fs + idx); }
                const T sumG = sG + (zfp[8] + zf.Gm);
                const T sumP = sP + (zfp[10] + zf.Pm);
                const T divU = dU + (zf.vel - zfp[11]);
                T un[7];
#pragma unroll
                for (int m = 0; m < 7; ++m)
                {
                    T br = (Sp[m] + zf.f[m]) - zfp[m];
                    if (m == 5) br = br - divU * sumG * factor6;
                    if (m == 6) br = br - divU * sumP * factor6;
                    const T rhs_m = dtinvh * br;
                    const T rhs = a * Rold[m] - rhs_m;
                    R[m * D.fs + idx] = rhs;
                    un[m] = b * rhs + Uold[m];
                    Un[m * D.fs + idx] = un[m];
                }
                ok = ok && physical<T>(un[0], un[4], un[5], un[6]);
                if (A.sos_bits)
                {
                    const T v = cell_sos_rn<Pol>(un[0], un[1], un[2], un[3], un[4], un[5], un[6]);
                    sbad = sbad || !(v >= (T)0);   // NaN (the maximum would drop it) or negative
                    smax = dmax(smax, v);
                }
                if (SUMS)
                {
#pragma unroll
                    for (int m = 0; m < 5; ++m) cs[m] += (double)un[m];
                }
            };
            FaceOut<T> zf;
            {
                // (C) per-cell reconstruction and faces of slab k.
                //  1. z (column threads): the right edge of cell k-1 (first
                //     slab of a chunk only; later it is carried), both edges
                //     of cell k, the z face k-1/2 from them, then cell k-1 is
                //     finalised;
                //  2. x and y edges of the own cell into the face slots: the
                //     right / upper edge to the minus side of the face right
                //     of / above the cell, the left / lower edge to the plus
                //     side of the face left of / below it.  The helper warp
                //     (without one: warps 0..2, or all warps in shares)
                //     reconstructs the ghost cells around the tile: row -1,
                //     row TY, columns -1 and 32;
                //  3. after a barrier, the x face left of the own cell and the
                //     y face below it, each evaluated in place in its slot;
                //     the helper (warps 3 and 4 without one) evaluates the y
                //     faces above the tile and the x faces right of it.  Without
                //     a helper no warp takes more than one of the extra jobs,
                //     which keeps the warps even at the barriers.
                constexpr bool kHelper = TileShape<TY>::kHelper;
                static_assert(TY <= 16, "ghost columns -1 and 32 take lanes 0..TY-1 and 16..15+TY");
                static_assert(kHelper || TY >= 5, "without a helper, warps 0..4 take the extra jobs");
                if (row)
                {
#pragma unroll 1
                    for (int cz = (k == z0) ? k - 1 : k; cz <= k; ++cz)
                    {
                        // ring slots of slabs cz-2 .. cz+2
                        const int zs = (cz + 4) % 6;
                        int ad[5];
#pragma unroll
                        for (int j = 0; j < 5; ++j) ad[j] = MPCF_IN((zs + j < 6 ? zs + j : zs + j - 6) * L::kRing + own, 0, L::kCurOff);
                        T Rv[7], Lv[7];
#pragma unroll
                        for (int q = 0; q < 7; ++q)
                        {
                            const T* pl = sm + q * L::kPP;
                            weno_cell<Pol>(pl[ad[0]], pl[ad[1]], pl[ad[2]], pl[ad[3]], pl[ad[4]], Rv[q], Lv[q]);
                        }
                        if (cz == k)
                        {
                            // z: normal w, transverse u, v
                            FaceState<T> S;
                            S.rm = Rzp[0]; S.rp = Lv[0]; S.nm = Rzp[3]; S.np = Lv[3];
                            S.t1m = Rzp[1]; S.t1p = Lv[1]; S.t2m = Rzp[2]; S.t2p = Lv[2];
                            S.pm = Rzp[4]; S.pp = Lv[4]; S.Gm = Rzp[5]; S.Gp = Lv[5]; S.Pm = Rzp[6]; S.Pp = Lv[6];
                            face_hllc<Pol>(S, 2, zf);
                        }
#pragma unroll
                        for (int q = 0; q < 7; ++q) Rzp[q] = Rv[q];
                    }
                    if (fin) finalize(zf);
#pragma unroll
                    for (int m = 0; m < 7; ++m) zfp[m] = zf.f[m];
                    zfp[7] = zf.Gm; zfp[8] = zf.Gp; zfp[9] = zf.Pm; zfp[10] = zf.Pp; zfp[11] = zf.vel;
                }
                // the fast forms run the x/y loops unrolled by two (both loops:
                // 3% faster at 512^3); the reference-rounding forms, with their
                // double-promoted weights, keep one copy of each
                constexpr int kXYUnroll = Pol::kFastWeno ? 2 : 1;
                if (k < z1)
                {
                    // Own cells (x, then y) and the three ghost jobs: with a
                    // helper, the helper warp takes them whole (it has no z
                    // part); without one, in the fast forms warps 0..2 take
                    // one each, and in the other forms every warp takes a
                    // share of their 21 planes (below).
                    constexpr bool kSplitGhosts = !kHelper && !Pol::kFastWeno;
                    const int nr = row ? ((!kHelper && !kSplitGhosts && ty < 3) ? 3 : 2) : 3;
#pragma unroll kXYUnroll
                    for (int j = 0; j < nr; ++j)
                    {
                        int base, step, dR = -1, dL = -1;
                        if (row && j < 2)
                        {
                            // own cell: j = 0 x, j = 1 y
                            base = L::kCurOff + (ty + 3) * L::kCurW + tx + 3;
                            step = j ? L::kCurW : 1;
                            dL = j ? L::kFy + ty * kTX + tx : L::kFx + ty * (kTX + 1) + tx;
                            dR = j ? dL + kTX : dL + 1;
                        }
                        else if (!ghost_job<L, TY>(row ? ty : j, tx, base, step, dR, dL)) continue;
#ifdef MPCF_CHECK_BOUNDS
                        if (base - 2 * step < L::kCurOff || base + 2 * step >= L::kPP) { oob = true; base = L::kCurOff + 2 * step; }
                        if (dR >= 0 && !face_slot(dR)) { oob = true; dR = -1; }
                        if (dL >= 0 && !face_slot(dL)) { oob = true; dL = -1; }
#endif
                        T Rv[7], Lv[7];
#pragma unroll
                        for (int q = 0; q < 7; ++q)
                        {
                            const T* pl = sm + q * L::kPP + base;
                            weno_cell<Pol>(pl[-2 * step], pl[-step], pl[0], pl[step], pl[2 * step], Rv[q], Lv[q]);
                        }
                        if (dR >= 0)
                        {
#pragma unroll
                            for (int q = 0; q < 7; ++q) sm[dR + q * L::kFP] = Rv[q];
                        }
                        if (dL >= 0)
                        {
#pragma unroll
                            for (int q = 0; q < 7; ++q) sm[dL + (7 + q) * L::kFP] = Lv[q];
                        }
                    }
                    if constexpr (kSplitGhosts)
                    {
                        // The 21 planes of the ghost jobs (3 jobs x 7
                        // quantities) in contiguous ranges over the warps
                        // (TY = 8: warps 0..4 take 3, the others 2), so that no
                        // warp reaches the barrier 7 planes after another.  In
                        // the reference-rounding forms this is 5% faster at
                        // TY = 8; the fast forms lose the independent chains of
                        // a whole job and are 3% slower with it.
                        constexpr int kPer = 21 / TY, kRem = 21 % TY;
                        int gi = ty * kPer + (ty < kRem ? ty : kRem);
                        const int ge = gi + kPer + (ty < kRem ? 1 : 0);
#pragma unroll 1
                        for (; gi < ge; ++gi)
                        {
                            const int g = gi >= 14 ? 2 : (gi >= 7 ? 1 : 0);
                            const int q = gi - 7 * g;
                            int base, step, dR = -1, dL = -1;
                            if (!ghost_job<L, TY>(g, tx, base, step, dR, dL)) continue;
#ifdef MPCF_CHECK_BOUNDS
                            if (base - 2 * step < L::kCurOff || base + 2 * step >= L::kPP) { oob = true; base = L::kCurOff + 2 * step; }
                            if (dR >= 0 && !face_slot(dR)) { oob = true; continue; }
                            if (dL >= 0 && !face_slot(dL)) { oob = true; continue; }
#endif
                            const T* pl = sm + q * L::kPP + base;
                            T rv, lv;
                            weno_cell<Pol>(pl[-2 * step], pl[-step], pl[0], pl[step], pl[2 * step], rv, lv);
                            // the right / upper edge fills a minus slot, the
                            // left / lower edge a plus slot
                            if (dR >= 0) sm[dR + q * L::kFP] = rv;
                            else         sm[dL + (7 + q) * L::kFP] = lv;
                        }
                    }
                    __syncthreads();
                    const int nh = row ? ((!kHelper && (ty == 3 || ty == 4)) ? 3 : 2) : 2;
#pragma unroll kXYUnroll
                    for (int j = 0; j < nh; ++j)
                    {
                        int src, dir;
                        if (row && j < 2) { dir = j; src = j ? L::kFy + ty * kTX + tx : L::kFx + ty * (kTX + 1) + tx; }
                        else
                        {
                            const int g = row ? ty - 2 : j + 1;   // 1: y faces above, 2: x faces right
                            if (g == 1) { dir = 1; src = L::kFy + TY * kTX + tx; }
                            else
                            {
                                if (tx >= TY) continue;
                                dir = 0; src = L::kFx + tx * (kTX + 1) + kTX;
                            }
                        }
#ifdef MPCF_CHECK_BOUNDS
                        if (!face_slot(src)) { oob = true; continue; }
#endif
                        // x: normal u, transverse v, w;  y: normal v, transverse u, w
                        T* pl = sm + src;
                        const int nq = 1 + dir, tq = 2 - dir;
                        FaceState<T> S;
                        S.rm  = pl[0];              S.rp  = pl[7 * L::kFP];
                        S.nm  = pl[nq * L::kFP];    S.np  = pl[(7 + nq) * L::kFP];
                        S.t1m = pl[tq * L::kFP];    S.t1p = pl[(7 + tq) * L::kFP];
                        S.t2m = pl[3 * L::kFP];     S.t2p = pl[10 * L::kFP];
                        S.pm  = pl[4 * L::kFP];     S.pp  = pl[11 * L::kFP];
                        S.Gm  = pl[5 * L::kFP];     S.Gp  = pl[12 * L::kFP];
                        S.Pm  = pl[6 * L::kFP];     S.Pp  = pl[13 * L::kFP];
                        FaceOut<T> o;
                        face_hllc<Pol>(S, dir, o);
#pragma unroll
                        for (int m = 0; m < 7; ++m) pl[m * L::kFP] = o.f[m];
                        pl[7 * L::kFP] = o.Gm;  pl[8 * L::kFP] = o.Gp;
                        pl[9 * L::kFP] = o.Pm;  pl[10 * L::kFP] = o.Pp;
                        pl[11 * L::kFP] = o.vel;
                    }
                }
            }
            __syncthreads();

            // (F) x/y part of cell k, carried to the next slab
            if (k < z1 && row)
            {
                // the slot right of / above the cell is read too
                const T* fx = sm + L::kFx + MPCF_IN(ty * (kTX + 1) + tx, 0, L::kFP - 1);
                const T* fy = sm + L::kFy + MPCF_IN(ty * kTX + tx, 0, L::kFP - kTX);
#pragma unroll
                for (int m = 0; m < 7; ++m)
                    Sp[m] = ((fx[m * L::kFP + 1] - fx[m * L::kFP]) + fy[m * L::kFP + kTX]) - fy[m * L::kFP];
                sG = fx[8 * L::kFP] + fx[7 * L::kFP + 1];
                sP = fx[10 * L::kFP] + fx[9 * L::kFP + 1];
                dU = fx[11 * L::kFP + 1] - fx[11 * L::kFP];
                sG = sG + (fy[8 * L::kFP] + fy[7 * L::kFP + kTX]);
                sP = sP + (fy[10 * L::kFP] + fy[9 * L::kFP + kTX]);
                dU = dU + (fy[11 * L::kFP + kTX] - fy[11 * L::kFP]);
            }
        }

        // ---- fused sound-speed maximum of the tile into its domain's
        // accumulator (the stand-alone reduction's order of the bits)
        if (A.sos_bits)
        {
            const bool bad = __syncthreads_or(sbad);
            const T m = shfl_max(smax);
            if (tx == 0) sos_w[ty] = m;
            __syncthreads();
            if (threadIdx.x < 32)
            {
                // every warp of the CTA wrote its slot (a helper warp its 0)
                T mm = threadIdx.x < TileShape<TY>::kWarps ? sos_w[threadIdx.x] : (T)0;
                mm = shfl_max(mm);
                if (threadIdx.x == 0) atomic_max_bits((char*)A.sos_bits + (size_t)d * sizeof(T), bad ? (T)NAN : mm);
            }
        }

        // ---- per-tile FP64 conservation sums (deterministic: fixed order)
        if (SUMS)
        {
#pragma unroll
            for (int m = 0; m < 5; ++m)
            {
                double v = cs[m];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                if (tx == 0 && row) red[ty * 5 + m] = v;
            }
            __syncthreads();
            if (threadIdx.x < 5)
            {
                double v = 0;
                for (int w = 0; w < TY; ++w) v += red[w * 5 + threadIdx.x];
                A.tile_sums[(long long)t * 5 + threadIdx.x] = v;
            }
        }

        // copies this CTA issued and no wait of thread 0 saw complete (only
        // after a wait ran out): wait for them, bounded, so that none lands
        // in shared memory the CTA no longer owns; a CTA that gave up takes
        // no further tile
        if (TMA && threadIdx.x == 0 && (pendA || pendB))
        {
            if (pendA && !mbar_wait(barA, parA)) tma_inflight = true;
            if (pendB && !mbar_wait(barB, parB)) tma_inflight = true;
            pendA = pendB = false;
        }
        if (!PERSIST) break;
        __syncthreads();
        if (threadIdx.x == 0) *tile_bc = tma_late ? A.ntiles : A.tile0 + (int)atomicAdd(A.counter, 1u);
        __syncthreads();
        t = *tile_bc;
    }

    if (!__all_sync(0xffffffffu, ok) && tx == 0) atomicOr(A.err, (unsigned)ERRBIT_NONPHYSICAL);
    if (TMA && tma_late) atomicOr(A.err, (unsigned)ERRBIT_TMA_TIMEOUT);
    if (TMA && tma_inflight) atomicOr(A.err, (unsigned)ERRBIT_TMA_INFLIGHT);
#ifdef MPCF_CHECK_BOUNDS
    if (__any_sync(0xffffffffu, oob) && tx == 0) atomicOr(A.err, (unsigned)ERRBIT_BOUNDS);
#endif
}

template <class Pol, int TY, bool TMA>
constexpr size_t stage_smem_bytes() { return StageLayout<typename Pol::T, TY, TMA>::kBytes; }

} // namespace mpcf
