// mpcf_aux.cu -- the small kernels around the stage: maximum speed of sound
// (CFL reduction), on-device dt, deterministic FP64 conservation sums, the
// bubble-cloud initial condition and an explicit ghost-buffer fill.
#include <cuda_runtime.h>
#include <math.h>
#include <cmath>
#include <algorithm>
#include <mutex>
#include "mpcf_math.cuh"
#include "mpcf_stage.cuh"
#include "mpcf_launch.h"
#include "mpcf_ic.h"

namespace mpcf {

// ---------------------------------------------------------------------------
// Maximum speed of sound.  Per cell (reference formula, GPUkernels.cu:1207-1209):
//   p = (E - (U*U + V*V + W*W)*(0.5f/rho) - P) / G        (U,V,W momenta)
//   c = sqrt(((p + P)/G + p)/rho)
//   s = c + max(|U|,|V|,|W|)/rho
// The mixed policy evaluates p in FP64.  Reduction: warp shuffle, block max
// through shared memory, one atomicMax per block on the bit pattern (all
// values are >= 0, so the unsigned order of the bits is the float order; a
// NaN compares above every finite value and surfaces as the result).
// ---------------------------------------------------------------------------
template <class Pol>
__device__ __forceinline__ typename Pol::T cell_sos(const typename Pol::T r, const typename Pol::T u,
        const typename Pol::T v, const typename Pol::T w, const typename Pol::T e,
        const typename Pol::T G, const typename Pol::T P)
{
    return cell_sos_rn<Pol>(r, u, v, w, e, G, P);
}


template <class Pol>
__global__ void __launch_bounds__(256) sos_kernel(const SosArgs A)
{
    typedef typename Pol::T T;
    __shared__ T wmax[8];
    const int c = A.chunk0 + blockIdx.x;
    int d = 0;
    while (d + 1 < A.ndom && A.doms[d + 1].sos_chunk_begin <= c) ++d;
    const DomDev& D = A.doms[d];
    const long long N = (long long)D.nx * D.ny * D.nz;
    const long long beg = (long long)(c - D.sos_chunk_begin) * A.chunk;
    const long long end = min(beg + (long long)A.chunk, N);
    const T* __restrict__ U = (const T*)D.U[A.parity];
    const long long fs = D.fs;

    T s = (T)0;
    bool bad = false;
    for (long long i = beg + threadIdx.x; i < end; i += blockDim.x)
    {
        const T v = cell_sos<Pol>(__ldg(U + i), __ldg(U + fs + i), __ldg(U + 2 * fs + i), __ldg(U + 3 * fs + i),
                                  __ldg(U + 4 * fs + i), __ldg(U + 5 * fs + i), __ldg(U + 6 * fs + i));
        bad = bad || !(v >= (T)0);   // NaN (fmax would drop it) or negative
        s = dmax(s, v);
    }
    bad = __syncthreads_or(bad);
    s = shfl_max(s);
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        T m = threadIdx.x < (blockDim.x >> 5) ? wmax[threadIdx.x] : (T)0;
        m = shfl_max(m);
        // a NaN's bit pattern orders above every finite non-negative value,
        // so it wins the atomic maximum and reaches the dt kernel
        if (threadIdx.x == 0) atomic_max_bits((char*)A.sos_bits + d * sizeof(T), bad ? (T)NAN : m);
    }
}

// dt = min(CFL*h/sos, dt_max), dt/h rounded to the stage type
// (LSRK3_IntegratorMPI.cpp:37-38, process_all(.., dt/h) converts to Real).
// The sound-speed accumulator is cleared for the next reduction.
template <class Pol>
__device__ __forceinline__ void dt_of_domain(const DtArgs& A, const int d, const typename Pol::T sos)
{
    typedef typename Pol::T T;
    const double h = A.doms[d].h;
    double dt = A.cfl*h/sos;
    dt = A.dt_max < dt ? A.dt_max : dt;
    if (!(sos > (T)0) || !(dt == dt) || isinf(dt))
    {
        atomicOr(A.err, (unsigned)ERRBIT_SOS_NONFINITE);
        dt = 0.0;   // freeze the domain rather than advance it with garbage
    }
    ((T*)A.dtinvh)[d] = (T)(dt/h);
    A.dt[d] = dt;
    A.time[d] += dt;
}

template <class Pol>
__global__ void dt_kernel(const DtArgs A)
{
    typedef typename Pol::T T;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= A.ndom) return;
    T* bits = (T*)A.sos_bits;
    dt_of_domain<Pol>(A, d, bits[d]);
    bits[d] = (T)0;
}

// Linked slabs of one global domain advance with one dt: each domain takes
// the maximum sound speed of its group (a NaN anywhere in the group stays
// NaN and is reported), the minimum dt over the slabs as the reference's
// MPI_Allreduce(MIN) gives it.  One block: the accumulators are cleared
// only after every domain has read its group's.
template <class Pol>
__global__ void dt_group_kernel(const DtArgs A)
{
    typedef typename Pol::T T;
    T* bits = (T*)A.sos_bits;
    for (int d = threadIdx.x; d < A.ndom; d += blockDim.x)
    {
        const int g = A.doms[d].group;
        T sos = bits[d];
        for (int e = 0; e < A.ndom; ++e)
        {
            const T v = bits[e];
            if (A.doms[e].group == g && sos == sos && !(v <= sos)) sos = v;
        }
        dt_of_domain<Pol>(A, d, sos);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < A.ndom; d += blockDim.x) bits[d] = (T)0;
}

cudaError_t launch_sos(int pol, const SosArgs& A, cudaStream_t st)
{
    switch (pol)
    {
        case 0: sos_kernel<PolRef32><<<A.nchunks, 256, 0, st>>>(A); break;
        case 1: sos_kernel<PolFast32><<<A.nchunks, 256, 0, st>>>(A); break;
        case 2: sos_kernel<PolMixed><<<A.nchunks, 256, 0, st>>>(A); break;
        case 3: sos_kernel<PolFP64><<<A.nchunks, 256, 0, st>>>(A); break;
        case 4: sos_kernel<PolFast64><<<A.nchunks, 256, 0, st>>>(A); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_dt(int pol, const DtArgs& A, cudaStream_t st)
{
    const int g = (A.ndom + 63) / 64;
    if (A.grouped)
    {
        switch (pol)
        {
            case 0: dt_group_kernel<PolRef32><<<1, 256, 0, st>>>(A); break;
            case 1: dt_group_kernel<PolFast32><<<1, 256, 0, st>>>(A); break;
            case 2: dt_group_kernel<PolMixed><<<1, 256, 0, st>>>(A); break;
            case 3: dt_group_kernel<PolFP64><<<1, 256, 0, st>>>(A); break;
            case 4: dt_group_kernel<PolFast64><<<1, 256, 0, st>>>(A); break;
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    switch (pol)
    {
        case 0: dt_kernel<PolRef32><<<g, 64, 0, st>>>(A); break;
        case 1: dt_kernel<PolFast32><<<g, 64, 0, st>>>(A); break;
        case 2: dt_kernel<PolMixed><<<g, 64, 0, st>>>(A); break;
        case 3: dt_kernel<PolFP64><<<g, 64, 0, st>>>(A); break;
        case 4: dt_kernel<PolFast64><<<g, 64, 0, st>>>(A); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// Per-domain totals of the per-tile FP64 partial sums.  One block per
// domain: thread i adds tiles i, i+256, ... in order, then a fixed-shape
// tree combines the 256 partials, so the result does not depend on
// scheduling (deterministic run to run).
constexpr int kSumTilesThreads = 256;

__global__ void __launch_bounds__(kSumTilesThreads) sum_tiles_kernel(const DomDev* doms, const double* tile_sums, double* out)
{
    __shared__ double red[5][kSumTilesThreads];
    const int d = blockIdx.x;
    const int tid = threadIdx.x;
    const long long b = doms[d].tile_begin;
    const int n = doms[d].tiles_x * doms[d].tiles_y * doms[d].tiles_z;
    double s[5] = {0, 0, 0, 0, 0};
    for (int t = tid; t < n; t += kSumTilesThreads)
        for (int m = 0; m < 5; ++m) s[m] += tile_sums[(b + t) * 5 + m];
    for (int m = 0; m < 5; ++m) red[m][tid] = s[m];
    __syncthreads();
    for (int w = kSumTilesThreads / 2; w > 0; w >>= 1)
    {
        if (tid < w)
            for (int m = 0; m < 5; ++m) red[m][tid] += red[m][tid + w];
        __syncthreads();
    }
    if (tid < 5) out[d * 5 + tid] = red[tid][0];
}

cudaError_t launch_sum_tiles(const DomDev* doms, int ndom, const double* tile_sums, double* out, cudaStream_t st)
{
    sum_tiles_kernel<<<ndom, kSumTilesThreads, 0, st>>>(doms, tile_sums, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Bubble-cloud initial condition (formula in mpcf_ic.h), one thread per cell,
// grid-stride; the register is cleared.
// ---------------------------------------------------------------------------
template <class T>
__global__ void ic_cloud_kernel(const DomDev* dom, int parity, const IcParams P,
                                const double* __restrict__ bub, int nb)
{
    const DomDev& D = *dom;
    const long long N = (long long)D.nx * D.ny * D.nz;
    T* U = (T*)D.U[parity];
    T* R = (T*)D.R;
    const long long fs = D.fs;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    {
        // the cell's place in the global grid (its noise stream too)
        const int gx = D.org[0] + (int)(i % D.nx);
        const int gy = D.org[1] + (int)((i / D.nx) % D.ny);
        const int gz = D.org[2] + (int)(i / ((long long)D.nx * D.ny));
        const unsigned long long lin = (unsigned long long)gx + (unsigned long long)D.gdim[0] *
                                       ((unsigned long long)gy + (unsigned long long)D.gdim[1] * (unsigned long long)gz);
        double c[7];
        ic_cell(P, bub, nb, D.h, gx, gy, gz, lin, c);
        for (int m = 0; m < 7; ++m) { U[m * fs + i] = (T)c[m]; R[m * fs + i] = (T)0; }
    }
}

cudaError_t launch_ic_cloud(int is_double, const DomDev* dom, int parity, const IcParams& P,
                            const double* bubbles, int nbubbles, cudaStream_t st)
{
    if (is_double) ic_cloud_kernel<double><<<148 * 16, 256, 0, st>>>(dom, parity, P, bubbles, nbubbles);
    else           ic_cloud_kernel<float><<<148 * 16, 256, 0, st>>>(dom, parity, P, bubbles, nbubbles);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Shock-induced cloud-collapse initial condition: the reference's
// Sim_SICCloudMPI case (Sim_SICCloudMPI.cpp:43-357, Sim_SICCloudMPI.h:27-301).
// A planar shock (Johnsen's post-shock state) ahead of a cloud of spheres;
// every cell holds the 3x3x3 Simpson average of the sampled mixture.  The
// arithmetic follows the reference's types: Real is the state's type, and
// the sub-expressions its double literals promote are evaluated in double
// (this translation unit contracts no multiply-adds, so the FP32 fields are
// bit-identical to the reference built with _FLOAT_PRECISION_).
// ---------------------------------------------------------------------------
template <class Real>
struct SicState
{
    Real rho0, u0, p0, rhoB, uB, pB, psi;
    Real n[3], S[3];
    Real g1, g2, pc1, pc2;
    Real rho1, u1, p1, mach;
};

// Host: parameters to Real, shock normal normalised, post-shock state
// (Sim_SICCloudMPI.cpp:76-103; pow(Real, int) promotes to double).
template <class Real>
SicState<Real> sic_setup(const SicParams& P)
{
    SicState<Real> st;
    st.rho0 = (Real)P.rho0; st.u0 = (Real)P.u0; st.p0 = (Real)P.p0;
    st.rhoB = (Real)P.rhoB; st.uB = (Real)P.uB; st.pB = (Real)P.pB;
    st.psi = (Real)P.pressure_ratio;
    for (int i = 0; i < 3; ++i) { st.n[i] = (Real)P.shock_n[i]; st.S[i] = (Real)P.shock_s[i]; }
    st.g1 = (Real)P.g1; st.g2 = (Real)P.g2; st.pc1 = (Real)P.pc1; st.pc2 = (Real)P.pc2;
    const Real mag = (Real)std::sqrt((double)st.n[0] * (double)st.n[0] + (double)st.n[1] * (double)st.n[1]
                                     + (double)st.n[2] * (double)st.n[2]);
    for (int i = 0; i < 3; ++i) st.n[i] /= mag;
    const Real gamma = st.g1, pc = st.pc1, p0 = st.p0, rho0 = st.rho0, u0 = st.u0, psi = st.psi;
    const Real p1   = p0 * psi;
    const Real tmp1 = (Real)(((double)gamma + 1.0) / ((double)gamma - 1.0));
    const Real tmp2 = (p1 + pc) / (p0 + pc);
    const Real c0   = std::sqrt(gamma * (p0 + pc) / rho0);           // sqrt of Real
    const Real mach = (Real)std::sqrt(((double)gamma + 1.0) / (2.0 * (double)gamma) * ((double)psi - 1.0) * (double)p0
                                      / (double)(p0 + pc) + 1.0);
    st.mach = mach;
    st.u1   = (Real)((double)u0 + (double)c0 * ((double)psi - 1.0) * (double)p0 / (double)(gamma * (p0 + pc) * mach));
    st.rho1 = (Real)((double)rho0 * ((double)(tmp1 * tmp2) + 1.0) / (double)(tmp1 + tmp2));
    st.p1   = p1;
    return st;
}

void sic_post_shock(int is_double, const SicParams& P, double post4[4])
{
    if (is_double)
    {
        const SicState<double> st = sic_setup<double>(P);
        post4[0] = st.rho1; post4[1] = st.u1; post4[2] = st.p1; post4[3] = st.mach;
    }
    else
    {
        const SicState<float> st = sic_setup<float>(P);
        post4[0] = st.rho1; post4[1] = st.u1; post4[2] = st.p1; post4[3] = st.mach;
    }
}

// |pos - c| - r: differences in Real, squares and sum in double
// (Sim_SICCloudMPI.h:97-101)
template <class Real>
__device__ __forceinline__ Real sic_shape_eval(const Real* shp, const Real pos[3])
{
    const double dx = (double)(pos[0] - shp[0]), dy = (double)(pos[1] - shp[1]), dz = (double)(pos[2] - shp[2]);
    return (Real)(sqrt(dx * dx + dy * dy + dz * dz) - (double)shp[3]);
}

// Cloud indicator: cosine ramp of half-width eps around the nearest sphere
// surface; eps = 0 gives 1 inside or on a sphere, 0 outside
// (Sim_SICCloudMPI.h:285-301, min/max with the comparisons of std::min/max).
template <class Real>
__device__ __forceinline__ Real sic_indicator(const Real* shp, int n, const Real pos[3], double eps)
{
    Real d = (Real)HUGE_VAL;
    for (int i = 0; i < n; ++i)
    {
        const Real nd = sic_shape_eval<Real>(shp + 4 * i, pos);
        d = (nd < d) ? nd : d;
    }
    const double x  = ((double)d + eps) / (2 * eps);
    const double mx = (0. < x) ? x : 0.;
    const double mn = (mx < 1.) ? mx : 1.;
    return (Real)(0.5 + 0.5 * cos(3.14159265358979323846 * mn));
}

// Mixture of one sample (Sim_SICCloudMPI.cpp:247-276)
template <class Real>
__device__ __forceinline__ void sic_mix(const SicState<Real>& st, const Real shock, const Real bubble, Real out[7])
{
    const Real G1 = st.g1 - 1, G2 = st.g2 - 1;
    const Real F1 = st.g1 * st.pc1, F2 = st.g2 * st.pc2;
    const Real rho = shock * st.rho1 + (1 - shock) * (st.rhoB * bubble + st.rho0 * (1 - bubble));
    const Real u   = (shock * st.u1 + (1 - shock) * (st.uB * bubble + st.u0 * (1 - bubble))) * rho;
    const Real v = 0, w = 0;
    const Real G = (Real)(1. / (double)G1 * (double)(1 - bubble) + 1. / (double)G2 * (double)bubble);
    const Real P = F1 / G1 * (1 - bubble) + F2 / G2 * bubble;
    const Real pressure = shock * st.p1 + (1 - shock) * (st.pB * bubble + st.p0 * (1 - bubble));
    const Real ke = (Real)(0.5 * (double)(u * u + v * v + w * w) / (double)rho);
    out[0] = rho; out[1] = u; out[2] = v; out[3] = w;
    out[4] = pressure * G + P + ke;
    out[5] = G; out[6] = P;
}

constexpr int kSicMaxShapes = 1024;   // shapes of one tile kept in shared memory

// One thread per cell of an 8x8x4 tile.  The tile first gathers the shapes
// within reach of its samples (centre within radius + eps + h of the tile's
// sample box): any other shape lies farther than eps + h from every sample,
// so it is neither inside nor within the ramp and cannot change the
// indicator.  More than kSicMaxShapes shapes in reach: every shape is used.
template <class Real>
__global__ void __launch_bounds__(256) sic_cloud_kernel(const DomDev* dom, int parity, const SicState<Real> st,
                                                        const double* __restrict__ shapes, int nshapes, double eps)
{
    __shared__ Real sh[4 * kSicMaxShapes];
    __shared__ int cnt;
    const DomDev& D = *dom;
    const double hd = D.h;
    const int ix = blockIdx.x * 8 + (threadIdx.x & 7);
    const int iy = blockIdx.y * 8 + ((threadIdx.x >> 3) & 7);
    const int iz = blockIdx.z * 4 + (threadIdx.x >> 6);
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    // the tile's sample box in global coordinates
    const double lo[3] = {hd * (D.org[0] + blockIdx.x * 8), hd * (D.org[1] + blockIdx.y * 8), hd * (D.org[2] + blockIdx.z * 4)};
    const double hi[3] = {hd * (D.org[0] + blockIdx.x * 8 + 8), hd * (D.org[1] + blockIdx.y * 8 + 8), hd * (D.org[2] + blockIdx.z * 4 + 4)};
    for (int i = threadIdx.x; i < nshapes; i += blockDim.x)
    {
        const double* c = shapes + 4 * (size_t)i;
        const double reach = c[3] + eps + hd;
        bool hit = true;
        for (int d = 0; d < 3; ++d) hit = hit && (c[d] >= lo[d] - reach) && (c[d] <= hi[d] + reach);
        if (hit)
        {
            const int k = atomicAdd(&cnt, 1);
            if (k < kSicMaxShapes)
                for (int j = 0; j < 4; ++j) sh[4 * k + j] = (Real)c[j];
        }
    }
    __syncthreads();
    if (ix >= D.nx || iy >= D.ny || iz >= D.nz) return;
    const int nc = cnt;
    const bool overflow = nc > kSicMaxShapes;   // then every shape, converted per use
    Real all[4];

    const Real h  = (Real)hd / 2;          // sample spacing: half the grid spacing
    const double p[3] = {hd * (D.org[0] + ix + 0.5), hd * (D.org[1] + iy + 0.5), hd * (D.org[2] + iz + 0.5)};
    const Real x0[3] = {(Real)(p[0] - (double)h), (Real)(p[1] - (double)h), (Real)(p[2] - (double)h)};
    const Real w6 = (Real)(1 / 6.), w23 = (Real)(2. / 3);
    Real acc[7];
    for (int jx = 0; jx < 3; ++jx)
    {
        Real yacc[7];
        for (int jy = 0; jy < 3; ++jy)
        {
            Real zs[3][7];
            for (int jz = 0; jz < 3; ++jz)
            {
                const Real pos[3] = {x0[0] + (Real)jx * h, x0[1] + (Real)jy * h, x0[2] + (Real)jz * h};
                const Real sd = -(st.n[0] * (st.S[0] - pos[0]) + st.n[1] * (st.S[1] - pos[1]) + st.n[2] * (st.S[2] - pos[2]));
                const Real shock = sd > 0 ? (Real)0 : (Real)1;
                Real bubble = 0;
                if (nshapes > 0)
                {
                    if (!overflow) bubble = sic_indicator<Real>(sh, nc, pos, eps);
                    else
                    {
                        Real d = (Real)HUGE_VAL;
                        for (int i = 0; i < nshapes; ++i)
                        {
                            for (int j = 0; j < 4; ++j) all[j] = (Real)shapes[4 * (size_t)i + j];
                            const Real nd = sic_shape_eval<Real>(all, pos);
                            d = (nd < d) ? nd : d;
                        }
                        const double x  = ((double)d + eps) / (2 * eps);
                        const double mx = (0. < x) ? x : 0.;
                        const double mn = (mx < 1.) ? mx : 1.;
                        bubble = (Real)(0.5 + 0.5 * cos(3.14159265358979323846 * mn));
                    }
                }
                sic_mix<Real>(st, shock, bubble, zs[jz]);
            }
            // z integral of this (x, y) column, then accumulated in y
            Real zi[7];
            for (int m = 0; m < 7; ++m) zi[m] = (w6 * zs[0][m] + w23 * zs[1][m]) + w6 * zs[2][m];
            for (int m = 0; m < 7; ++m)
                yacc[m] = jy == 0 ? w6 * zi[m] : (jy == 1 ? yacc[m] + w23 * zi[m] : yacc[m] + w6 * zi[m]);
        }
        for (int m = 0; m < 7; ++m)
            acc[m] = jx == 0 ? w6 * yacc[m] : (jx == 1 ? acc[m] + w23 * yacc[m] : acc[m] + w6 * yacc[m]);
    }
    Real* U = (Real*)D.U[parity];
    Real* R = (Real*)D.R;
    const long long c = ix + (long long)D.nx * (iy + (long long)D.ny * iz);
    for (int m = 0; m < 7; ++m) { U[m * D.fs + c] = acc[m]; R[m * D.fs + c] = (Real)0; }
}

cudaError_t launch_sic_cloud(int is_double, const DomDev* dom, int nx, int ny, int nz, int parity,
                             const SicParams& P, const double* shapes, int nshapes, cudaStream_t st)
{
    const dim3 grid((nx + 7) / 8, (ny + 7) / 8, (nz + 3) / 4);
    if (is_double) sic_cloud_kernel<double><<<grid, 256, 0, st>>>(dom, parity, sic_setup<double>(P), shapes, nshapes, P.eps);
    else           sic_cloud_kernel<float><<<grid, 256, 0, st>>>(dom, parity, sic_setup<float>(P), shapes, nshapes, P.eps);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The reference's other case set-ups: SteadyState (Sim_SteadyStateMPI.cpp:
// 95-135), Sod (Sim_SodMPI.cpp:20-95) and 2DSBI (Sim_2DSBIMPI.cpp:83-233).
// Each evaluates in double where the reference's options are doubles and in
// the state's type where it stores to Real; the register is cleared.
// ---------------------------------------------------------------------------
template <class T>
__global__ void fill_state_kernel(const DomDev* dom, int parity, const T v0, const T v1, const T v2, const T v3,
                                  const T v4, const T v5, const T v6)
{
    const DomDev& D = *dom;
    T* U = (T*)D.U[parity];
    T* R = (T*)D.R;
    const long long n = (long long)D.nx * D.ny * D.nz;
    const T v[7] = {v0, v1, v2, v3, v4, v5, v6};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        for (int m = 0; m < 7; ++m) { U[m * D.fs + i] = v[m]; R[m * D.fs + i] = (T)0; }
}

cudaError_t launch_ic_steady(int is_double, const DomDev* dom, int parity, const SteadyParams& P, cudaStream_t st)
{
    // the uniform state in double (Sim_SteadyStateMPI.cpp:111-117)
    const double ru = P.rho * P.u, rv = P.rho * P.v, rw = P.rho * P.w;
    const double G  = 1.0 / (P.g - 1.0);
    const double Pc = P.g * P.pc * G;
    const double e  = G * P.p + Pc + 0.5 * P.rho * (P.u * P.u + P.v * P.v + P.w * P.w);
    if (is_double) fill_state_kernel<double><<<148 * 8, 256, 0, st>>>(dom, parity, P.rho, ru, rv, rw, e, G, Pc);
    else           fill_state_kernel<float><<<148 * 8, 256, 0, st>>>(dom, parity, (float)P.rho, (float)ru, (float)rv,
                                                                       (float)rw, (float)e, (float)G, (float)Pc);
    return cudaGetLastError();
}

template <class T>
__global__ void sod_kernel(const DomDev* dom, int parity, const SodParams P)
{
    const DomDev& D = *dom;
    T* U = (T*)D.U[parity];
    T* R = (T*)D.R;
    const long long n = (long long)D.nx * D.ny * D.nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const int idx[3] = {(int)(i % D.nx), (int)((i / D.nx) % D.ny), (int)(i / ((long long)D.nx * D.ny))};
        const double pos = D.h * (D.org[P.axis] + idx[P.axis] + 0.5);
        const bool x = P.reverse ? pos > P.x0 : pos < P.x0;
        const bool nx = !x;
        // the reference's boolean-weighted mixture (Sim_SodMPI.cpp:69-75)
        const double r = x * P.rho1 + nx * P.rho2;
        const double p = x * P.p1 + nx * P.p2;
        const double u = x * P.rho1 * P.u1 + nx * P.rho2 * P.u2;
        const double G = x * 1. / (P.g1 - 1.) + nx * 1. / (P.g2 - 1.);
        const double Pc = x * P.pc1 * P.g1 / (P.g1 - 1.) + nx * P.pc2 * P.g2 / (P.g2 - 1.);
        const T v[7] = {(T)r, (T)(P.axis == 0 ? u : 0.), (T)(P.axis == 1 ? u : 0.), (T)(P.axis == 2 ? u : 0.),
                        (T)(G * p + Pc + 0.5 * u * u / r), (T)G, (T)Pc};
        for (int m = 0; m < 7; ++m) { U[m * D.fs + i] = v[m]; R[m * D.fs + i] = (T)0; }
    }
}

cudaError_t launch_ic_sod(int is_double, const DomDev* dom, int parity, const SodParams& P, cudaStream_t st)
{
    if (is_double) sod_kernel<double><<<148 * 8, 256, 0, st>>>(dom, parity, P);
    else           sod_kernel<float><<<148 * 8, 256, 0, st>>>(dom, parity, P);
    return cudaGetLastError();
}

// 2DSBI: post-shock state of the planar shock in Real (SimTools::
// getPostShockRatio, with pow of Real), mixture constants in double.
template <class Real>
struct SbiState
{
    double rho1, u1, p1;            // post-shock state (from Real)
    double G1, G2, F1, F2, eps;     // mixture constants, SimTools::EPSILON
};

template <class Real>
static SbiState<Real> sbi_setup(const SbiParams& P, double h)
{
    const Real pre[3] = {(Real)P.rho, (Real)P.u, (Real)P.p};
    const Real mach = (Real)P.mach, gamma = (Real)P.g1, pc = (Real)P.pc1;
    Real post[3];
    const Real m2 = std::pow(mach, (Real)2.);
    const double mpost = std::sqrt((m2 * (gamma - 1.) + 2.) / (2. * gamma * m2 - (gamma - 1.)));
    post[0] = (gamma + 1.) * m2 / ((gamma - 1.) * m2 + 2.) * pre[0];
    post[2] = 1. / (gamma + 1.) * (2. * gamma * m2 - (gamma - 1.)) * pre[2];
    const double u_pre  = mach * std::sqrt(gamma * (pc + pre[2]) / pre[0]);
    const double u_post = mpost * std::sqrt(gamma * (pc + post[2]) / post[0]);
    post[1] = u_pre - u_post;
    SbiState<Real> S;
    S.rho1 = post[0]; S.u1 = post[1]; S.p1 = post[2];
    S.G1 = P.g1 - 1; S.G2 = P.g2 - 1; S.F1 = P.g1 * P.pc1; S.F2 = P.g2 * P.pc2;
    S.eps = (double)(Real)P.mollfactor * std::sqrt(3.) * h;
    return S;
}

template <class Real>
__device__ __forceinline__ void sbi_cell(const DomDev& D, const SbiParams& P, const SbiState<Real>& S,
                                         const double* __restrict__ bub, int nb, const int idx[3], Real v[7])
{
    const double p[3] = {D.h * (idx[0] + 0.5), D.h * (idx[1] + 0.5), D.h * (idx[2] + 0.5)};
    const int a0 = P.axis0, a1 = P.axis1;
    const Real shock = (Real)(p[a0] - P.x0) > 0 ? (Real)0 : (Real)1;
    Real bubble = 0;
    for (int i = 0; i < nb; ++i)
    {
        const double dx = p[a0] - (double)(Real)bub[4 * i + a0], dy = p[a1] - (double)(Real)bub[4 * i + a1];
        const Real r = (Real)sqrt(dx * dx + dy * dy);
        const Real phi = r - (Real)bub[4 * i + 3];
        // SimTools::heaviside_smooth: cosine ramp of half-width EPSILON
        const double x  = 0.5 * ((double)phi + S.eps) / S.eps;
        const double mx = (0. < x) ? x : 0.;
        const double mn = (mx < 1.) ? mx : 1.;
        const Real alpha = (Real)(3.14159265358979323846 * mn);
        bubble = (Real)(0.5 + 0.5 * (double)cos(alpha));
        if (bubble > 0) break;
    }
    const double b = (double)bubble, s = (double)shock;
    const Real rho = (Real)(s * S.rho1 + (double)(1 - shock) * (P.rhobubble * b + P.rho * (double)(1 - bubble)));
    const Real mom = (Real)((s * S.u1 + (double)(1 - shock) * P.u) * (double)rho);
    const Real G = (Real)(1. / S.G1 * (double)(1 - bubble) + 1. / S.G2 * b);
    const Real Pc = (Real)(S.F1 / S.G1 * (double)(1 - bubble) + S.F2 / S.G2 * b);
    const Real pressure = (Real)(s * S.p1 + (double)(1 - shock) * (P.pbubble * b + P.p * (double)(1 - bubble)));
    const double m = (double)mom;
    const Real ke = (Real)(0.5 * (m * m + 0. + 0.) / (double)rho);
    v[0] = rho;
    v[1] = a0 == 0 ? mom : (Real)0;
    v[2] = a0 == 1 ? mom : (Real)0;
    v[3] = a0 == 2 ? mom : (Real)0;
    v[4] = pressure * G + Pc + ke;
    v[5] = G;
    v[6] = Pc;
}

// With `reverse`, every cell takes the state of its mirror image through the
// domain centre (all three axes) with the momentum negated, except the middle
// plane of an odd extent along the shock axis, which the reference's swap
// loop (Sim_2DSBIMPI.cpp:196-229) leaves as it is.
template <class Real>
__global__ void sbi_kernel(const DomDev* dom, int parity, const SbiParams P, const SbiState<Real> S,
                           const double* __restrict__ bub, int nb)
{
    const DomDev& D = *dom;
    Real* U = (Real*)D.U[parity];
    Real* R = (Real*)D.R;
    // global indices: the mirror is through the global domain's centre
    const int n3[3] = {D.gdim[0], D.gdim[1], D.gdim[2]};
    const long long n = (long long)D.nx * D.ny * D.nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        int idx[3] = {D.org[0] + (int)(i % D.nx), D.org[1] + (int)((i / D.nx) % D.ny),
                      D.org[2] + (int)(i / ((long long)D.nx * D.ny))};
        bool flip = false;
        if (P.reverse && !((n3[P.axis0] & 1) && idx[P.axis0] == n3[P.axis0] / 2))
        {
            for (int d = 0; d < 3; ++d) idx[d] = n3[d] - 1 - idx[d];
            flip = true;
        }
        Real v[7];
        sbi_cell<Real>(D, P, S, bub, nb, idx, v);
        if (flip) { v[1] = -v[1]; v[2] = -v[2]; v[3] = -v[3]; }
        for (int m = 0; m < 7; ++m) { U[m * D.fs + i] = v[m]; R[m * D.fs + i] = (Real)0; }
    }
}

cudaError_t launch_ic_sbi(int is_double, const DomDev* dom, int nx, int ny, int nz, int parity, const SbiParams& P,
                          const double* bubbles, int nbubbles, cudaStream_t st)
{
    const double h = 1.0 / (double)std::max(nx, std::max(ny, nz));
    if (is_double) sbi_kernel<double><<<148 * 8, 256, 0, st>>>(dom, parity, P, sbi_setup<double>(P, h), bubbles, nbubbles);
    else           sbi_kernel<float><<<148 * 8, 256, 0, st>>>(dom, parity, P, sbi_setup<float>(P, h), bubbles, nbubbles);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Output packing of the reference's dump and save (source/Types.h:192-277,
// source/IO/HDF5Dumper_MPI.h:104-121,243-253): cell (ix,iy,iz) of slabs
// [z0, z1) to out[NCH*(ix + nx*(iy + ny*(iz - z0))) + ch], channels
//   kind 0 (myTensorialStreamer): rho, u, v, w, p, G, P, 0, 0 with
//          p = (E - 0.5*(ru^2+rv^2+rw^2)/rho - P)/G, the 0.5 literal making
//          that part double (the momentum squares are summed in Real);
//   kind 1 (mySaveStreamer): the 7 conserved fields.
// unpack_save_kernel is the restart direction of kind 1.
// ---------------------------------------------------------------------------
template <class T, int KIND>
__global__ void pack_kernel(const DomDev* dom, int parity, int z0, int z1, T* __restrict__ out)
{
    const DomDev& D = *dom;
    const T* U = (const T*)D.U[parity];
    const long long plane = (long long)D.nx * D.ny;
    const long long n = plane * (z1 - z0);
    const long long base = plane * z0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const long long c = base + i;
        const T r = U[c], mu = U[D.fs + c], mv = U[2 * D.fs + c], mw = U[3 * D.fs + c];
        const T e = U[4 * D.fs + c], G = U[5 * D.fs + c], P = U[6 * D.fs + c];
        if (KIND == 0)
        {
            T* o = out + 9 * i;
            o[0] = r;
            o[1] = mu / r;
            o[2] = mv / r;
            o[3] = mw / r;
            o[4] = (T)(((double)e - 0.5 * (double)(mu * mu + mv * mv + mw * mw) / (double)r - (double)P) / (double)G);
            o[5] = G;
            o[6] = P;
            o[7] = (T)0;
            o[8] = (T)0;
        }
        else
        {
            T* o = out + 7 * i;
            o[0] = r; o[1] = mu; o[2] = mv; o[3] = mw; o[4] = e; o[5] = G; o[6] = P;
        }
    }
}

template <class T>
__global__ void unpack_save_kernel(const DomDev* dom, int parity, int z0, int z1, const T* __restrict__ in)
{
    const DomDev& D = *dom;
    T* U = (T*)D.U[parity];
    T* R = (T*)D.R;
    const long long plane = (long long)D.nx * D.ny;
    const long long n = plane * (z1 - z0);
    const long long base = plane * z0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const long long c = base + i;
        for (int m = 0; m < 7; ++m) { U[m * D.fs + c] = in[7 * i + m]; R[m * D.fs + c] = (T)0; }
    }
}

cudaError_t launch_pack(int is_double, int kind, const DomDev* dom, int parity, int z0, int z1, void* out, cudaStream_t st)
{
    const int grid = 148 * 8;
    if (is_double)
    {
        if (kind == 0) pack_kernel<double, 0><<<grid, 256, 0, st>>>(dom, parity, z0, z1, (double*)out);
        else           pack_kernel<double, 1><<<grid, 256, 0, st>>>(dom, parity, z0, z1, (double*)out);
    }
    else
    {
        if (kind == 0) pack_kernel<float, 0><<<grid, 256, 0, st>>>(dom, parity, z0, z1, (float*)out);
        else           pack_kernel<float, 1><<<grid, 256, 0, st>>>(dom, parity, z0, z1, (float*)out);
    }
    return cudaGetLastError();
}

cudaError_t launch_unpack_save(int is_double, const DomDev* dom, int parity, int z0, int z1, const void* in, cudaStream_t st)
{
    const int grid = 148 * 8;
    if (is_double) unpack_save_kernel<double><<<grid, 256, 0, st>>>(dom, parity, z0, z1, (const double*)in);
    else           unpack_save_kernel<float><<<grid, 256, 0, st>>>(dom, parity, z0, z1, (const float*)in);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Explicit ghost buffers in the reference layouts, from the same boundary
// map the stage kernel applies on the fly:
//   gx[side][q][GHOSTMAPX(ix,iy,iz)]  = ix + 3*(iy + NY*iz),     ix 0..2
//   gy[side][q][GHOSTMAPY(ix,iy,iz)]  = ix + NX*(iy + 3*iz),     iy 0..2
//   gz[side][q][ID3(ix,iy,iz,NX,NY)],                             iz 0..2
// left side: layer 0 = outermost cell (-3); right side: layer 0 = cell N
// (Types.h:42-43, BoundaryConditions.h:60-109, GPUlab.h:69-91).
// ---------------------------------------------------------------------------
template <class T>
__global__ void fill_ghosts_kernel(const DomDev* dom, int parity, T* gx, T* gy, T* gz)
{
    const DomDev& DD = *dom;
    DomRegs D;
    D.nx = DD.nx; D.ny = DD.ny; D.nz = DD.nz;
    D.bc0 = DD.bc[0]; D.bc1 = DD.bc[1]; D.bc2 = DD.bc[2];
    D.bc3 = DD.bc[3]; D.bc4 = DD.bc[4]; D.bc5 = DD.bc[5];
    D.fs = DD.fs;
    const T* U = (const T*)DD.U[parity];
    const long long sx = 3LL * D.ny * D.nz, sy = 3LL * D.nx * D.nz, sz = 3LL * D.nx * D.ny;
    const long long total = 2 * (sx + sy + sz);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
    {
        int ix, iy, iz, dir, side;
        long long o = i, li;
        if (o < 2 * sx)          { dir = 0; side = (int)(o / sx); li = o % sx; ix = (int)(li % 3); iy = (int)((li / 3) % D.ny); iz = (int)(li / (3LL * D.ny)); }
        else if ((o -= 2 * sx) < 2 * sy) { dir = 1; side = (int)(o / sy); li = o % sy; ix = (int)(li % D.nx); iy = (int)((li / D.nx) % 3); iz = (int)(li / (3LL * D.nx)); }
        else { o -= 2 * sy; dir = 2; side = (int)(o / sz); li = o % sz; ix = (int)(li % D.nx); iy = (int)((li / D.nx) % D.ny); iz = (int)(li / ((long long)D.nx * D.ny)); }
        // ghost layer -> cell coordinate outside the domain
        int cx = ix, cy = iy, cz = iz;
        if (dir == 0) cx = side == 0 ? ix - 3 : D.nx + ix;
        if (dir == 1) cy = side == 0 ? iy - 3 : D.ny + iy;
        if (dir == 2) cz = side == 0 ? iz - 3 : D.nz + iz;
        bool fx, fy, fz;
        const int mx = bc_map(cx, D.nx, D.bc0, D.bc1, fx);
        const int my = bc_map(cy, D.ny, D.bc2, D.bc3, fy);
        // a halo face's ghost planes are stored state
        const bool zhalo = (cz < 0 && D.bc4 == BC_HALO) || (cz >= D.nz && D.bc5 == BC_HALO);
        const int mz = zhalo ? cz : bc_map(cz, D.nz, D.bc4, D.bc5, fz);
        if (zhalo) fz = false;
        const long long idx = (long long)mx + (long long)D.nx * ((long long)my + (long long)D.ny * mz);
        T* dst = dir == 0 ? gx : (dir == 1 ? gy : gz);
        const long long s = dir == 0 ? sx : (dir == 1 ? sy : sz);
        for (int q = 0; q < 7; ++q)
        {
            T v = U[q * D.fs + idx];
            if ((q == 1 && fx) || (q == 2 && fy) || (q == 3 && fz)) v = -v;
            dst[(side * 7 + q) * s + li] = v;
        }
    }
}

cudaError_t launch_fill_ghosts(int is_double, const DomDev* dom, int parity,
                               void* gx, void* gy, void* gz, cudaStream_t st)
{
    if (is_double) fill_ghosts_kernel<double><<<148 * 4, 256, 0, st>>>(dom, parity, (double*)gx, (double*)gy, (double*)gz);
    else           fill_ghosts_kernel<float><<<148 * 4, 256, 0, st>>>(dom, parity, (float*)gx, (float*)gy, (float*)gz);
    return cudaGetLastError();
}

// Ghost planes of linked slabs (GPUlab::load_ghosts of a rank between two
// neighbours, GPUlab.cpp:622-644, as device-to-device copies): for link l
// (lower, upper) and field q, direction 0 fills the 3 planes above the lower
// slab with planes 0..2 of the upper slab, direction 1 the 3 planes below
// the upper slab with planes nz-3..nz-1 of the lower one.  Each block row
// (blockIdx.y = 14 l + 7 direction + q) copies one contiguous 3-plane block.
template <class E>
__global__ void halo_kernel(const DomDev* doms, const int* links, int parity)
{
    const int l = blockIdx.y / 14, r = blockIdx.y % 14, dir = r / 7, q = r % 7;
    const DomDev& Lo = doms[links[2 * l]];
    const DomDev& Hi = doms[links[2 * l + 1]];
    const long long plane = (long long)Lo.nx * Lo.ny;
    const long long n = kHaloPlanes * plane;
    const E* src;
    E* dst;
    if (dir == 0) { dst = (E*)Lo.U[parity] + q * Lo.fs + Lo.nz * plane;          src = (const E*)Hi.U[parity] + q * Hi.fs; }
    else          { dst = (E*)Hi.U[parity] + q * Hi.fs - kHaloPlanes * plane;   src = (const E*)Lo.U[parity] + q * Lo.fs + (Lo.nz - kHaloPlanes) * plane; }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

cudaError_t launch_halo(int esz, const DomDev* doms, const int* links, int nlinks, long long max_plane,
                        int parity, cudaStream_t st)
{
    if (nlinks <= 0) return cudaSuccess;
    const long long n = kHaloPlanes * max_plane;
    const dim3 grid((unsigned)std::min<long long>((n + 255) / 256, 64), (unsigned)(14 * nlinks));
    if (esz == 8) halo_kernel<unsigned long long><<<grid, 256, 0, st>>>(doms, links, parity);
    else          halo_kernel<unsigned><<<grid, 256, 0, st>>>(doms, links, parity);
    return cudaGetLastError();
}

// Ghost planes of one slot of a windowed run (mpcf_run_window): the slot
// holds nz planes of a z-chunk of a larger domain at dst (plane 0), with 3
// stored ghost planes on each side.  Block row blockIdx.y = 7 side + q fills
// field q's 3 planes below (side 0) or above (side 1) the slot: from the top 3
// planes of the slot below (lo) or the bottom 3 of the slot above (hi), or,
// at the domain's own z faces (lo / hi null), by its boundary condition as
// the stage kernel's own mapping gives it (BoundaryConditions.h:60-109):
// absorbing repeats the face plane, reflecting mirrors the planes and negates
// the normal momentum (a flip of the sign bit, as the negation in the
// kernel's load).  The copies move bit patterns.
template <class E>
__global__ void window_ghosts_kernel(E* dst, const E* lo, const E* hi, long long fs, long long plane, int nz,
                                     int bc_lo, int bc_hi)
{
    const int side = blockIdx.y / 7, q = blockIdx.y % 7;
    const E sign = (E)1 << (sizeof(E) * 8 - 1);
    const long long n = kHaloPlanes * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const int g = (int)(i / plane) + 1;            // planes away from the slot's own planes, 1..3
        const long long xy = i - (long long)(g - 1) * plane;
        const E* src;
        long long sp, dp;
        bool flip = false;
        if (side == 0)
        {
            dp = -(long long)g;
            if (lo) { src = lo; sp = nz - g; }
            else    { src = dst; const bool refl = bc_lo == BC_REFLECTING; sp = refl ? g - 1 : 0; flip = refl && q == 3; }
        }
        else
        {
            dp = nz - 1 + g;
            if (hi) { src = hi; sp = g - 1; }
            else    { src = dst; const bool refl = bc_hi == BC_REFLECTING; sp = refl ? nz - g : nz - 1; flip = refl && q == 3; }
        }
        const E v = src[q * fs + sp * plane + xy];
        dst[q * fs + dp * plane + xy] = flip ? (v ^ sign) : v;
    }
}

cudaError_t launch_window_ghosts(int esz, void* dst, const void* lo, const void* hi, long long fs, long long plane,
                                 int nz, int bc_lo, int bc_hi, cudaStream_t st)
{
    const long long n = kHaloPlanes * plane;
    const dim3 grid((unsigned)std::min<long long>((n + 255) / 256, 64), 14u);
    if (esz == 8)
        window_ghosts_kernel<unsigned long long><<<grid, 256, 0, st>>>((unsigned long long*)dst, (const unsigned long long*)lo,
                                                                        (const unsigned long long*)hi, fs, plane, nz, bc_lo, bc_hi);
    else
        window_ghosts_kernel<unsigned><<<grid, 256, 0, st>>>((unsigned*)dst, (const unsigned*)lo, (const unsigned*)hi,
                                                             fs, plane, nz, bc_lo, bc_hi);
    return cudaGetLastError();
}

__global__ void zero_kernel(unsigned* p, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = 0u;
}

cudaError_t launch_zero(void* p, size_t bytes, cudaStream_t st)
{
    const size_t n = bytes / 4;
    const int g = (int)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
    zero_kernel<<<g > 0 ? g : 1, 256, 0, st>>>((unsigned*)p, n);
    return cudaGetLastError();
}

// FP64 sums of (rho, rho u, rho v, rho w, E) of the current state: one block
// per chunk (same chunking as the sound-speed reduction) writes its partials,
// then the per-domain totals are summed in chunk order.  Fixed block size and
// fixed reduction trees make the result independent of scheduling.
template <class T>
__global__ void __launch_bounds__(256) sum_state_kernel(const DomDev* doms, int ndom, int parity, int chunk, double* partial)
{
    __shared__ double red[5][256];
    const int c = blockIdx.x;
    int d = 0;
    while (d + 1 < ndom && doms[d + 1].sos_chunk_begin <= c) ++d;
    const DomDev& D = doms[d];
    const long long N = (long long)D.nx * D.ny * D.nz;
    const long long beg = (long long)(c - D.sos_chunk_begin) * chunk;
    const long long end = min(beg + (long long)chunk, N);
    const T* U = (const T*)D.U[parity];
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long i = beg + threadIdx.x; i < end; i += 256)
        for (int m = 0; m < 5; ++m) acc[m] += (double)U[m * D.fs + i];
    for (int m = 0; m < 5; ++m) red[m][threadIdx.x] = acc[m];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if ((int)threadIdx.x < w)
            for (int m = 0; m < 5; ++m) red[m][threadIdx.x] += red[m][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 5) partial[(long long)c * 5 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void sum_chunks_kernel(const DomDev* doms, const double* partial, double* out)
{
    const int d = blockIdx.x;
    const int m = threadIdx.x;
    if (m >= 5) return;
    double s = 0;
    for (int c = 0; c < doms[d].sos_chunks; ++c) s += partial[(long long)(doms[d].sos_chunk_begin + c) * 5 + m];
    out[d * 5 + m] = s;
}

cudaError_t launch_sum_state(const DomDev* doms, int ndom, int parity, int nchunks, int chunk, int is_double,
                             double* chunk_sums, double* out, cudaStream_t st)
{
    if (is_double) sum_state_kernel<double><<<nchunks, 256, 0, st>>>(doms, ndom, parity, chunk, chunk_sums);
    else           sum_state_kernel<float><<<nchunks, 256, 0, st>>>(doms, ndom, parity, chunk, chunk_sums);
    sum_chunks_kernel<<<ndom, 32, 0, st>>>(doms, chunk_sums, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP32 pipe probe: independent FMA chains, 8 per thread, enough warps to
// saturate every SM.  Used to measure the CUDA-core FP32 peak that bounds
// the stage kernel (no such figure is provided by the platform).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float seed)
{
    float a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i)
    {
#pragma unroll
        for (int k = 0; k < 16; ++k)
        {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.678f) out[0] = r;   // keeps the chains alive
}

cudaError_t launch_fma_probe(int blocks, int iters, float* out, cudaStream_t st)
{
    fma_probe_kernel<<<blocks, 256, 0, st>>>(out, iters, 1.0f);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// State update alone, U_next = b*R + U (the reference's _update,
// GPUkernels.cu:1142-1179), for callers that run Convection and Update as
// two separate steps (Convection_CUDA / Update_CUDA).  The fused stage
// kernel does the same arithmetic inline.
// ---------------------------------------------------------------------------
template <class T>
__global__ void update_kernel(const DomDev* doms, int ndom, int parity, T b)
{
    for (int d = 0; d < ndom; ++d)
    {
        const DomDev& D = doms[d];
        const long long N = (long long)D.nx * D.ny * D.nz;
        const T* U = (const T*)D.U[parity];
        T* Un = (T*)D.U[parity ^ 1];
        const T* R = (const T*)D.R;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
            for (int m = 0; m < 7; ++m)
                Un[m * D.fs + i] = b * R[m * D.fs + i] + U[m * D.fs + i];
    }
}

cudaError_t launch_update(int is_double, const DomDev* doms, int ndom, int parity, double b, cudaStream_t st)
{
    if (is_double) update_kernel<double><<<148 * 8, 256, 0, st>>>(doms, ndom, parity, b);
    else           update_kernel<float><<<148 * 8, 256, 0, st>>>(doms, ndom, parity, (float)b);
    return cudaGetLastError();
}

// ===========================================================================
// Conservation sums without allocating (mpcf_conserved_sums_noalloc).
//
// For callers that may not allocate device memory themselves or through a
// library: hosts that give a plug-in a fixed device-memory budget at start-up
// and forbid cudaMalloc afterwards, and tight loops where cudaMalloc/cudaFree
// (which can synchronise the whole device) are not acceptable.  The caller
// passes its own device field pointers and an output; the per-chunk partials
// live in a fixed array of this library instead of solver-owned memory.
// ===========================================================================
namespace {

// cells per chunk and chunk limit: inputs up to 8192 * 32768 = 2^28 cells
constexpr int kNoAllocChunk = 32768;
constexpr int kNoAllocMaxChunks = 8192;

// per-chunk partials [chunk][5], then 5 totals; every device that loads the
// library keeps this ~320 KB array until the process exits
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxChunks * 5 + 8];

// device address of g_noalloc_scratch per device, looked up on the first call
// made with that device current (the name is only a host-side handle)
constexpr int kMaxDevices = 64;
void* g_noalloc_addr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;

template <class T>
__global__ void __launch_bounds__(256) sum_fields_kernel(const T* __restrict__ f0, const T* __restrict__ f1,
        const T* __restrict__ f2, const T* __restrict__ f3, const T* __restrict__ f4,
        long long n, int chunk, double* partial)
{
    // same chunking, accumulation and reduction tree as sum_state_kernel, so
    // the result is bit-identical to the solver's mpcf_conserved_sums
    __shared__ double red[5][256];
    const long long beg = (long long)blockIdx.x * chunk;
    const long long end = min(beg + (long long)chunk, n);
    const T* f[5] = {f0, f1, f2, f3, f4};
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long i = beg + threadIdx.x; i < end; i += 256)
        for (int m = 0; m < 5; ++m) acc[m] += (double)f[m][i];
    for (int m = 0; m < 5; ++m) red[m][threadIdx.x] = acc[m];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if ((int)threadIdx.x < w)
            for (int m = 0; m < 5; ++m) red[m][threadIdx.x] += red[m][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 5) partial[(long long)blockIdx.x * 5 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void sum_partials_kernel(const double* partial, int nchunks, double* out)
{
    const int m = threadIdx.x;
    if (m >= 5) return;
    double s = 0;
    for (int c = 0; c < nchunks; ++c) s += partial[(long long)c * 5 + m];
    out[m] = s;
}

} // namespace

} // namespace mpcf

#include "../../include/mpcf_b200.h"

extern "C" int mpcf_conserved_sums_noalloc(const void* const* state7, long long ncells, int elem_size,
                                           double* out5, int out_is_device, int device, void* stream)
{
    using namespace mpcf;
    if (!state7 || !out5) return mpcf_fail_external(MPCF_ERR_ARG, "null state or output pointer");
    if (elem_size != 4 && elem_size != 8) return mpcf_fail_external(MPCF_ERR_ARG, "elem_size must be 4 or 8");
    if (ncells < 1) return mpcf_fail_external(MPCF_ERR_ARG, "ncells must be positive");
    if (ncells > (long long)kNoAllocMaxChunks * kNoAllocChunk)
        return mpcf_fail_external(MPCF_ERR_ARG, "ncells = %lld exceeds the no-allocation limit of %lld cells "
                                  "(%d chunks of %d); use mpcf_conserved_sums", ncells,
                                  (long long)kNoAllocMaxChunks * kNoAllocChunk, kNoAllocMaxChunks, kNoAllocChunk);
    if (device < 0 || device >= kMaxDevices) return mpcf_fail_external(MPCF_ERR_ARG, "device %d out of range", device);
    for (int q = 0; q < 5; ++q)
        if (!state7[q]) return mpcf_fail_external(MPCF_ERR_ARG, "field %d pointer is null", q);

    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); prev = -1; }
    if (prev != device && cudaSetDevice(device) != cudaSuccess)
    { cudaGetLastError(); return mpcf_fail_external(MPCF_ERR_CUDA, "cannot make device %d current", device); }
    struct Restore { int p; int d; ~Restore() { if (p >= 0 && p != d) cudaSetDevice(p); } } restore{prev, device};

    // one-time set-up on this device: the device address of the scratch array
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[device])
        {
            void* addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || !addr)
            {
                cudaGetLastError();
                return mpcf_fail_external(MPCF_ERR_CUDA, "cudaGetSymbolAddress(no-allocation scratch) failed on device %d: %s",
                                          device, cudaGetErrorString(e));
            }
            g_noalloc_addr[device] = addr;
        }
        scratch = (double*)g_noalloc_addr[device];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int nchunks = (int)((ncells + kNoAllocChunk - 1) / kNoAllocChunk);
    double* totals = scratch + (size_t)kNoAllocMaxChunks * 5;
    // every partial slot the second kernel reads is written by the first, so
    // nothing left by an earlier call is read
    if (elem_size == 8)
        sum_fields_kernel<double><<<nchunks, 256, 0, st>>>((const double*)state7[0], (const double*)state7[1],
            (const double*)state7[2], (const double*)state7[3], (const double*)state7[4], ncells, kNoAllocChunk, scratch);
    else
        sum_fields_kernel<float><<<nchunks, 256, 0, st>>>((const float*)state7[0], (const float*)state7[1],
            (const float*)state7[2], (const float*)state7[3], (const float*)state7[4], ncells, kNoAllocChunk, scratch);
    sum_partials_kernel<<<1, 32, 0, st>>>(scratch, nchunks, out_is_device ? out5 : totals);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && !out_is_device)
    {
        e = cudaMemcpyAsync(out5, totals, 5 * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return mpcf_fail_external(MPCF_ERR_CUDA, "no-allocation sums: %s", cudaGetErrorString(e));
    return MPCF_OK;
}
