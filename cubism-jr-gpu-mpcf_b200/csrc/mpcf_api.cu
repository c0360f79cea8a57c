// mpcf_api.cu -- host runtime behind the C ABI of include/mpcf_b200.h.
//
// A solver owns, per domain, two state buffers (ping-pong) and the LSRK3
// register in HBM, plus per-domain device scalars (dt/h, dt, time, the
// sound-speed accumulator) and one CUDA stream.  Nothing is staged through
// the host between stages: the reference's chunked PCIe streaming
// (GPUlab.cpp:202-372,703-793) and its host-side halo fills
// (BoundaryConditions.h:60-109) are replaced by the fused stage kernel.
#include <cuda_runtime.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <functional>
#include <random>
#include <string>
#include <vector>
#include <limits>

#include "../../include/mpcf_b200.h"
#include "mpcf_types.h"
#include "mpcf_launch.h"
#include "mpcf_ic.h"

using namespace mpcf;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

} // namespace

// error recording for entry points defined in other translation units
int mpcf_fail_external(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

namespace {

#define CK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) \
    return fail(MPCF_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); } while (0)

// NVTX range over an entry point (header-only NVTX 3: no-ops unless a
// profiler is attached), so a timeline shows the host calls of the path.
struct Range
{
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};

struct DeviceGuard
{
    int prev = -1;
    explicit DeviceGuard(int dev) { cudaGetDevice(&prev); if (prev != dev) cudaSetDevice(dev); else prev = -1; }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

const double kLSRK3[3][2] = {{0.0, 1.0/4.0}, {-17.0/32.0, 8.0/9.0}, {-32.0/27.0, 3.0/4.0}};

} // namespace

struct mpcf_solver
{
    int device = 0;
    int pol = 0;
    int ndom = 0;
    size_t esz = 4;
    cudaStream_t stream = nullptr;
    int num_sms = 148;

    std::vector<DomDev> hdoms;
    DomDev* ddoms = nullptr;
    std::vector<void*> allocs;      // device allocations owned by the solver
    int parity = 0;

    // device scalars
    void* sos_bits = nullptr;       // ndom * esz
    void* dtinvh = nullptr;         // ndom * esz
    double* dt = nullptr;           // ndom
    double* time = nullptr;         // ndom
    unsigned* err = nullptr;        // 1
    unsigned* counter = nullptr;    // 1
    double* tile_sums = nullptr;    // ntiles * 5
    double* chunk_sums = nullptr;   // nchunks * 5
    double* sums = nullptr;         // ndom * 5
    double* bubbles = nullptr;      // scratch for IC
    int bubbles_cap = 0;
    void* host_stage = nullptr;     // pinned host scratch (ndom doubles/elems)

    void* tmaps = nullptr;          // ndom * 4 CUtensorMap (128 B each)

    // linked z-slabs (lower, upper) and their device copy
    std::vector<int> links;         // 2 per link
    int* dlinks = nullptr;
    long long link_plane = 0;       // largest nx*ny of a linked domain

    // launch configuration
    int ty = 7, dz = 64, persist = 0, tma = 0;
    int ntiles = 0;
    int sos_chunk = 32768, nchunks = 0;
    bool track_cons = false;
    bool sums_valid = false;
    // the sound-speed accumulator holds the maximum of the current state,
    // fused into the last stage of the previous step; any other change of
    // the state clears this and the next step runs the stand-alone reduction
    bool sos_fresh = false;

    // graphs of one step for the two parities
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    double graph_cfl = -1, graph_dtmax = -1;
    bool graph_cons = false;

    unsigned test_flags = 0;        // MPCF_TEST_* (failure-detection tests only)
    bool weno3 = false;             // the reference's compile-time WENO3 reconstruction

    // runs over host-resident state (mpcf_run_host): two copy streams and
    // per-chunk events, made on first use
    cudaStream_t up = nullptr, down = nullptr;
    std::vector<cudaEvent_t> ev_up, ev_st, ev_down;
    cudaEvent_t ev_start = nullptr;

    // windowed runs (mpcf_create_window / mpcf_run_window): the domains are
    // slots of win_nslices planes that z-chunks of a win_nz-plane domain
    // held in host memory pass through; win_bc: its z faces.  Per slot, the
    // events that free it for the next chunk (compute stream, download).
    int win_nz = 0, win_nslices = 0, win_nch = 0;
    int win_bc[2] = {0, 0};
    std::vector<cudaEvent_t> ev_free_c, ev_free_d;
};

namespace {

// Tile heights with stage-kernel instances: 3 and 7 rows (CTAs of 4 and 8
// warps: one warp per row plus the helper warp), 8 rows (8 warps, no
// helper), and 15 rows (16 warps) for the FP32 reference-rounding form.
// Threads of one stage CTA: a warp per row, plus the helper warp for
// heights 2^n - 1 (TileShape in mpcf_stage.cuh).
int stage_block_threads(int ty) { return ((ty + 1) & ty) == 0 ? 32 * (ty + 1) : 32 * ty; }

bool valid_ty(const mpcf_solver* s, int ty)
{
    if (ty == 3 || ty == 7 || ty == 8) return true;
    return ty == 15 && s->pol == 0;
}

StageKernelInfo stage_info(const mpcf_solver* s, int ty, bool persist, bool sums, bool tma)
{
    if (s->weno3) return s->pol == 0 ? stage_info_ref_w3(ty, persist, sums, tma) : stage_info_fp64_w3(ty, persist, sums, tma);
    switch (s->pol)
    {
        case 0: return stage_info_ref(ty, persist, sums, tma);
        case 1: return stage_info_fast32(ty, persist, sums, tma);
        case 2: return stage_info_mixed(ty, persist, sums, tma);
        case 4: return stage_info_fast64(ty, persist, sums, tma);
        default: return stage_info_fp64(ty, persist, sums, tma);
    }
}

cudaError_t launch_stage(const mpcf_solver* s, const StageArgs& A, int grid, cudaStream_t st)
{
    if (s->weno3)
        return s->pol == 0 ? launch_stage_ref_w3(s->ty, s->persist != 0, s->tma != 0, A, grid, st)
                           : launch_stage_fp64_w3(s->ty, s->persist != 0, s->tma != 0, A, grid, st);
    switch (s->pol)
    {
        case 0: return launch_stage_ref(s->ty, s->persist != 0, s->tma != 0, A, grid, st);
        case 1: return launch_stage_fast32(s->ty, s->persist != 0, s->tma != 0, A, grid, st);
        case 2: return launch_stage_mixed(s->ty, s->persist != 0, s->tma != 0, A, grid, st);
        case 4: return launch_stage_fast64(s->ty, s->persist != 0, s->tma != 0, A, grid, st);
        default: return launch_stage_fp64(s->ty, s->persist != 0, s->tma != 0, A, grid, st);
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library needed)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried)
    {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// Tensor maps of every domain for the current tile height: per state buffer a
// 40 x (ty+6) x 1 x 7 halo box and a 32 x ty x 1 x 7 interior box over the
// 4-D view (x, y, z, field) of the buffer.  A domain qualifies when its row
// and plane pitches are multiples of 16 bytes (nx*elem % 16 == 0).
bool any_tma_ok(const mpcf_solver* s)
{
    for (const auto& D : s->hdoms) if (D.tma_ok) return true;
    return false;
}

int encode_tensor_maps(mpcf_solver* s)
{
    std::vector<CUtensorMap> h((size_t)s->ndom * 4);
    memset(h.data(), 0, h.size() * sizeof(CUtensorMap));
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    for (int d = 0; d < s->ndom; ++d)
    {
        DomDev& D = s->hdoms[d];
        const size_t e = s->esz;
        bool ok = enc != nullptr && ((size_t)D.nx * e) % 16 == 0 && ((size_t)D.nx * D.ny * e) % 16 == 0 &&
                  ((size_t)D.fs * e) % 16 == 0;
        for (int b = 0; b < 2 && ok; ++b)
            for (int box = 0; box < 2 && ok; ++box)
            {
                // over the stored planes, ghost planes included (the kernel
                // adds zlo to its z coordinates)
                const cuuint64_t dims[4] = {(cuuint64_t)D.nx, (cuuint64_t)D.ny, (cuuint64_t)(D.nz + D.zlo + D.zhi), 7};
                const cuuint64_t strides[3] = {(cuuint64_t)D.nx * e, (cuuint64_t)D.nx * D.ny * e, (cuuint64_t)D.fs * e};
                const cuuint32_t boxd[4] = {box == 0 ? 40u : 32u, (cuuint32_t)(box == 0 ? s->ty + 6 : s->ty), 1u, 7u};
                const cuuint32_t estr[4] = {1, 1, 1, 1};
                CUresult r = enc(&h[(size_t)d * 4 + b * 2 + box],
                                 e == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                 4, (char*)D.U[b] - (size_t)D.zlo * D.nx * D.ny * e, dims, strides, boxd, estr,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                ok = (r == CUDA_SUCCESS);
            }
        D.tma_ok = ok ? 1 : 0;
    }
    CK(cudaMemcpyAsync(s->tmaps, h.data(), h.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s->stream));
    return MPCF_OK;
}

void destroy_graphs(mpcf_solver* s)
{
    for (int i = 0; i < 2; ++i)
        if (s->graph[i]) { cudaGraphExecDestroy(s->graph[i]); s->graph[i] = nullptr; }
}

int dev_alloc(mpcf_solver* s, void** p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return fail(MPCF_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    s->allocs.push_back(*p);
    return MPCF_OK;
}

// Recompute the tile tables for the current tiling and upload the domain
// descriptors.
int apply_tiling(mpcf_solver* s)
{
    int t = 0, c = 0;
    for (auto& D : s->hdoms)
    {
        const size_t zsh = (size_t)D.zlo * D.nx * D.ny * s->esz;
        for (int b = 0; b < 2; ++b) D.Ux[b] = (char*)D.U[b] - zsh;
        D.Rx = (char*)D.R - zsh;
        D.nzx = D.nz + D.zlo + D.zhi;
        D.tiles_x = (D.nx + 31) / 32;
        D.tiles_y = (D.ny + s->ty - 1) / s->ty;
        D.tiles_z = (D.nz + s->dz - 1) / s->dz;
        D.tile_begin = t;
        t += D.tiles_x * D.tiles_y * D.tiles_z;
        const long long N = (long long)D.nx * D.ny * D.nz;
        D.sos_chunk_begin = c;
        D.sos_chunks = (int)((N + s->sos_chunk - 1) / s->sos_chunk);
        c += D.sos_chunks;
    }
    s->ntiles = t;
    s->nchunks = c;
    if (s->tile_sums)
    {
        cudaFree(s->tile_sums);
        s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), (void*)s->tile_sums), s->allocs.end());
        s->tile_sums = nullptr;
    }
    int rc = dev_alloc(s, (void**)&s->tile_sums, sizeof(double) * 5 * (size_t)std::max(t, 1));
    if (rc) return rc;
    if (!s->chunk_sums)
        if ((rc = dev_alloc(s, (void**)&s->chunk_sums, sizeof(double) * 5 * (size_t)std::max(c, 1)))) return rc;
    if ((rc = encode_tensor_maps(s))) return rc;
    if (s->tma && !any_tma_ok(s)) s->tma = 0;
    CK(cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    destroy_graphs(s);
    return MPCF_OK;
}

// Allow the large shared-memory footprints of every tiling variant of the
// solver's stage kernel (its precision form and reconstruction order).
int grant_shared_memory(const mpcf_solver* s)
{
    const int tys[4] = {3, 7, 8, 15};
    for (int i = 0; i < 4; ++i)
    {
        if (!valid_ty(s, tys[i])) continue;
        for (int p = 0; p < 8; ++p)
        {
            StageKernelInfo I = stage_info(s, tys[i], (p & 1) != 0, (p & 2) != 0, (p & 4) != 0);
            if (!I.fn) continue;
            if (cudaFuncSetAttribute(I.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)I.smem) != cudaSuccess)
            {
                cudaGetLastError();
                return fail(MPCF_ERR_CUDA, "cannot grant %zu B shared memory to the stage kernel (ty=%d)", I.smem, tys[i]);
            }
        }
    }
    return MPCF_OK;
}

int persistent_grid(mpcf_solver* s, int ty)
{
    StageKernelInfo I = stage_info(s, ty, true, false, s->tma != 0);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, I.fn, stage_block_threads(ty), I.smem) != cudaSuccess || nb < 1)
    {
        cudaGetLastError();
        nb = 1;
    }
    return std::min(s->ntiles, nb * s->num_sms);
}

StageArgs stage_args(mpcf_solver* s, double a, double b, bool sums)
{
    StageArgs A;
    A.doms = s->ddoms;
    A.ndom = s->ndom;
    A.ntiles = s->ntiles;
    A.tile0 = 0;
    A.dz = s->dz;
    A.parity = s->parity;
    A.a = a;
    A.b = b;
    A.dtinvh = s->dtinvh;
    A.counter = s->counter;
    A.err = s->err;
    A.tile_sums = sums ? s->tile_sums : nullptr;
    A.tmaps = s->tmaps;
    A.sos_bits = nullptr;
    A.test_flags = s->test_flags;
    return A;
}

// Enqueue the stage of tiles [tile_lo, tile_hi) on the solver's stream
// (device dt/h); the parity is left as it is (the caller flips it once the
// whole stage is enqueued).
int enqueue_stage_tiles(mpcf_solver* s, double a, double b, bool sums, bool sos, int tile_lo, int tile_hi)
{
    StageArgs A = stage_args(s, a, b, sums);
    if (sos) A.sos_bits = s->sos_bits;
    A.tile0 = tile_lo;
    A.ntiles = tile_hi;
    int grid = tile_hi - tile_lo;
    if (s->persist)
    {
        grid = std::min(grid, persistent_grid(s, s->ty));
        CK(cudaMemsetAsync(s->counter, 0, sizeof(unsigned), s->stream));
    }
    cudaError_t e = launch_stage(s, A, grid, s->stream);
    if (e != cudaSuccess) return fail(MPCF_ERR_CUDA, "stage launch failed: %s", cudaGetErrorString(e));
    return MPCF_OK;
}

// Enqueue one stage on the solver's stream (device dt/h) and flip parity.
int enqueue_stage(mpcf_solver* s, double a, double b, bool sums, bool sos = false)
{
    // linked slabs first take their neighbours' boundary planes of the state
    // this stage reads
    if (!s->links.empty())
        CK(launch_halo((int)s->esz, s->ddoms, s->dlinks, (int)s->links.size() / 2, s->link_plane, s->parity, s->stream));
    int rc = enqueue_stage_tiles(s, a, b, sums, sos, 0, s->ntiles);
    if (rc) return rc;
    s->parity ^= 1;
    if (sums)
    {
        CK(launch_sum_tiles(s->ddoms, s->ndom, s->tile_sums, s->sums, s->stream));
        s->sums_valid = true;
    }
    else s->sums_valid = false;
    return MPCF_OK;
}

int enqueue_sos(mpcf_solver* s)
{
    CK(cudaMemsetAsync(s->sos_bits, 0, s->esz * s->ndom, s->stream));
    SosArgs A;
    A.doms = s->ddoms;
    A.ndom = s->ndom;
    A.nchunks = s->nchunks;
    A.chunk = s->sos_chunk;
    A.chunk0 = 0;
    A.parity = s->parity;
    A.sos_bits = s->sos_bits;
    CK(launch_sos(s->pol, A, s->stream));
    return MPCF_OK;
}

int enqueue_dt(mpcf_solver* s, double cfl, double dt_max)
{
    DtArgs A;
    A.doms = s->ddoms;
    A.ndom = s->ndom;
    A.cfl = cfl;
    A.dt_max = dt_max;
    A.sos_bits = s->sos_bits;
    A.dtinvh = s->dtinvh;
    A.dt = s->dt;
    A.time = s->time;
    A.err = s->err;
    A.grouped = (s->links.empty() && !s->win_nch) ? 0 : 1;
    CK(launch_dt(s->pol, A, s->stream));
    return MPCF_OK;
}

// The whole LSRK3 step on the stream: sound speed (the stand-alone reduction
// when the accumulator does not hold the current state's), dt (which clears
// the accumulator), three stages; the last stage accumulates the sound speed
// of the state it writes, the next step's.
int enqueue_step(mpcf_solver* s, double cfl, double dt_max, bool standalone_sos)
{
    int rc;
    if (standalone_sos && (rc = enqueue_sos(s))) return rc;
    if ((rc = enqueue_dt(s, cfl, dt_max))) return rc;
    for (int k = 0; k < 3; ++k)
        if ((rc = enqueue_stage(s, kLSRK3[k][0], kLSRK3[k][1], s->track_cons && k == 2, k == 2))) return rc;
    return MPCF_OK;
}

// A windowed solver's domains are slots that z-chunks pass through; only
// mpcf_run_window advances them.
int window_only(const mpcf_solver* s, const char* what)
{
    return fail(MPCF_ERR_STATE, "%s: a windowed solver (%d slots of %d planes) is advanced by mpcf_run_window",
                what, s->ndom, s->win_nslices);
}

int check_dom(const mpcf_solver* s, int dom)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (dom < 0 || dom >= s->ndom) return fail(MPCF_ERR_ARG, "domain index %d out of range [0,%d)", dom, s->ndom);
    return MPCF_OK;
}

// Copy 7 fields between caller arrays and a device buffer (field stride fs).
int copy_fields(mpcf_solver* s, void* dev_base, long long fs, long long n,
                const void* const* src7, void* const* dst7, bool to_device, bool user_is_device)
{
    for (int q = 0; q < 7; ++q)
    {
        char* dev = (char*)dev_base + (size_t)q * fs * s->esz;
        const size_t bytes = (size_t)n * s->esz;
        if (to_device)
        {
            if (!src7[q]) return fail(MPCF_ERR_ARG, "field %d pointer is null", q);
            CK(cudaMemcpyAsync(dev, src7[q], bytes, user_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s->stream));
        }
        else
        {
            if (!dst7[q]) return fail(MPCF_ERR_ARG, "field %d pointer is null", q);
            CK(cudaMemcpyAsync(dst7[q], dev, bytes, user_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s->stream));
        }
    }
    return MPCF_OK;
}

} // namespace

// ===========================================================================
extern "C" {

int mpcf_version(void) { return MPCF_API_VERSION; }
const char* mpcf_last_error(void) { return g_err.c_str(); }
int mpcf_elem_size(int precision)
{
    if (precision < 0 || precision > MPCF_PREC_FP64_FAST) return fail(MPCF_ERR_ARG, "unknown precision %d", precision);
    return (precision == MPCF_PREC_FP64 || precision == MPCF_PREC_FP64_FAST) ? 8 : 4;
}

int mpcf_create(mpcf_solver** out, int ndomains, const int* dims, const int* bc, int precision, int device)
{
    if (!out) return fail(MPCF_ERR_ARG, "null output handle");
    *out = nullptr;
    if (ndomains < 1) return fail(MPCF_ERR_ARG, "ndomains must be >= 1 (got %d)", ndomains);
    if (!dims) return fail(MPCF_ERR_ARG, "null dims");
    if (precision < 0 || precision > MPCF_PREC_FP64_FAST) return fail(MPCF_ERR_ARG, "unknown precision %d", precision);
    for (int d = 0; d < ndomains; ++d)
    {
        const int nx = dims[3 * d], ny = dims[3 * d + 1], nz = dims[3 * d + 2];
        if (nx < 5 || ny < 5 || nz < 3)
            return fail(MPCF_ERR_ARG, "domain %d: size %dx%dx%d below the minimum 5x5x3", d, nx, ny, nz);
        if ((long long)nx * ny * nz > (1LL << 34))
            return fail(MPCF_ERR_ARG, "domain %d: %lld cells exceed the supported 2^34", d, (long long)nx * ny * nz);
        if (bc)
            for (int f = 0; f < 6; ++f)
            {
                const int c = bc[6 * d + f];
                if (c != MPCF_BC_ABSORBING && c != MPCF_BC_REFLECTING && !(c == MPCF_BC_HALO && f >= 4))
                    return fail(MPCF_ERR_ARG, "domain %d: boundary condition %d not valid on face %d%s", d, c, f,
                                c == MPCF_BC_HALO ? " (halo faces are z faces)" : "");
            }
    }
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(MPCF_ERR_ARG, "device %d not present (%d devices)", device, ndev);

    mpcf_solver* s = new mpcf_solver();
    s->device = device;
    s->pol = precision;
    s->ndom = ndomains;
    s->esz = (precision == MPCF_PREC_FP64 || precision == MPCF_PREC_FP64_FAST) ? 8 : 4;
    DeviceGuard g(device);
    int rc = MPCF_OK;
    auto bail = [&](int code) { mpcf_destroy(s); return code; };

    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    { cudaGetLastError(); delete s; return fail(MPCF_ERR_CUDA, "cudaStreamCreate failed"); }
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);

    s->hdoms.resize(ndomains);
    for (int d = 0; d < ndomains; ++d)
    {
        DomDev& D = s->hdoms[d];
        memset(&D, 0, sizeof(D));
        D.nx = dims[3 * d]; D.ny = dims[3 * d + 1]; D.nz = dims[3 * d + 2];
        for (int f = 0; f < 6; ++f) D.bc[f] = bc ? bc[6 * d + f] : MPCF_BC_ABSORBING;
        D.h = 1.0 / (double)std::max(D.nx, std::max(D.ny, D.nz));
        D.org[0] = D.org[1] = D.org[2] = 0;
        D.gdim[0] = D.nx; D.gdim[1] = D.ny; D.gdim[2] = D.nz;
        D.zlo = D.bc[4] == MPCF_BC_HALO ? kHaloPlanes : 0;
        D.zhi = D.bc[5] == MPCF_BC_HALO ? kHaloPlanes : 0;
        D.group = d;
        // a field holds the domain's planes plus its stored ghost planes;
        // U[b] points at plane 0 (the register has no ghost planes)
        const long long plane = (long long)D.nx * D.ny;
        const long long N = plane * (D.nz + D.zlo + D.zhi);
        D.fs = (N + 63) / 64 * 64;
        for (int b = 0; b < 2; ++b)
        {
            if ((rc = dev_alloc(s, &D.U[b], (size_t)7 * D.fs * s->esz))) return bail(rc);
            if (cudaMemsetAsync(D.U[b], 0, (size_t)7 * D.fs * s->esz, s->stream) != cudaSuccess) return bail(fail(MPCF_ERR_CUDA, "memset"));
            D.U[b] = (char*)D.U[b] + (size_t)D.zlo * plane * s->esz;
        }
        if ((rc = dev_alloc(s, &D.R, (size_t)7 * D.fs * s->esz))) return bail(rc);
        if (cudaMemsetAsync(D.R, 0, (size_t)7 * D.fs * s->esz, s->stream) != cudaSuccess) return bail(fail(MPCF_ERR_CUDA, "memset"));
    }
    if ((rc = dev_alloc(s, (void**)&s->ddoms, sizeof(DomDev) * ndomains))) return bail(rc);
    if ((rc = dev_alloc(s, &s->sos_bits, 8 * ndomains))) return bail(rc);
    if ((rc = dev_alloc(s, &s->dtinvh, 8 * ndomains))) return bail(rc);
    if ((rc = dev_alloc(s, (void**)&s->dt, 8 * ndomains))) return bail(rc);
    if ((rc = dev_alloc(s, (void**)&s->time, 8 * ndomains))) return bail(rc);
    if ((rc = dev_alloc(s, (void**)&s->sums, 8 * 5 * ndomains))) return bail(rc);
    if ((rc = dev_alloc(s, (void**)&s->err, 16))) return bail(rc);
    if ((rc = dev_alloc(s, (void**)&s->counter, 16))) return bail(rc);
    if ((rc = dev_alloc(s, &s->tmaps, (size_t)128 * 4 * ndomains))) return bail(rc);
    cudaMemsetAsync(s->sos_bits, 0, 8 * ndomains, s->stream);
    cudaMemsetAsync(s->dtinvh, 0, 8 * ndomains, s->stream);
    cudaMemsetAsync(s->dt, 0, 8 * ndomains, s->stream);
    cudaMemsetAsync(s->time, 0, 8 * ndomains, s->stream);
    cudaMemsetAsync(s->sums, 0, 8 * 5 * ndomains, s->stream);
    cudaMemsetAsync(s->err, 0, 16, s->stream);
    cudaMemsetAsync(s->counter, 0, 16, s->stream);
    if (cudaMallocHost(&s->host_stage, 8 * (size_t)ndomains * 8) != cudaSuccess)
    { cudaGetLastError(); return bail(fail(MPCF_ERR_NOMEM, "cudaMallocHost failed")); }

    if ((rc = grant_shared_memory(s))) return bail(rc);
    s->ty = 7;
    s->dz = 64;
    s->persist = 0;
    s->tma = 1;                       // dropped by apply_tiling when no domain qualifies
    if ((rc = apply_tiling(s))) return bail(rc);
    *out = s;
    return MPCF_OK;
}

int mpcf_destroy(mpcf_solver* s)
{
    if (!s) return MPCF_OK;
    DeviceGuard g(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (cudaStream_t c : {s->up, s->down})
        if (c) { cudaStreamSynchronize(c); cudaStreamDestroy(c); }
    for (auto* v : {&s->ev_up, &s->ev_st, &s->ev_down, &s->ev_free_c, &s->ev_free_d})
        for (cudaEvent_t e : *v) cudaEventDestroy(e);
    if (s->ev_start) cudaEventDestroy(s->ev_start);
    destroy_graphs(s);
    for (void* p : s->allocs) cudaFree(p);
    if (s->host_stage) cudaFreeHost(s->host_stage);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return MPCF_OK;
}

int mpcf_num_domains(const mpcf_solver* s) { return s ? s->ndom : fail(MPCF_ERR_ARG, "null solver"); }
int mpcf_precision(const mpcf_solver* s) { return s ? s->pol : fail(MPCF_ERR_ARG, "null solver"); }

int mpcf_set_state(mpcf_solver* s, int dom, const void* const* state7, const void* const* reg7, int src_is_device)
{
    Range nvtx("mpcf_set_state");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!state7) return fail(MPCF_ERR_ARG, "null state pointers");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    DomDev& D = s->hdoms[dom];
    const long long N = (long long)D.nx * D.ny * D.nz;
    if ((rc = copy_fields(s, D.U[s->parity], D.fs, N, state7, nullptr, true, src_is_device != 0))) return rc;
    if (reg7) { if ((rc = copy_fields(s, D.R, D.fs, N, reg7, nullptr, true, src_is_device != 0))) return rc; }
    else CK(cudaMemsetAsync(D.R, 0, (size_t)7 * D.fs * s->esz, s->stream));
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_get_state(mpcf_solver* s, int dom, void* const* state7, void* const* reg7, int dst_is_device)
{
    Range nvtx("mpcf_get_state");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    DeviceGuard g(s->device);
    DomDev& D = s->hdoms[dom];
    const long long N = (long long)D.nx * D.ny * D.nz;
    if (state7) { if ((rc = copy_fields(s, D.U[s->parity], D.fs, N, nullptr, state7, false, dst_is_device != 0))) return rc; }
    if (reg7)   { if ((rc = copy_fields(s, D.R, D.fs, N, nullptr, reg7, false, dst_is_device != 0))) return rc; }
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_device_pointers(mpcf_solver* s, int dom, void** state7, void** reg7)
{
    int rc = check_dom(s, dom);
    if (rc) return rc;
    DomDev& D = s->hdoms[dom];
    s->sos_fresh = false;   // the caller may write the state through these
    for (int q = 0; q < 7; ++q)
    {
        if (state7) state7[q] = (char*)D.U[s->parity] + (size_t)q * D.fs * s->esz;
        if (reg7)   reg7[q]   = (char*)D.R + (size_t)q * D.fs * s->esz;
    }
    return MPCF_OK;
}

int mpcf_max_sos(mpcf_solver* s, double* sos)
{
    Range nvtx("mpcf_max_sos");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->win_nch) return window_only(s, "mpcf_max_sos");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    int rc = enqueue_sos(s);
    if (rc) return rc;
    std::vector<char> buf(s->esz * s->ndom);
    CK(cudaMemcpyAsync(buf.data(), s->sos_bits, buf.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemsetAsync(s->sos_bits, 0, s->esz * s->ndom, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (sos)
        for (int d = 0; d < s->ndom; ++d)
            sos[d] = s->esz == 8 ? ((double*)buf.data())[d] : (double)((float*)buf.data())[d];
    return MPCF_OK;
}

int mpcf_stage(mpcf_solver* s, double a, double b, const double* dtinvh)
{
    Range nvtx("mpcf_stage");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->win_nch) return window_only(s, "mpcf_stage");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    if (dtinvh)
    {
        CK(cudaStreamSynchronize(s->stream));   // host staging buffer reuse
        for (int d = 0; d < s->ndom; ++d)
        {
            if (s->esz == 8) ((double*)s->host_stage)[d] = dtinvh[d];
            else ((float*)s->host_stage)[d] = (float)dtinvh[d];
        }
        CK(cudaMemcpyAsync(s->dtinvh, s->host_stage, s->esz * s->ndom, cudaMemcpyHostToDevice, s->stream));
    }
    int rc = enqueue_stage(s, a, b, false);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_stream(mpcf_solver* s, void** stream)
{
    if (!s || !stream) return fail(MPCF_ERR_ARG, "null argument");
    *stream = (void*)s->stream;
    return MPCF_OK;
}

int mpcf_sos_accumulator(mpcf_solver* s, void** dev_ptr)
{
    if (!s || !dev_ptr) return fail(MPCF_ERR_ARG, "null argument");
    *dev_ptr = s->sos_bits;
    return MPCF_OK;
}

int mpcf_enqueue_sos(mpcf_solver* s)
{
    Range nvtx("mpcf_enqueue_sos");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    DeviceGuard g(s->device);
    s->sos_fresh = false;
    return enqueue_sos(s);
}

int mpcf_enqueue_dt(mpcf_solver* s, double cfl, double dt_max)
{
    Range nvtx("mpcf_enqueue_dt");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (!(cfl > 0) || !(dt_max > 0)) return fail(MPCF_ERR_ARG, "cfl and dt_max must be positive");
    DeviceGuard g(s->device);
    s->sos_fresh = false;
    return enqueue_dt(s, cfl, dt_max);
}

int mpcf_enqueue_stage(mpcf_solver* s, double a, double b)
{
    Range nvtx("mpcf_enqueue_stage");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->win_nch) return window_only(s, "mpcf_enqueue_stage");
    DeviceGuard g(s->device);
    s->sos_fresh = false;
    return enqueue_stage(s, a, b, false);
}

int mpcf_compute_dt(mpcf_solver* s, double cfl, double dt_max, double* dt_out)
{
    Range nvtx("mpcf_compute_dt");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (!(cfl > 0) || !(dt_max > 0)) return fail(MPCF_ERR_ARG, "cfl and dt_max must be positive");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    int rc;
    if ((rc = enqueue_sos(s))) return rc;
    if ((rc = enqueue_dt(s, cfl, dt_max))) return rc;
    if (dt_out) CK(cudaMemcpyAsync(dt_out, s->dt, sizeof(double) * s->ndom, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_step(mpcf_solver* s, double cfl, double dt_max, double* dt_out)
{
    Range nvtx("mpcf_step");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->win_nch) return window_only(s, "mpcf_step");
    if (!(cfl > 0) || !(dt_max > 0)) return fail(MPCF_ERR_ARG, "cfl and dt_max must be positive");
    DeviceGuard g(s->device);
    int rc = enqueue_step(s, cfl, dt_max, !s->sos_fresh);
    if (rc) return rc;
    s->sos_fresh = true;
    if (dt_out)
    {
        CK(cudaMemcpyAsync(dt_out, s->dt, sizeof(double) * s->ndom, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    return MPCF_OK;
}

int mpcf_run(mpcf_solver* s, int nsteps, double cfl, double dt_max, int use_graph, double* time_out)
{
    Range nvtx("mpcf_run");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->win_nch) return window_only(s, "mpcf_run");
    if (nsteps < 0) return fail(MPCF_ERR_ARG, "nsteps < 0");
    if (!(cfl > 0) || !(dt_max > 0)) return fail(MPCF_ERR_ARG, "cfl and dt_max must be positive");
    DeviceGuard g(s->device);
    int rc;
    if (use_graph)
    {
        if (s->graph_cfl != cfl || s->graph_dtmax != dt_max || s->graph_cons != s->track_cons) destroy_graphs(s);
        for (int p = 0; p < 2; ++p)
        {
            if (s->graph[p]) continue;
            const int saved = s->parity;
            s->parity = p;
            cudaGraph_t gr = nullptr;
            CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_step(s, cfl, dt_max, false);
            cudaError_t ec = cudaStreamEndCapture(s->stream, &gr);
            s->parity = saved;
            if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
            if (ec != cudaSuccess) return fail(MPCF_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ec));
            ec = cudaGraphInstantiate(&s->graph[p], gr, 0);
            cudaGraphDestroy(gr);
            if (ec != cudaSuccess) { s->graph[p] = nullptr; return fail(MPCF_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ec)); }
        }
        s->graph_cfl = cfl;
        s->graph_dtmax = dt_max;
        s->graph_cons = s->track_cons;
        for (int n = 0; n < nsteps; ++n)
        {
            if (!s->sos_fresh && (rc = enqueue_sos(s))) return rc;
            CK(cudaGraphLaunch(s->graph[s->parity], s->stream));
            s->parity ^= 1;   // three stages: odd number of buffer swaps
            s->sos_fresh = true;
        }
        if (nsteps > 0) s->sums_valid = s->track_cons;
    }
    else
    {
        for (int n = 0; n < nsteps; ++n)
        {
            if ((rc = enqueue_step(s, cfl, dt_max, !s->sos_fresh))) return rc;
            s->sos_fresh = true;
        }
    }
    if (time_out) CK(cudaMemcpyAsync(time_out, s->time, sizeof(double) * s->ndom, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_run_host(mpcf_solver* s, int nsteps, double cfl, double dt_max, void* const* host7, int nchunks,
                  double* time_out)
{
    Range nvtx("mpcf_run_host");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->win_nch) return window_only(s, "mpcf_run_host");
    if (nsteps < 0 || nchunks < 1) return fail(MPCF_ERR_ARG, "nsteps < 0 or nchunks < 1");
    if (!(cfl > 0) || !(dt_max > 0)) return fail(MPCF_ERR_ARG, "cfl and dt_max must be positive");
    if (!host7) return fail(MPCF_ERR_ARG, "null host state");
    for (int q = 0; q < 7; ++q) if (!host7[q]) return fail(MPCF_ERR_ARG, "host field %d is null", q);
    if (s->ndom != 1) return fail(MPCF_ERR_ARG, "mpcf_run_host streams one domain (the solver has %d)", s->ndom);
    if (!s->links.empty() || s->hdoms[0].zlo || s->hdoms[0].zhi)
        return fail(MPCF_ERR_ARG, "mpcf_run_host: slabs with halo faces are not streamed");
    DeviceGuard g(s->device);
    const DomDev& D = s->hdoms[0];
    const long long plane = (long long)D.nx * D.ny;
    const size_t esz = s->esz;
    // chunks of whole tile layers (tiles never straddle two chunks); the
    // tiles of layers l0..l1-1 are the contiguous range l0*txy .. l1*txy-1
    const int layers = D.tiles_z, txy = D.tiles_x * D.tiles_y;
    const int nch = std::min(nchunks, layers);
    std::vector<int> lc(nch + 1), zc(nch + 1);
    for (int c = 0; c <= nch; ++c)
    {
        lc[c] = (int)((long long)layers * c / nch);
        zc[c] = std::min(D.nz, lc[c] * s->dz);
    }
    // streams and events, made once
    if (!s->up)
    {
        CK(cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&s->ev_start, cudaEventDisableTiming));
    }
    for (auto* v : {&s->ev_up, &s->ev_st, &s->ev_down})
        while ((int)v->size() < nch)
        {
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            v->push_back(e);
        }
    // hi[c]: the last chunk within 3 planes above chunk c (a stage reads 3
    // planes beyond its cells); a stage of chunk c may run once the stage
    // before it (or the upload) has covered chunks 0..hi[c]
    std::vector<int> hi(nch);
    for (int c = 0; c < nch; ++c)
    {
        int j = c;
        while (j + 1 < nch && zc[j + 1] < zc[c + 1] + 3) ++j;
        hi[c] = j;
    }
    // the first upload overwrites the state only after the work already
    // queued on the solver's stream
    CK(cudaEventRecord(s->ev_start, s->stream));
    CK(cudaStreamWaitEvent(s->up, s->ev_start, 0));
    int rc;
    for (int n = 0; n < nsteps; ++n)
    {
        const int p = s->parity;
        // (1) the step's input: chunk c of the host state into the state
        // buffer, once the previous step's result of chunk c is on the host
        char* dev = (char*)D.U[p];
        for (int c = 0; c < nch; ++c)
        {
            if (n > 0) CK(cudaStreamWaitEvent(s->up, s->ev_down[c], 0));
            const size_t off = (size_t)zc[c] * plane * esz, bytes = (size_t)(zc[c + 1] - zc[c]) * plane * esz;
            for (int q = 0; q < 7; ++q)
                CK(cudaMemcpyAsync(dev + (size_t)q * D.fs * esz + off, (const char*)host7[q] + off, bytes,
                                   cudaMemcpyHostToDevice, s->up));
            CK(cudaEventRecord(s->ev_up[c], s->up));
        }
        // (2) the maximum sound speed of the input.  First step: reduced
        // chunk by chunk as the chunks land.  Later steps: the input is the
        // previous step's result, whose sound speed stage 3 accumulated as
        // it wrote it (as in a resident run), so dt needs no whole upload.
        if (n == 0)
        {
            CK(cudaMemsetAsync(s->sos_bits, 0, esz, s->stream));
            int done = 0;
            for (int c = 0; c < nch; ++c)
            {
                CK(cudaStreamWaitEvent(s->stream, s->ev_up[c], 0));
                const int upto = c == nch - 1 ? s->nchunks : (int)((long long)zc[c + 1] * plane / s->sos_chunk);
                if (upto <= done) continue;
                SosArgs A;
                A.doms = s->ddoms;
                A.ndom = 1;
                A.nchunks = upto - done;
                A.chunk = s->sos_chunk;
                A.chunk0 = done;
                A.parity = p;
                A.sos_bits = s->sos_bits;
                CK(launch_sos(s->pol, A, s->stream));
                done = upto;
            }
        }
        if ((rc = enqueue_dt(s, cfl, dt_max))) return rc;
        // (3) the three stages as a wavefront over the chunks: stage k of
        // chunk c follows stage k-1 (stage 1: the upload) of chunks
        // 0..hi[c].  Stage k reads buffer p ^ (k & 1) and writes the other;
        // a chunk's stage overwrites planes that only the previous stage of
        // chunks up to hi[c] read, so these read-after-write orders also
        // cover the buffers' reuse.  Stage 3 accumulates the sound speed of
        // the state it writes (the next step's dt) and hands each chunk to
        // the download stream.
        int d[3] = {0, 0, 0};
        while (d[2] < nch)
        {
            int k = 0;
            if (d[1] > hi[d[2]]) k = 2;
            else if (d[1] < nch && d[0] > hi[d[1]]) k = 1;
            const int c = d[k]++;
            if (k == 0) CK(cudaStreamWaitEvent(s->stream, s->ev_up[hi[c]], 0));
            s->parity = p ^ (k & 1);
            rc = enqueue_stage_tiles(s, kLSRK3[k][0], kLSRK3[k][1], false, k == 2, lc[c] * txy, lc[c + 1] * txy);
            s->parity = p;
            if (rc) return rc;
            if (k == 2) CK(cudaEventRecord(s->ev_st[c], s->stream));
        }
        s->parity = p ^ 1;
        const char* res = (const char*)D.U[p ^ 1];
        for (int c = 0; c < nch; ++c)
        {
            CK(cudaStreamWaitEvent(s->down, s->ev_st[c], 0));
            const size_t off = (size_t)zc[c] * plane * esz, bytes = (size_t)(zc[c + 1] - zc[c]) * plane * esz;
            for (int q = 0; q < 7; ++q)
                CK(cudaMemcpyAsync((char*)host7[q] + off, res + (size_t)q * D.fs * esz + off, bytes,
                                   cudaMemcpyDeviceToHost, s->down));
            CK(cudaEventRecord(s->ev_down[c], s->down));
        }
    }
    // the device state equals the host result, and the sound-speed
    // accumulator holds its maximum (from the last stage 3)
    if (nsteps > 0) s->sos_fresh = true;
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->down));
    CK(cudaStreamSynchronize(s->up));
    if (time_out) CK(cudaMemcpyAsync(time_out, s->time, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

// ---------------------------------------------------------------------------
// Windowed runs: a domain held in host memory that may exceed device memory
// (GPUlab's z-chunks of nslices planes streamed through the GPU,
// GPUlab.cpp:202-372,703-793).  The solver's domains are slots of nslices
// planes with 3 stored ghost planes on each z side.
// ---------------------------------------------------------------------------
namespace {

// Slot of chunk c of step n: the chunks of successive steps take the slots
// in turn, so the first chunks of a step reuse slots freed in the middle of
// the step before (had every step restarted at slot 0, its first upload
// would wait for the previous step's last chunks).  The sound-speed pass
// (step -1) starts at slot 0.
inline int window_slot(const int n, const int c, const int nch, const int ns)
{
    return n < 0 ? c % ns : (int)(((long long)n * nch + c) % ns);
}

// One operation of a windowed run in the order the host enqueues it.  step
// -1: the sound-speed pass of the first step's input.
struct WinOp { int op, step, stage, chunk; };
enum { WOP_UPLOAD = 0, WOP_SOS = 1, WOP_DT = 2, WOP_STAGE = 3, WOP_DOWNLOAD = 4 };

// The plan of nsteps steps of nch chunks through ns slots.  Stage k of chunk
// c needs stage k-1 (stage 1: the upload) of chunks up to c+1, whose planes
// its upper ghost planes copy; a slot is free for its next chunk once that
// chunk's stage 3 has been downloaded and the stage 3 of the chunk above
// (which copies its top planes) is queued.  Each step's dt needs the sound
// speed of all of its input: the first from a pass that streams every chunk
// through the slots and reduces it, later ones from what stage 3 of the
// step before accumulated.  That pass runs from the last chunk down, so it
// leaves chunks 0 .. ns-1 in their slots, where the first step finds them
// without uploading them again.  Operations are taken greedily, downloads and
// the later stages first; false if nothing can proceed (too few slots).
bool window_plan(const int nch, const int ns, const int nsteps, std::vector<WinOp>& plan)
{
    plan.clear();
    if (nsteps <= 0) return true;
    if (nch < 1 || ns < 1) return false;
    auto hi = [&](const int c) { return std::min(c + 1, nch - 1); };
    // the sound-speed pass, from the last chunk down: chunk c into slot
    // c % ns once chunk c + ns has been reduced
    for (int u = 0, q = 0; q < nch;)
    {
        if (u < nch && u - q < ns) plan.push_back({WOP_UPLOAD, -1, 0, nch - 1 - u++});
        else plan.push_back({WOP_SOS, -1, 0, nch - 1 - q++});
    }
    plan.push_back({WOP_DT, 0, 0, 0});
    int dts = 1;                                   // steps whose dt is queued
    const long long total = (long long)nsteps * nch;
    const int kept = std::min(ns, nch);           // the first step's chunks the pass left in place
    long long up = kept, dn = 0, st[3] = {0, 0, 0};   // next operation of each kind (step * nch + chunk)
    std::vector<long long> occ(ns, -1);
    std::vector<char> busy(ns, 0);
    for (int k = 0; k < kept; ++k) { busy[k] = 1; occ[k] = k; }
    auto released = [&](const long long j)
    {
        const long long above = (j % nch == nch - 1) ? j : j + 1;
        return st[2] > above && dn > j;
    };
    while (dn < total)
    {
        for (int k = 0; k < ns; ++k)
            if (busy[k] && released(occ[k])) busy[k] = 0;
        if (st[2] > dn)
        {
            plan.push_back({WOP_DOWNLOAD, (int)(dn / nch), 0, (int)(dn % nch)});
            ++dn;
            continue;
        }
        if (dts < nsteps && st[2] >= (long long)dts * nch)
        {
            plan.push_back({WOP_DT, dts, 0, 0});
            ++dts;
            continue;
        }
        bool did = false;
        for (int k = 2; k >= 0 && !did; --k)
        {
            const long long j = st[k];
            if (j >= total) continue;
            const int n = (int)(j / nch), c = (int)(j % nch);
            if (n >= dts) continue;
            const long long need = (long long)n * nch + hi(c);
            if ((k == 0 ? up : st[k - 1]) > need)
            {
                plan.push_back({WOP_STAGE, n, k, c});
                ++st[k];
                did = true;
            }
        }
        if (did) continue;
        if (up < total)
        {
            const int slot = (int)(up % ns);   // window_slot of (up / nch, up % nch)
            if (!busy[slot])
            {
                busy[slot] = 1;
                occ[slot] = up;
                plan.push_back({WOP_UPLOAD, (int)(up / nch), 0, (int)(up % nch)});
                ++up;
                continue;
            }
        }
        return false;
    }
    return true;
}

// The plan of one stage of a block whose state and register live in host
// memory (mpcf_window_stage, the reference's process_all over nslices
// chunks): chunk c's state and register go into slot c % ns, its stage runs
// once chunk c+1 is there (its upper ghost planes), then both come back; a
// slot takes its next chunk once its chunk was downloaded and the stage of
// the chunk above, which reads its top planes, is queued.
bool window_stage_plan(const int nch, const int ns, std::vector<WinOp>& plan)
{
    plan.clear();
    if (nch < 1 || ns < 1) return false;
    int up = 0, st = 0, dn = 0;
    std::vector<int> occ(ns, -1);
    std::vector<char> busy(ns, 0);
    auto released = [&](const int j) { return st > (j == nch - 1 ? j : j + 1) && dn > j; };
    while (dn < nch)
    {
        for (int k = 0; k < ns; ++k)
            if (busy[k] && released(occ[k])) busy[k] = 0;
        if (st > dn) { plan.push_back({WOP_DOWNLOAD, 0, 0, dn++}); continue; }
        if (st < nch && up > std::min(st + 1, nch - 1)) { plan.push_back({WOP_STAGE, 0, 0, st++}); continue; }
        if (up < nch && !busy[up % ns])
        {
            busy[up % ns] = 1;
            occ[up % ns] = up;
            plan.push_back({WOP_UPLOAD, 0, 0, up++});
            continue;
        }
        return false;
    }
    return true;
}

// Streams and events of a windowed call, made on first use; the slots'
// last use by work already queued on the solver's stream frees them.
int window_begin(mpcf_solver* s)
{
    const int nch = s->win_nch, ns = s->ndom;
    if (!s->up)
    {
        CK(cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&s->ev_start, cudaEventDisableTiming));
    }
    auto grow = [&](std::vector<cudaEvent_t>& v, const int n)
    {
        while ((int)v.size() < n)
        {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
            v.push_back(e);
        }
        return true;
    };
    if (!grow(s->ev_up, nch) || !grow(s->ev_st, nch) || !grow(s->ev_free_c, ns) || !grow(s->ev_free_d, ns))
    { cudaGetLastError(); return fail(MPCF_ERR_CUDA, "cudaEventCreate failed"); }
    CK(cudaEventRecord(s->ev_start, s->stream));
    CK(cudaStreamWaitEvent(s->up, s->ev_start, 0));
    CK(cudaStreamWaitEvent(s->down, s->ev_start, 0));
    for (int k = 0; k < ns; ++k)
    {
        CK(cudaEventRecord(s->ev_free_c[k], s->stream));
        CK(cudaEventRecord(s->ev_free_d[k], s->down));
    }
    return MPCF_OK;
}

int window_end(mpcf_solver* s)
{
    s->sos_fresh = false;
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->down));
    CK(cudaStreamSynchronize(s->up));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

} // namespace

int mpcf_window_plan(int nchunks, int nslots, int nsteps, int* ops4, int cap)
{
    std::vector<WinOp> plan;
    if (nchunks < 1 || nslots < 1 || nsteps < 0) return fail(MPCF_ERR_ARG, "nchunks, nslots >= 1 and nsteps >= 0");
    if (!window_plan(nchunks, nslots, nsteps, plan))
        return fail(MPCF_ERR_ARG, "%d slots are too few for %d chunks", nslots, nchunks);
    if (ops4)
        for (int i = 0; i < (int)plan.size() && i < cap; ++i)
        {
            ops4[4 * i] = plan[i].op;
            ops4[4 * i + 1] = plan[i].step;
            ops4[4 * i + 2] = plan[i].stage;
            ops4[4 * i + 3] = plan[i].chunk;
        }
    return (int)plan.size();
}

int mpcf_window_stage_plan(int nchunks, int nslots, int* ops4, int cap)
{
    std::vector<WinOp> plan;
    if (nchunks < 1 || nslots < 1) return fail(MPCF_ERR_ARG, "nchunks and nslots must be >= 1");
    if (!window_stage_plan(nchunks, nslots, plan))
        return fail(MPCF_ERR_ARG, "%d slots are too few for %d chunks", nslots, nchunks);
    if (ops4)
        for (int i = 0; i < (int)plan.size() && i < cap; ++i)
        {
            ops4[4 * i] = plan[i].op;
            ops4[4 * i + 1] = plan[i].step;
            ops4[4 * i + 2] = plan[i].stage;
            ops4[4 * i + 3] = plan[i].chunk;
        }
    return (int)plan.size();
}

int mpcf_create_window(mpcf_solver** out, int nx, int ny, int nz, int nslices, int nslots, int precision,
                       const int* bc6, int device)
{
    if (!out) return fail(MPCF_ERR_ARG, "null output handle");
    *out = nullptr;
    if (nslices < kHaloPlanes || nz < nslices || nz % nslices)
        return fail(MPCF_ERR_ARG, "nslices (%d) must be at least %d and divide nz (%d)", nslices, kHaloPlanes, nz);
    const int nch = nz / nslices;
    const int ns = std::min(nslots, nch);
    std::vector<WinOp> plan;
    if (nslots < 1 || !window_plan(nch, ns, 2, plan))
        return fail(MPCF_ERR_ARG, "%d slots are too few for %d chunks (at least %d)", nslots, nch, std::min(5, nch));
    int bc[6] = {MPCF_BC_ABSORBING, MPCF_BC_ABSORBING, MPCF_BC_ABSORBING, MPCF_BC_ABSORBING,
                 MPCF_BC_ABSORBING, MPCF_BC_ABSORBING};
    if (bc6)
        for (int f = 0; f < 6; ++f)
        {
            if (bc6[f] != MPCF_BC_ABSORBING && bc6[f] != MPCF_BC_REFLECTING)
                return fail(MPCF_ERR_ARG, "boundary condition %d on face %d: absorbing or reflecting", bc6[f], f);
            bc[f] = bc6[f];
        }
    std::vector<int> dims(3 * ns), bcs(6 * ns);
    for (int d = 0; d < ns; ++d)
    {
        dims[3 * d] = nx; dims[3 * d + 1] = ny; dims[3 * d + 2] = nslices;
        for (int f = 0; f < 4; ++f) bcs[6 * d + f] = bc[f];
        bcs[6 * d + 4] = bcs[6 * d + 5] = MPCF_BC_HALO;
    }
    mpcf_solver* s = nullptr;
    int rc = mpcf_create(&s, ns, dims.data(), bcs.data(), precision, device);
    if (rc) return rc;
    s->win_nz = nz;
    s->win_nslices = nslices;
    s->win_nch = nch;
    s->win_bc[0] = bc[4];
    s->win_bc[1] = bc[5];
    // the domain's spacing and geometry; all slots advance with one dt
    const double h = 1.0 / (double)std::max(nx, std::max(ny, nz));
    for (int d = 0; d < ns; ++d)
    {
        DomDev& D = s->hdoms[d];
        D.h = h;
        D.group = 0;
        D.gdim[0] = nx; D.gdim[1] = ny; D.gdim[2] = nz;
    }
    DeviceGuard g(s->device);
    if (cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom, cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
    {
        cudaGetLastError();
        mpcf_destroy(s);
        return fail(MPCF_ERR_CUDA, "window set-up copy failed");
    }
    *out = s;
    return MPCF_OK;
}

int mpcf_window_info(const mpcf_solver* s, int* info4)
{
    if (!s || !info4) return fail(MPCF_ERR_ARG, "null argument");
    if (!s->win_nch) return fail(MPCF_ERR_STATE, "not a windowed solver");
    info4[0] = s->win_nz;
    info4[1] = s->win_nslices;
    info4[2] = s->win_nch;
    info4[3] = s->ndom;
    return MPCF_OK;
}

int mpcf_run_window(mpcf_solver* s, int nsteps, double cfl, double dt_max, void* const* host7, double* time_out)
{
    Range nvtx("mpcf_run_window");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (!s->win_nch) return fail(MPCF_ERR_STATE, "mpcf_run_window needs a windowed solver (mpcf_create_window)");
    if (nsteps < 0) return fail(MPCF_ERR_ARG, "nsteps < 0");
    if (!(cfl > 0) || !(dt_max > 0)) return fail(MPCF_ERR_ARG, "cfl and dt_max must be positive");
    if (!host7) return fail(MPCF_ERR_ARG, "null host state");
    for (int q = 0; q < 7; ++q) if (!host7[q]) return fail(MPCF_ERR_ARG, "host field %d is null", q);
    const int nch = s->win_nch, ns = s->ndom, nsl = s->win_nslices;
    std::vector<WinOp> plan;
    if (!window_plan(nch, ns, nsteps, plan)) return fail(MPCF_ERR_STATE, "window plan stalled (%d slots, %d chunks)", ns, nch);
    DeviceGuard g(s->device);
    const long long plane = (long long)s->hdoms[0].nx * s->hdoms[0].ny;
    const size_t esz = s->esz;
    const size_t cbytes = (size_t)nsl * plane * esz;        // one field of one chunk
    const long long fs = s->hdoms[0].fs;
    int rc;
    if ((rc = window_begin(s))) return rc;
    CK(cudaMemsetAsync(s->sos_bits, 0, esz * ns, s->stream));
    const int p0 = s->parity;
    for (const WinOp& o : plan)
    {
        const int c = o.chunk, slot = window_slot(o.step, c, nch, ns);
        const int p = o.step < 0 ? p0 : (p0 ^ (o.step & 1));      // the step's input buffer
        DomDev& D = s->hdoms[slot];
        const size_t off = (size_t)c * cbytes;
        switch (o.op)
        {
            case WOP_UPLOAD:
                CK(cudaStreamWaitEvent(s->up, s->ev_free_c[slot], 0));
                CK(cudaStreamWaitEvent(s->up, s->ev_free_d[slot], 0));
                for (int q = 0; q < 7; ++q)
                    CK(cudaMemcpyAsync((char*)D.U[p] + (size_t)q * fs * esz, (const char*)host7[q] + off, cbytes,
                                       cudaMemcpyHostToDevice, s->up));
                CK(cudaEventRecord(s->ev_up[c], s->up));
                break;
            case WOP_SOS:
            {
                CK(cudaStreamWaitEvent(s->stream, s->ev_up[c], 0));
                SosArgs A;
                A.doms = s->ddoms;
                A.ndom = ns;
                A.nchunks = D.sos_chunks;
                A.chunk = s->sos_chunk;
                A.chunk0 = D.sos_chunk_begin;
                A.parity = p;
                A.sos_bits = s->sos_bits;
                CK(launch_sos(s->pol, A, s->stream));
                CK(cudaEventRecord(s->ev_free_c[slot], s->stream));
                break;
            }
            case WOP_DT:
                if ((rc = enqueue_dt(s, cfl, dt_max))) return rc;
                break;
            case WOP_STAGE:
            {
                const int k = o.stage, b = p ^ (k & 1);
                if (k == 0) CK(cudaStreamWaitEvent(s->stream, s->ev_up[std::min(c + 1, nch - 1)], 0));
                const void* lo = c > 0 ? s->hdoms[window_slot(o.step, c - 1, nch, ns)].U[b] : nullptr;
                const void* hi = c < nch - 1 ? s->hdoms[window_slot(o.step, c + 1, nch, ns)].U[b] : nullptr;
                CK(launch_window_ghosts((int)esz, D.U[b], lo, hi, fs, plane, nsl, s->win_bc[0], s->win_bc[1], s->stream));
                s->parity = b;
                rc = enqueue_stage_tiles(s, kLSRK3[k][0], kLSRK3[k][1], false, k == 2, D.tile_begin,
                                         D.tile_begin + D.tiles_x * D.tiles_y * D.tiles_z);
                s->parity = p0;
                if (rc) return rc;
                if (k == 2)
                {
                    CK(cudaEventRecord(s->ev_st[c], s->stream));
                    // the chunk below is no longer read (its top planes were
                    // this stage's lower ghost planes); the last chunk frees
                    // its own slot
                    if (c > 0) CK(cudaEventRecord(s->ev_free_c[window_slot(o.step, c - 1, nch, ns)], s->stream));
                    if (c == nch - 1) CK(cudaEventRecord(s->ev_free_c[slot], s->stream));
                }
                break;
            }
            case WOP_DOWNLOAD:
                CK(cudaStreamWaitEvent(s->down, s->ev_st[c], 0));
                for (int q = 0; q < 7; ++q)
                    CK(cudaMemcpyAsync((char*)host7[q] + off, (const char*)D.U[p ^ 1] + (size_t)q * fs * esz, cbytes,
                                       cudaMemcpyDeviceToHost, s->down));
                CK(cudaEventRecord(s->ev_free_d[slot], s->down));
                break;
        }
    }
    s->parity = p0 ^ (nsteps & 1);
    if ((rc = window_end(s))) return rc;
    if (time_out)
    {
        CK(cudaMemcpyAsync(time_out, s->time, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    return MPCF_OK;
}

int mpcf_window_stage(mpcf_solver* s, double a, double b, double dtinvh, void* const* state7, void* const* reg7)
{
    Range nvtx("mpcf_window_stage");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (!s->win_nch) return fail(MPCF_ERR_STATE, "mpcf_window_stage needs a windowed solver (mpcf_create_window)");
    if (!state7 || !reg7) return fail(MPCF_ERR_ARG, "null host state or register");
    for (int q = 0; q < 7; ++q)
        if (!state7[q] || !reg7[q]) return fail(MPCF_ERR_ARG, "host field %d is null", q);
    const int nch = s->win_nch, ns = s->ndom, nsl = s->win_nslices;
    std::vector<WinOp> plan;
    if (!window_stage_plan(nch, ns, plan)) return fail(MPCF_ERR_STATE, "window stage plan stalled (%d slots, %d chunks)", ns, nch);
    DeviceGuard g(s->device);
    int rc;
    // dt/h of the stage for every slot
    CK(cudaStreamSynchronize(s->stream));   // host staging buffer reuse
    for (int d = 0; d < ns; ++d)
    {
        if (s->esz == 8) ((double*)s->host_stage)[d] = dtinvh;
        else ((float*)s->host_stage)[d] = (float)dtinvh;
    }
    CK(cudaMemcpyAsync(s->dtinvh, s->host_stage, s->esz * ns, cudaMemcpyHostToDevice, s->stream));
    if ((rc = window_begin(s))) return rc;
    const long long plane = (long long)s->hdoms[0].nx * s->hdoms[0].ny;
    const size_t esz = s->esz;
    const size_t cbytes = (size_t)nsl * plane * esz;
    const long long fs = s->hdoms[0].fs;
    const int p = s->parity;
    for (const WinOp& o : plan)
    {
        const int c = o.chunk, slot = c % ns;
        DomDev& D = s->hdoms[slot];
        const size_t off = (size_t)c * cbytes;
        if (o.op == WOP_UPLOAD)
        {
            CK(cudaStreamWaitEvent(s->up, s->ev_free_c[slot], 0));
            CK(cudaStreamWaitEvent(s->up, s->ev_free_d[slot], 0));
            for (int q = 0; q < 7; ++q)
            {
                CK(cudaMemcpyAsync((char*)D.U[p] + (size_t)q * fs * esz, (const char*)state7[q] + off, cbytes,
                                   cudaMemcpyHostToDevice, s->up));
                CK(cudaMemcpyAsync((char*)D.R + (size_t)q * fs * esz, (const char*)reg7[q] + off, cbytes,
                                   cudaMemcpyHostToDevice, s->up));
            }
            CK(cudaEventRecord(s->ev_up[c], s->up));
        }
        else if (o.op == WOP_STAGE)
        {
            CK(cudaStreamWaitEvent(s->stream, s->ev_up[std::min(c + 1, nch - 1)], 0));
            const void* lo = c > 0 ? s->hdoms[(c - 1) % ns].U[p] : nullptr;
            const void* hi = c < nch - 1 ? s->hdoms[(c + 1) % ns].U[p] : nullptr;
            CK(launch_window_ghosts((int)esz, D.U[p], lo, hi, fs, plane, nsl, s->win_bc[0], s->win_bc[1], s->stream));
            if ((rc = enqueue_stage_tiles(s, a, b, false, false, D.tile_begin, D.tile_begin + D.tiles_x * D.tiles_y * D.tiles_z)))
                return rc;
            CK(cudaEventRecord(s->ev_st[c], s->stream));
            if (c > 0) CK(cudaEventRecord(s->ev_free_c[(c - 1) % ns], s->stream));
            if (c == nch - 1) CK(cudaEventRecord(s->ev_free_c[slot], s->stream));
        }
        else
        {
            CK(cudaStreamWaitEvent(s->down, s->ev_st[c], 0));
            for (int q = 0; q < 7; ++q)
            {
                CK(cudaMemcpyAsync((char*)state7[q] + off, (const char*)D.U[p ^ 1] + (size_t)q * fs * esz, cbytes,
                                   cudaMemcpyDeviceToHost, s->down));
                CK(cudaMemcpyAsync((char*)reg7[q] + off, (const char*)D.R + (size_t)q * fs * esz, cbytes,
                                   cudaMemcpyDeviceToHost, s->down));
            }
            CK(cudaEventRecord(s->ev_free_d[slot], s->down));
        }
    }
    return window_end(s);
}

int mpcf_window_max_sos(mpcf_solver* s, const void* const* state7, double* sos)
{
    Range nvtx("mpcf_window_max_sos");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (!s->win_nch) return fail(MPCF_ERR_STATE, "mpcf_window_max_sos needs a windowed solver (mpcf_create_window)");
    if (!state7) return fail(MPCF_ERR_ARG, "null host state");
    for (int q = 0; q < 7; ++q) if (!state7[q]) return fail(MPCF_ERR_ARG, "host field %d is null", q);
    const int nch = s->win_nch, ns = s->ndom, nsl = s->win_nslices;
    DeviceGuard g(s->device);
    int rc;
    if ((rc = window_begin(s))) return rc;
    const long long plane = (long long)s->hdoms[0].nx * s->hdoms[0].ny;
    const size_t esz = s->esz;
    const size_t cbytes = (size_t)nsl * plane * esz;
    const long long fs = s->hdoms[0].fs;
    const int p = s->parity;
    CK(cudaMemsetAsync(s->sos_bits, 0, esz * ns, s->stream));
    for (int c = 0; c < nch; ++c)
    {
        const int slot = c % ns;
        DomDev& D = s->hdoms[slot];
        CK(cudaStreamWaitEvent(s->up, s->ev_free_c[slot], 0));
        for (int q = 0; q < 7; ++q)
            CK(cudaMemcpyAsync((char*)D.U[p] + (size_t)q * fs * esz, (const char*)state7[q] + (size_t)c * cbytes, cbytes,
                               cudaMemcpyHostToDevice, s->up));
        CK(cudaEventRecord(s->ev_up[c], s->up));
        CK(cudaStreamWaitEvent(s->stream, s->ev_up[c], 0));
        SosArgs A;
        A.doms = s->ddoms;
        A.ndom = ns;
        A.nchunks = D.sos_chunks;
        A.chunk = s->sos_chunk;
        A.chunk0 = D.sos_chunk_begin;
        A.parity = p;
        A.sos_bits = s->sos_bits;
        CK(launch_sos(s->pol, A, s->stream));
        CK(cudaEventRecord(s->ev_free_c[slot], s->stream));
    }
    std::vector<char> buf(esz * ns);
    CK(cudaMemcpyAsync(buf.data(), s->sos_bits, buf.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemsetAsync(s->sos_bits, 0, esz * ns, s->stream));
    if ((rc = window_end(s))) return rc;
    // the largest over the slots; a NaN anywhere (its bit pattern orders
    // above every finite value in the device's maximum) stays NaN
    double m = 0;
    bool nan = false;
    for (int d = 0; d < ns; ++d)
    {
        const double v = esz == 8 ? ((double*)buf.data())[d] : (double)((float*)buf.data())[d];
        if (v != v) nan = true;
        else if (v > m) m = v;
    }
    if (sos) *sos = nan ? std::numeric_limits<double>::quiet_NaN() : m;
    return MPCF_OK;
}

int mpcf_synchronize(mpcf_solver* s)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    DeviceGuard g(s->device);
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_set_track_conservation(mpcf_solver* s, int on)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    s->track_cons = on != 0;
    return MPCF_OK;
}

int mpcf_conserved_sums(mpcf_solver* s, double* out)
{
    Range nvtx("mpcf_conserved_sums");
    if (!s || !out) return fail(MPCF_ERR_ARG, "null argument");
    DeviceGuard g(s->device);
    if (!s->sums_valid)
    {
        // deterministic two-pass reduction of the current state
        CK(launch_sum_state(s->ddoms, s->ndom, s->parity, s->nchunks, s->sos_chunk, s->esz == 8,
                            s->chunk_sums, s->sums, s->stream));
        s->sums_valid = true;
    }
    CK(cudaMemcpyAsync(out, s->sums, sizeof(double) * 5 * s->ndom, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_error_word(mpcf_solver* s, unsigned* word, int clear)
{
    if (!s || !word) return fail(MPCF_ERR_ARG, "null argument");
    DeviceGuard g(s->device);
    CK(cudaMemcpyAsync(s->host_stage, s->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    if (clear) CK(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->stream));
    CK(cudaStreamSynchronize(s->stream));
    *word = *(unsigned*)s->host_stage;
    return MPCF_OK;
}

int mpcf_set_bc(mpcf_solver* s, int dom, const int* bc6)
{
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!bc6) return fail(MPCF_ERR_ARG, "null bc");
    if (s->win_nch)
    {
        // a windowed solver: the domain's faces; x/y go to every slot, z to
        // the ghost planes at the domain's own z faces
        if (dom != 0) return fail(MPCF_ERR_ARG, "a windowed solver has one domain (index 0)");
        for (int f = 0; f < 6; ++f)
            if (bc6[f] != MPCF_BC_ABSORBING && bc6[f] != MPCF_BC_REFLECTING)
                return fail(MPCF_ERR_ARG, "boundary condition %d on face %d: absorbing or reflecting", bc6[f], f);
        DeviceGuard g(s->device);
        for (int d = 0; d < s->ndom; ++d)
            for (int f = 0; f < 4; ++f) s->hdoms[d].bc[f] = bc6[f];
        s->win_bc[0] = bc6[4];
        s->win_bc[1] = bc6[5];
        CK(cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom, cudaMemcpyHostToDevice, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        return MPCF_OK;
    }
    for (int f = 0; f < 6; ++f)
    {
        if (bc6[f] != MPCF_BC_ABSORBING && bc6[f] != MPCF_BC_REFLECTING && bc6[f] != MPCF_BC_HALO)
            return fail(MPCF_ERR_ARG, "unknown boundary condition %d on face %d", bc6[f], f);
        if ((bc6[f] == MPCF_BC_HALO) != (s->hdoms[dom].bc[f] == MPCF_BC_HALO))
            return fail(MPCF_ERR_ARG, "face %d: halo faces are fixed when the solver is created", f);
    }
    DeviceGuard g(s->device);
    for (int f = 0; f < 6; ++f) s->hdoms[dom].bc[f] = bc6[f];
    CK(cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_link_z(mpcf_solver* s, int lower, int upper)
{
    Range nvtx("mpcf_link_z");
    int rc = check_dom(s, lower);
    if (rc) return rc;
    if (s->win_nch) return window_only(s, "mpcf_link_z");
    if ((rc = check_dom(s, upper))) return rc;
    if (lower == upper) return fail(MPCF_ERR_ARG, "a domain cannot be linked to itself");
    const DomDev& L = s->hdoms[lower];
    const DomDev& H = s->hdoms[upper];
    if (L.bc[5] != MPCF_BC_HALO) return fail(MPCF_ERR_ARG, "domain %d: the z-right face is not a halo face", lower);
    if (H.bc[4] != MPCF_BC_HALO) return fail(MPCF_ERR_ARG, "domain %d: the z-left face is not a halo face", upper);
    if (L.nx != H.nx || L.ny != H.ny)
        return fail(MPCF_ERR_ARG, "linked slabs differ in x-y size (%dx%d vs %dx%d)", L.nx, L.ny, H.nx, H.ny);
    for (size_t i = 0; i < s->links.size(); i += 2)
        if (s->links[i] == lower || s->links[i + 1] == upper)
            return fail(MPCF_ERR_ARG, "face already linked (domains %d, %d)", lower, upper);
    // the exchange kernel gives every link 14 block rows (grid y <= 65535)
    if (s->links.size() / 2 + 1 > 65535 / 14)
        return fail(MPCF_ERR_ARG, "at most %d links per solver", 65535 / 14);
    DeviceGuard g(s->device);
    s->links.push_back(lower);
    s->links.push_back(upper);
    s->link_plane = std::max(s->link_plane, (long long)L.nx * L.ny);
    // groups: connected components of the links, named by their lowest domain
    std::vector<int> grp(s->ndom);
    for (int d = 0; d < s->ndom; ++d) grp[d] = d;
    for (bool changed = true; changed;)
    {
        changed = false;
        for (size_t i = 0; i < s->links.size(); i += 2)
        {
            const int a = s->links[i], b = s->links[i + 1];
            const int m = std::min(grp[a], grp[b]);
            if (grp[a] != m || grp[b] != m) { grp[a] = grp[b] = m; changed = true; }
        }
    }
    for (int d = 0; d < s->ndom; ++d) s->hdoms[d].group = grp[d];
    if (s->dlinks)
    {
        cudaFree(s->dlinks);
        s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), (void*)s->dlinks), s->allocs.end());
        s->dlinks = nullptr;
    }
    if ((rc = dev_alloc(s, (void**)&s->dlinks, sizeof(int) * s->links.size()))) return rc;
    CK(cudaMemcpyAsync(s->dlinks, s->links.data(), sizeof(int) * s->links.size(), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    destroy_graphs(s);               // the step now begins each stage with the exchange
    s->sos_fresh = false;            // dt of the group comes from the stand-alone reduction
    return MPCF_OK;
}

int mpcf_set_spacing(mpcf_solver* s, int dom, double h)
{
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!(h > 0.0) || std::isinf(h)) return fail(MPCF_ERR_ARG, "grid spacing must be positive and finite");
    DeviceGuard g(s->device);
    s->hdoms[dom].h = h;
    CK(cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_set_origin(mpcf_solver* s, int dom, const int* org3, const int* global3)
{
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!org3 || !global3) return fail(MPCF_ERR_ARG, "null origin or global size");
    DomDev& D = s->hdoms[dom];
    const int n[3] = {D.nx, D.ny, D.nz};
    for (int a = 0; a < 3; ++a)
        if (org3[a] < 0 || global3[a] < n[a] || org3[a] > global3[a] - n[a])
            return fail(MPCF_ERR_ARG, "axis %d: cells %d..%d outside the global extent %d", a, org3[a], org3[a] + n[a] - 1, global3[a]);
    DeviceGuard g(s->device);
    for (int a = 0; a < 3; ++a) { D.org[a] = org3[a]; D.gdim[a] = global3[a]; }
    CK(cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_exchange_halos(mpcf_solver* s)
{
    Range nvtx("mpcf_exchange_halos");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->links.empty()) return MPCF_OK;
    DeviceGuard g(s->device);
    CK(launch_halo((int)s->esz, s->ddoms, s->dlinks, (int)s->links.size() / 2, s->link_plane, s->parity, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_fill_ghosts(mpcf_solver* s, int dom, void* gx, void* gy, void* gz, int dst_is_device)
{
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!gx || !gy || !gz) return fail(MPCF_ERR_ARG, "null ghost buffer");
    DeviceGuard g(s->device);
    DomDev& D = s->hdoms[dom];
    const size_t sx = 2 * 7 * 3 * (size_t)D.ny * D.nz * s->esz;
    const size_t sy = 2 * 7 * 3 * (size_t)D.nx * D.nz * s->esz;
    const size_t sz = 2 * 7 * 3 * (size_t)D.nx * D.ny * s->esz;
    void *dx = gx, *dy = gy, *dzp = gz;
    void* tmp = nullptr;
    if (!dst_is_device)
    {
        if (cudaMalloc(&tmp, sx + sy + sz) != cudaSuccess) { cudaGetLastError(); return fail(MPCF_ERR_NOMEM, "ghost scratch"); }
        dx = tmp; dy = (char*)tmp + sx; dzp = (char*)tmp + sx + sy;
    }
    cudaError_t e = launch_fill_ghosts(s->esz == 8, s->ddoms + dom, s->parity, dx, dy, dzp, s->stream);
    if (e == cudaSuccess && !dst_is_device)
    {
        e = cudaMemcpyAsync(gx, dx, sx, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(gy, dy, sy, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(gz, dzp, sz, cudaMemcpyDeviceToHost, s->stream);
    }
    cudaError_t e2 = cudaStreamSynchronize(s->stream);
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess) return fail(MPCF_ERR_CUDA, "ghost fill: %s", cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(MPCF_ERR_CUDA, "ghost fill: %s", cudaGetErrorString(e2));
    return MPCF_OK;
}

int mpcf_ic_cloud(mpcf_solver* s, int dom, const mpcf_ic_params* p, int nbubbles, const double* bubbles4)
{
    Range nvtx("mpcf_ic_cloud");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!p || nbubbles < 0 || (nbubbles > 0 && !bubbles4)) return fail(MPCF_ERR_ARG, "bad IC arguments");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    if (nbubbles > s->bubbles_cap)
    {
        if (s->bubbles)
        {
            CK(cudaStreamSynchronize(s->stream));
            cudaFree(s->bubbles);
            s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), (void*)s->bubbles), s->allocs.end());
            s->bubbles = nullptr;
        }
        if ((rc = dev_alloc(s, (void**)&s->bubbles, sizeof(double) * 4 * (size_t)nbubbles))) return rc;
        s->bubbles_cap = nbubbles;
    }
    if (nbubbles > 0) CK(cudaMemcpyAsync(s->bubbles, bubbles4, sizeof(double) * 4 * nbubbles, cudaMemcpyHostToDevice, s->stream));
    IcParams P;
    memcpy(&P, p, sizeof(P));
    CK(launch_ic_cloud(s->esz == 8, s->ddoms + dom, s->parity, P, s->bubbles, nbubbles, s->stream));
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

void mpcf_sic_default_params(mpcf_sic_params* p)
{
    if (!p) return;
    *p = mpcf_sic_params();
    p->rho0 = 1000; p->u0 = 0; p->p0 = 1;
    p->rhoB = 1; p->uB = 0; p->pB = 0.0234;
    p->pressure_ratio = 40;
    p->shock_n[0] = 1; p->shock_n[1] = 0; p->shock_n[2] = 0;
    p->shock_s[0] = 0.05; p->shock_s[1] = 0; p->shock_s[2] = 0;
    p->g1 = 6.59; p->g2 = 1.4; p->pc1 = 4096.0; p->pc2 = 1.0;
    p->eps = 0;
}

static int sic_check(const mpcf_sic_params* p)
{
    if (!p) return fail(MPCF_ERR_ARG, "null SIC parameters");
    const double mag2 = p->shock_n[0] * p->shock_n[0] + p->shock_n[1] * p->shock_n[1] + p->shock_n[2] * p->shock_n[2];
    if (!(mag2 > 0)) return fail(MPCF_ERR_ARG, "shock normal must be non-zero");
    if (!(p->g1 > 1) || !(p->g2 > 1)) return fail(MPCF_ERR_ARG, "gamma must exceed 1");
    if (!(p->rho0 > 0) || !(p->rhoB > 0)) return fail(MPCF_ERR_ARG, "densities must be positive");
    if (!(p->eps >= 0)) return fail(MPCF_ERR_ARG, "eps must be >= 0");
    return MPCF_OK;
}

int mpcf_sic_post_shock(const mpcf_sic_params* p, int precision, double* post4)
{
    int rc = sic_check(p);
    if (rc) return rc;
    if (!post4 || precision < 0 || precision > MPCF_PREC_FP64_FAST) return fail(MPCF_ERR_ARG, "bad arguments");
    SicParams P;
    static_assert(sizeof(SicParams) == sizeof(mpcf_sic_params), "SIC parameter layout");
    memcpy(&P, p, sizeof(P));
    sic_post_shock(precision == MPCF_PREC_FP64 || precision == MPCF_PREC_FP64_FAST, P, post4);
    return MPCF_OK;
}

int mpcf_ic_sic_cloud(mpcf_solver* s, int dom, const mpcf_sic_params* p, int nshapes, const double* shapes4)
{
    Range nvtx("mpcf_ic_sic_cloud");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if ((rc = sic_check(p))) return rc;
    if (nshapes < 0 || (nshapes > 0 && !shapes4)) return fail(MPCF_ERR_ARG, "bad shape arguments");
    for (int i = 0; i < nshapes; ++i)
        if (!(shapes4[4 * i + 3] > 0)) return fail(MPCF_ERR_ARG, "shape %d has a non-positive radius", i);
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    if (nshapes > s->bubbles_cap)
    {
        if (s->bubbles)
        {
            CK(cudaStreamSynchronize(s->stream));
            cudaFree(s->bubbles);
            s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), (void*)s->bubbles), s->allocs.end());
            s->bubbles = nullptr;
        }
        if ((rc = dev_alloc(s, (void**)&s->bubbles, sizeof(double) * 4 * (size_t)nshapes))) return rc;
        s->bubbles_cap = nshapes;
    }
    if (nshapes > 0) CK(cudaMemcpyAsync(s->bubbles, shapes4, sizeof(double) * 4 * nshapes, cudaMemcpyHostToDevice, s->stream));
    SicParams P;
    memcpy(&P, p, sizeof(P));
    const DomDev& D = s->hdoms[dom];
    CK(launch_sic_cloud(s->esz == 8, s->ddoms + dom, D.nx, D.ny, D.nz, s->parity, P, s->bubbles, nshapes, s->stream));
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

void mpcf_case_default_params(mpcf_steady_params* st, mpcf_sod_params* sod, mpcf_sbi_params* sbi)
{
    if (st) { *st = mpcf_steady_params(); st->rho = 1; st->p = 1; st->g = 1.4; }
    if (sod)
    {
        *sod = mpcf_sod_params();
        sod->x0 = 0.5; sod->rho1 = 1; sod->rho2 = 0.125; sod->p1 = 1; sod->p2 = 0.1; sod->g1 = 1.4; sod->g2 = 1.4;
    }
    if (sbi)
    {
        *sbi = mpcf_sbi_params();
        sbi->x0 = 0.1; sbi->mach = 1.22; sbi->rho = 1; sbi->rhobubble = 0.138; sbi->p = 1; sbi->pbubble = 1;
        sbi->g1 = 1.4; sbi->g2 = 1.67; sbi->mollfactor = 1; sbi->axis0 = 0; sbi->axis1 = 1;
    }
}

int mpcf_ic_steady(mpcf_solver* s, int dom, const mpcf_steady_params* p)
{
    Range nvtx("mpcf_ic_steady");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!p || !(p->g > 1) || !(p->rho > 0)) return fail(MPCF_ERR_ARG, "bad SteadyState parameters");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    SteadyParams P;
    static_assert(sizeof(SteadyParams) == sizeof(mpcf_steady_params), "parameter layout");
    memcpy(&P, p, sizeof(P));
    CK(launch_ic_steady(s->esz == 8, s->ddoms + dom, s->parity, P, s->stream));
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_ic_sod(mpcf_solver* s, int dom, const mpcf_sod_params* p)
{
    Range nvtx("mpcf_ic_sod");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!p || p->axis < 0 || p->axis > 2 || !(p->g1 > 1) || !(p->g2 > 1) || !(p->rho1 > 0) || !(p->rho2 > 0))
        return fail(MPCF_ERR_ARG, "bad Sod parameters");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    SodParams P;
    static_assert(sizeof(SodParams) == sizeof(mpcf_sod_params), "parameter layout");
    memcpy(&P, p, sizeof(P));
    CK(launch_ic_sod(s->esz == 8, s->ddoms + dom, s->parity, P, s->stream));
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_ic_sbi(mpcf_solver* s, int dom, const mpcf_sbi_params* p, int nbubbles, const double* bubbles4)
{
    Range nvtx("mpcf_ic_sbi");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!p || p->axis0 < 0 || p->axis0 > 2 || p->axis1 < 0 || p->axis1 > 2 || p->axis0 == p->axis1 ||
        !(p->g1 > 1) || !(p->g2 > 1) || !(p->mach >= 1) || p->mollfactor < 1)
        return fail(MPCF_ERR_ARG, "bad 2DSBI parameters");
    if (nbubbles < 0 || (nbubbles > 0 && !bubbles4)) return fail(MPCF_ERR_ARG, "bad bubble arguments");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    if (nbubbles > s->bubbles_cap)
    {
        if (s->bubbles)
        {
            CK(cudaStreamSynchronize(s->stream));
            cudaFree(s->bubbles);
            s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), (void*)s->bubbles), s->allocs.end());
            s->bubbles = nullptr;
        }
        if ((rc = dev_alloc(s, (void**)&s->bubbles, sizeof(double) * 4 * (size_t)nbubbles))) return rc;
        s->bubbles_cap = nbubbles;
    }
    if (nbubbles > 0) CK(cudaMemcpyAsync(s->bubbles, bubbles4, sizeof(double) * 4 * nbubbles, cudaMemcpyHostToDevice, s->stream));
    SbiParams P;
    static_assert(sizeof(SbiParams) == sizeof(mpcf_sbi_params), "parameter layout");
    memcpy(&P, p, sizeof(P));
    const DomDev& D = s->hdoms[dom];
    // h of the global domain (the bubble interface width)
    CK(launch_ic_sbi(s->esz == 8, s->ddoms + dom, D.gdim[0], D.gdim[1], D.gdim[2], s->parity, P, s->bubbles, nbubbles, s->stream));
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

// ---------------------------------------------------------------------------
// Output and restart (the reference's _dump / _save / _restart,
// Sim_SteadyStateMPI.cpp:138-180, with the arrays of HDF5Dumper_MPI.h).
// The interleaved array moves in z-chunks of at most kIoChunk bytes through
// one device buffer and one pinned host buffer.
// ---------------------------------------------------------------------------
static const size_t kIoChunk = 64u << 20;

// op(host chunk, bytes, byte offset of the chunk in the whole array)
typedef std::function<int(void*, size_t, size_t)> IoOp;

static int io_run(mpcf_solver* s, int dom, int kind, bool to_host, const IoOp& op)
{
    const DomDev& D = s->hdoms[dom];
    const int nch = kind == MPCF_DUMP_TENSOR ? 9 : 7;
    const size_t slab = (size_t)D.nx * D.ny * nch * s->esz;
    const int zc = (int)std::max<size_t>(1, std::min<size_t>((size_t)D.nz, kIoChunk / slab));
    void* dbuf = nullptr;
    void* hbuf = nullptr;
    int rc = MPCF_OK;
    if (cudaMalloc(&dbuf, slab * zc) != cudaSuccess) { cudaGetLastError(); return fail(MPCF_ERR_NOMEM, "cannot allocate the %zu B I/O staging buffer", slab * zc); }
    if (cudaMallocHost(&hbuf, slab * zc) != cudaSuccess) { cudaGetLastError(); cudaFree(dbuf); return fail(MPCF_ERR_NOMEM, "cannot allocate the pinned I/O buffer"); }
    for (int z0 = 0; z0 < D.nz && !rc; z0 += zc)
    {
        const int z1 = std::min(D.nz, z0 + zc);
        const size_t bytes = slab * (z1 - z0);
        cudaError_t e = cudaSuccess;
        if (to_host)
        {
            e = launch_pack(s->esz == 8, kind, s->ddoms + dom, s->parity, z0, z1, dbuf, s->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(hbuf, dbuf, bytes, cudaMemcpyDeviceToHost, s->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
            if (e == cudaSuccess) rc = op(hbuf, bytes, slab * z0);
        }
        else
        {
            rc = op(hbuf, bytes, slab * z0);
            if (!rc) e = cudaMemcpyAsync(dbuf, hbuf, bytes, cudaMemcpyHostToDevice, s->stream);
            if (!rc && e == cudaSuccess) e = launch_unpack_save(s->esz == 8, s->ddoms + dom, s->parity, z0, z1, dbuf, s->stream);
            if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        }
        if (e != cudaSuccess) rc = fail(MPCF_ERR_CUDA, "output transfer: %s", cudaGetErrorString(e));
    }
    cudaFreeHost(hbuf);
    cudaFree(dbuf);
    return rc;
}

static std::string join_path(const char* dir, const std::string& name)
{
    std::string d = (dir && dir[0]) ? dir : ".";
    return d + "/" + name;
}

int mpcf_pack(mpcf_solver* s, int dom, int kind, void* host_out)
{
    Range nvtx("mpcf_pack");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!host_out || (kind != MPCF_DUMP_TENSOR && kind != MPCF_DUMP_SAVE)) return fail(MPCF_ERR_ARG, "bad arguments");
    DeviceGuard g(s->device);
    return io_run(s, dom, kind, true, [&](void* h, size_t b, size_t off) {
        memcpy((char*)host_out + off, h, b);
        return MPCF_OK;
    });
}

int mpcf_unpack_save(mpcf_solver* s, int dom, const void* host_in)
{
    Range nvtx("mpcf_unpack_save");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!host_in) return fail(MPCF_ERR_ARG, "null input");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    rc = io_run(s, dom, MPCF_DUMP_SAVE, false, [&](void* h, size_t b, size_t off) {
        memcpy(h, (const char*)host_in + off, b);
        return MPCF_OK;
    });
    s->sums_valid = false;
    return rc;
}

int mpcf_dump(mpcf_solver* s, int dom, int kind, const char* dir, const char* name, int step)
{
    Range nvtx("mpcf_dump");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!name || !name[0] || (kind != MPCF_DUMP_TENSOR && kind != MPCF_DUMP_SAVE)) return fail(MPCF_ERR_ARG, "bad arguments");
    DeviceGuard g(s->device);
    const DomDev& D = s->hdoms[dom];
    const std::string bin = join_path(dir, std::string(name) + ".bin");
    FILE* f = fopen(bin.c_str(), "wb");
    if (!f) return fail(MPCF_ERR_ARG, "cannot open %s for writing", bin.c_str());
    rc = io_run(s, dom, kind, true, [&](void* h, size_t b, size_t) {
        return fwrite(h, 1, b, f) == b ? MPCF_OK : fail(MPCF_ERR_ARG, "short write to %s", bin.c_str());
    });
    if (fclose(f) != 0 && !rc) rc = fail(MPCF_ERR_ARG, "cannot close %s", bin.c_str());
    if (rc) return rc;
    // XDMF wrapper describing the array: node-centred data on a uniform mesh of
    // spacing h with the origin at 0 (the dimensions listed z, y, x, channels)
    const std::string xmf = join_path(dir, std::string(name) + ".xmf");
    FILE* x = fopen(xmf.c_str(), "w");
    if (!x) return fail(MPCF_ERR_ARG, "cannot open %s for writing", xmf.c_str());
    const int nch = kind == MPCF_DUMP_TENSOR ? 9 : 7;
    const char* attr = kind == MPCF_DUMP_TENSOR ? "Tensor" : "Save Data";
    fprintf(x,
            "<?xml version=\"1.0\" ?>\n"
            "<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n"
            "<Xdmf Version=\"2.0\">\n"
            " <Domain>\n"
            "   <Grid GridType=\"Uniform\">\n"
            "     <Time Value=\"%05d\"/>\n"
            "     <Topology TopologyType=\"3DCORECTMesh\" Dimensions=\"%d %d %d\"/>\n"
            "     <Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n"
            "       <DataItem Name=\"Origin\" Dimensions=\"3\" NumberType=\"Float\" Precision=\"4\" Format=\"XML\">\n"
            "        %e %e %e\n"
            "       </DataItem>\n"
            "       <DataItem Name=\"Spacing\" Dimensions=\"3\" NumberType=\"Float\" Precision=\"4\" Format=\"XML\">\n"
            "        %e %e %e\n"
            "       </DataItem>\n"
            "     </Geometry>\n"
            "     <Attribute Name=\"data\" AttributeType=\"%s\" Center=\"Node\">\n"
            "       <DataItem Dimensions=\"%d %d %d %d\" NumberType=\"Float\" Precision=\"%d\" Format=\"Binary\" Endian=\"Little\">\n"
            "        %s.bin\n"
            "       </DataItem>\n"
            "     </Attribute>\n"
            "   </Grid>\n"
            " </Domain>\n"
            "</Xdmf>\n",
            step, D.nz, D.ny, D.nx, 0., 0., 0., D.h, D.h, D.h, attr, D.nz, D.ny, D.nx, nch, (int)s->esz, name);
    if (fclose(x) != 0) return fail(MPCF_ERR_ARG, "cannot close %s", xmf.c_str());
    return MPCF_OK;
}

int mpcf_set_time(mpcf_solver* s, int dom, double t)
{
    int rc = check_dom(s, dom);
    if (rc) return rc;
    DeviceGuard g(s->device);
    CK(cudaMemcpyAsync(s->time + dom, &t, sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_get_time(mpcf_solver* s, int dom, double* t)
{
    int rc = check_dom(s, dom);
    if (rc) return rc;
    if (!t) return fail(MPCF_ERR_ARG, "null output");
    DeviceGuard g(s->device);
    CK(cudaMemcpyAsync(t, s->time + dom, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_save(mpcf_solver* s, int dom, const char* dir, double t, int step, int fcount)
{
    Range nvtx("mpcf_save");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    const std::string info = join_path(dir, "save.info");
    FILE* f = fopen(info.c_str(), "w");
    if (!f) return fail(MPCF_ERR_ARG, "cannot open %s for writing", info.c_str());
    fprintf(f, "%.15g\n%d\n%d\n", t, step, fcount);
    if (fclose(f) != 0) return fail(MPCF_ERR_ARG, "cannot close %s", info.c_str());
    return mpcf_dump(s, dom, MPCF_DUMP_SAVE, dir, "save.data", step);
}

int mpcf_restart(mpcf_solver* s, int dom, const char* dir, double* t, int* step, int* fcount)
{
    Range nvtx("mpcf_restart");
    int rc = check_dom(s, dom);
    if (rc) return rc;
    const std::string info = join_path(dir, "save.info");
    FILE* f = fopen(info.c_str(), "r");
    if (!f) return 0;                                    // nothing to restart from
    double tt = 0;
    int st = 0, fc = 0;
    const int got = fscanf(f, "%lf %d %d", &tt, &st, &fc);
    fclose(f);
    if (got != 3) return fail(MPCF_ERR_ARG, "%s is not a save record", info.c_str());
    const DomDev& D = s->hdoms[dom];
    const size_t want = (size_t)D.nx * D.ny * D.nz * 7 * s->esz;
    const std::string bin = join_path(dir, "save.data.bin");
    FILE* b = fopen(bin.c_str(), "rb");
    if (!b) return fail(MPCF_ERR_ARG, "cannot open %s", bin.c_str());
    fseek(b, 0, SEEK_END);
    const long size = ftell(b);
    fseek(b, 0, SEEK_SET);
    if (size < 0 || (size_t)size != want)
    {
        fclose(b);
        return fail(MPCF_ERR_ARG, "%s holds %ld bytes, the domain needs %zu", bin.c_str(), size, want);
    }
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    rc = io_run(s, dom, MPCF_DUMP_SAVE, false, [&](void* h, size_t n, size_t) {
        return fread(h, 1, n, b) == n ? MPCF_OK : fail(MPCF_ERR_ARG, "short read from %s", bin.c_str());
    });
    fclose(b);
    s->sums_valid = false;
    if (rc) return rc;
    if ((rc = mpcf_set_time(s, dom, tt))) return rc;
    if (t) *t = tt;
    if (step) *step = st;
    if (fcount) *fcount = fc;
    return 1;
}

int mpcf_ic_cloud_host(int nx, int ny, int nz, const mpcf_ic_params* p, int nbubbles,
                       const double* bubbles4, int elem_size, void* const* out7)
{
    if (nx < 1 || ny < 1 || nz < 1 || !p || !out7 || nbubbles < 0 || (nbubbles > 0 && !bubbles4))
        return fail(MPCF_ERR_ARG, "bad IC arguments");
    if (elem_size != 4 && elem_size != 8) return fail(MPCF_ERR_ARG, "elem_size must be 4 or 8");
    for (int q = 0; q < 7; ++q) if (!out7[q]) return fail(MPCF_ERR_ARG, "null output field %d", q);
    IcParams P;
    memcpy(&P, p, sizeof(P));
    const double h = 1.0 / (double)std::max(nx, std::max(ny, nz));
    const long long N = (long long)nx * ny * nz;
    for (long long i = 0; i < N; ++i)
    {
        const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((long long)nx * ny));
        double c[7];
        ic_cell(P, bubbles4, nbubbles, h, ix, iy, iz, (unsigned long long)i, c);
        for (int q = 0; q < 7; ++q)
        {
            if (elem_size == 8) ((double*)out7[q])[i] = c[q];
            else ((float*)out7[q])[i] = (float)c[q];
        }
    }
    return MPCF_OK;
}

int mpcf_bubbles(unsigned long long seed, int n, double rmin, double rmax,
                 const double* lo3, const double* hi3, double gap, int max_tries, double* out4)
{
    if (n < 0 || !lo3 || !hi3 || (n > 0 && !out4) || !(rmin > 0) || rmax < rmin)
        return fail(MPCF_ERR_ARG, "bad bubble arguments");
    std::mt19937_64 rng(seed);
    // explicit 53-bit uniforms: independent of the standard library's
    // distribution implementations
    auto uni = [&](double a, double b) { return a + (b - a) * ((double)(rng() >> 11) * (1.0 / 9007199254740992.0)); };
    int placed = 0;
    const int tries = max_tries > 0 ? max_tries : 100000;
    for (int t = 0; t < tries && placed < n; ++t)
    {
        const double x = uni(lo3[0], hi3[0]), y = uni(lo3[1], hi3[1]), z = uni(lo3[2], hi3[2]);
        const double r = uni(rmin, rmax);
        bool ok = true;
        for (int k = 0; k < placed && ok; ++k)
        {
            const double dx = x - out4[4 * k], dy = y - out4[4 * k + 1], dz = z - out4[4 * k + 2];
            ok = std::sqrt(dx * dx + dy * dy + dz * dz) >= r + out4[4 * k + 3] + gap;
        }
        if (!ok) continue;
        out4[4 * placed] = x; out4[4 * placed + 1] = y; out4[4 * placed + 2] = z; out4[4 * placed + 3] = r;
        ++placed;
    }
    return placed;
}

int mpcf_set_tiling(mpcf_solver* s, int ty, int dz, int flags)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (!valid_ty(s, ty)) return fail(MPCF_ERR_ARG, "unsupported tile height ty=%d for this precision", ty);
    if (dz < 1) return fail(MPCF_ERR_ARG, "dz must be >= 1");
    if (flags & ~(MPCF_TILE_PERSISTENT | MPCF_TILE_TMA)) return fail(MPCF_ERR_ARG, "unknown tiling flags 0x%x", flags);
    DeviceGuard g(s->device);
    s->ty = ty;
    s->dz = dz;
    s->persist = (flags & MPCF_TILE_PERSISTENT) != 0;
    s->tma = (flags & MPCF_TILE_TMA) != 0;
    return apply_tiling(s);
}

int mpcf_set_test_flags(mpcf_solver* s, unsigned flags)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (flags & ~(unsigned)(MPCF_TEST_DROP_LAST_COPY | MPCF_TEST_DROP_MID_COPY))
        return fail(MPCF_ERR_ARG, "unknown test flags 0x%x", flags);
    static_assert((unsigned)MPCF_TEST_DROP_LAST_COPY == (unsigned)TEST_DROP_LAST_COPY, "test flag");
    static_assert((unsigned)MPCF_TEST_DROP_MID_COPY == (unsigned)TEST_DROP_MID_COPY, "test flag");
    s->test_flags = flags;
    destroy_graphs(s);   // captured launches carry the old flags
    return MPCF_OK;
}

int mpcf_test_copy_count(mpcf_solver* s, unsigned* count, int clear)
{
    if (!s || !count) return fail(MPCF_ERR_ARG, "null argument");
    DeviceGuard g(s->device);
    CK(cudaMemcpyAsync(s->host_stage, s->counter + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
    if (clear) CK(cudaMemsetAsync(s->counter + 1, 0, sizeof(unsigned), s->stream));
    CK(cudaStreamSynchronize(s->stream));
    *count = *(unsigned*)s->host_stage;
    return MPCF_OK;
}

int mpcf_set_weno_order(mpcf_solver* s, int order)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (order != 5 && order != 3) return fail(MPCF_ERR_ARG, "reconstruction order %d: 5 or 3", order);
    if (order == 3 && s->pol != MPCF_PREC_FP32_REF && s->pol != MPCF_PREC_FP64)
        return fail(MPCF_ERR_ARG, "WENO3 is built for the reference-rounding forms (MPCF_PREC_FP32_REF, MPCF_PREC_FP64)");
    DeviceGuard g(s->device);
    CK(cudaStreamSynchronize(s->stream));
    const bool was = s->weno3;
    s->weno3 = order == 3;
    int rc = grant_shared_memory(s);
    if (rc) { s->weno3 = was; return rc; }
    destroy_graphs(s);    // captured launches are of the other kernel
    return MPCF_OK;
}

int mpcf_get_weno_order(const mpcf_solver* s)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    return s->weno3 ? 3 : 5;
}

int mpcf_get_tiling(const mpcf_solver* s, int* ty, int* dz, int* flags)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (ty) *ty = s->ty;
    if (dz) *dz = s->dz;
    if (flags) *flags = (s->persist ? MPCF_TILE_PERSISTENT : 0) | (s->tma ? MPCF_TILE_TMA : 0);
    return MPCF_OK;
}

int mpcf_launch_shape(const mpcf_solver* s, long long* ntiles, long long* grid, int* threads)
{
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (ntiles) *ntiles = s->ntiles;
    if (grid) *grid = s->persist ? persistent_grid(const_cast<mpcf_solver*>(s), s->ty) : s->ntiles;
    if (threads) *threads = stage_block_threads(s->ty);
    return MPCF_OK;
}

int mpcf_time_stages(mpcf_solver* s, int reps, double dtinvh, double* ms_per_stage)
{
    Range nvtx("mpcf_time_stages");
    if (!s || reps < 1) return fail(MPCF_ERR_ARG, "bad arguments");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    std::vector<double> dv(s->ndom, dtinvh);
    CK(cudaStreamSynchronize(s->stream));
    for (int d = 0; d < s->ndom; ++d)
    {
        if (s->esz == 8) ((double*)s->host_stage)[d] = dtinvh;
        else ((float*)s->host_stage)[d] = (float)dtinvh;
    }
    CK(cudaMemcpyAsync(s->dtinvh, s->host_stage, s->esz * s->ndom, cudaMemcpyHostToDevice, s->stream));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int rc = MPCF_OK;
    CK(cudaEventRecord(e0, s->stream));
    for (int r = 0; r < reps && !rc; ++r) rc = enqueue_stage(s, kLSRK3[r % 3][0], kLSRK3[r % 3][1], false);
    CK(cudaEventRecord(e1, s->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (ms_per_stage) *ms_per_stage = ms / reps;
    return MPCF_OK;
}

// z-chunk depths the autotuner tries for tile height ty: 16, 32, 64 and 128
// below the deepest domain, and the whole depth.  When 16-deep chunks do not
// fill one wave of resident CTAs (small domains), also the shallowest depth
// whose CTAs still fit in one wave, and 8: a CTA walks its chunk slab by
// slab, so there the chunk depth is the latency of the stage (64^3, mixed:
// 4-deep chunks of 32x8 tiles, 256 CTAs, run a step 1.9x faster than the
// best 16-deep tiling).
static std::vector<int> dz_candidates(mpcf_solver* s, int ty, int maxn, bool tma)
{
    auto tiles = [&](int dz)
    {
        long long t = 0;
        for (auto& D : s->hdoms) t += (long long)((D.nx + 31) / 32) * ((D.ny + ty - 1) / ty) * ((D.nz + dz - 1) / dz);
        return t;
    };
    std::vector<int> dzs;
    for (int v : {16, 32, 64, 128}) if (v < maxn) dzs.push_back(v);
    dzs.push_back(maxn);
    const StageKernelInfo I = stage_info(s, ty, false, false, tma);
    int nb = 0;
    if (!I.fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, I.fn, stage_block_threads(ty), I.smem) != cudaSuccess || nb < 1)
    {
        cudaGetLastError();
        nb = 1;
    }
    const long long slots = (long long)nb * s->num_sms;
    if (maxn > 4 && tiles(std::min(16, maxn)) < slots)
    {
        int fit = 0;
        for (int dz = 4; dz < 16 && dz < maxn && !fit; ++dz) if (tiles(dz) <= slots) fit = dz;
        if (fit) dzs.push_back(fit);
        if (fit != 8 && 8 < maxn) dzs.push_back(8);
    }
    std::sort(dzs.begin(), dzs.end());
    dzs.erase(std::unique(dzs.begin(), dzs.end()), dzs.end());
    return dzs;
}

int mpcf_autotune(mpcf_solver* s, int reps, int* best3, double* best_ms)
{
    Range nvtx("mpcf_autotune");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    if (s->win_nch) return window_only(s, "mpcf_autotune");
    if (reps < 1) reps = 3;
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    CK(cudaStreamSynchronize(s->stream));
    // Trials read the current state and write the other state buffer; the
    // register is redirected to a scratch copy so the solver's state is
    // unchanged afterwards.
    std::vector<void*> saved_R(s->ndom);
    std::vector<void*> scratch(s->ndom, nullptr);
    int rc = MPCF_OK;
    for (int d = 0; d < s->ndom && !rc; ++d)
    {
        DomDev& D = s->hdoms[d];
        const size_t bytes = (size_t)7 * D.fs * s->esz;
        if (cudaMalloc(&scratch[d], bytes) != cudaSuccess) { cudaGetLastError(); rc = fail(MPCF_ERR_NOMEM, "autotune scratch"); break; }
        saved_R[d] = D.R;
    }
    const int saved_ty = s->ty, saved_dz = s->dz, saved_p = s->persist, saved_m = s->tma, saved_parity = s->parity;
    std::vector<char> saved_dtinvh(s->esz * s->ndom);
    CK(cudaMemcpy(saved_dtinvh.data(), s->dtinvh, saved_dtinvh.size(), cudaMemcpyDeviceToHost));
    int bty = saved_ty, bdz = saved_dz, bp = saved_p, bm = saved_m;
    double bms = 1e300;
    const bool can_tma = any_tma_ok(s);
    if (!rc)
    {
        int maxn = 0;
        for (auto& D : s->hdoms) maxn = std::max(maxn, D.nz);
        const int tys[4] = {3, 7, 8, 15};
        for (int i = 0; i < 4 && !rc; ++i)
        {
            if (!valid_ty(s, tys[i])) continue;
            for (int dz : dz_candidates(s, tys[i], maxn, can_tma))
            {
                for (int f = 0; f < 4 && !rc; ++f)
                {
                    const int p = f & 1, m = (f >> 1) & 1;
                    if (m && !can_tma) continue;
                    s->ty = tys[i]; s->dz = dz; s->persist = p; s->tma = m;
                    for (int d = 0; d < s->ndom; ++d)
                    {
                        s->hdoms[d].R = scratch[d];
                        cudaMemcpyAsync(scratch[d], saved_R[d], (size_t)7 * s->hdoms[d].fs * s->esz, cudaMemcpyDeviceToDevice, s->stream);
                    }
                    if ((rc = apply_tiling(s))) break;
                    double ms = 0;
                    // one warm-up launch, then the timed ones; parity is reset
                    // so every trial reads the same state
                    s->parity = saved_parity;
                    if ((rc = mpcf_time_stages(s, 1, 0.0, &ms))) break;
                    s->parity = saved_parity;
                    double tot = 0;
                    for (int r = 0; r < reps && !rc; ++r)
                    {
                        rc = mpcf_time_stages(s, 1, 0.0, &ms);
                        s->parity = saved_parity;
                        tot += ms;
                    }
                    if (!rc && tot / reps < bms) { bms = tot / reps; bty = tys[i]; bdz = dz; bp = p; bm = m; }
                }
            }
        }
    }
    for (int d = 0; d < s->ndom; ++d) if (saved_R[d]) s->hdoms[d].R = saved_R[d];
    s->parity = saved_parity;
    s->ty = rc ? saved_ty : bty;
    s->dz = rc ? saved_dz : bdz;
    s->persist = rc ? saved_p : bp;
    s->tma = rc ? saved_m : bm;
    int rc2 = apply_tiling(s);
    for (void* p : scratch) if (p) cudaFree(p);
    if (cudaMemcpy(s->dtinvh, saved_dtinvh.data(), saved_dtinvh.size(), cudaMemcpyHostToDevice) != cudaSuccess && !rc2)
        rc2 = fail(MPCF_ERR_CUDA, "restoring dt/h after autotune failed");
    if (rc) return rc;
    if (rc2) return rc2;
    if (best3) { best3[0] = s->ty; best3[1] = s->dz; best3[2] = (s->persist ? MPCF_TILE_PERSISTENT : 0) | (s->tma ? MPCF_TILE_TMA : 0); }
    if (best_ms) *best_ms = bms;
    return MPCF_OK;
}

int mpcf_probe_fp32_peak(int device, double* tflops)
{
    if (!tflops) return fail(MPCF_ERR_ARG, "null output");
    DeviceGuard g(device);
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float* out = nullptr;
    CK(cudaMalloc(&out, 16));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int blocks = sms * 8, iters = 4096;
    double best = 0;
    for (int r = 0; r < 4; ++r)
    {
        CK(cudaEventRecord(e0, 0));
        CK(launch_fma_probe(blocks, iters, out, 0));
        CK(cudaEventRecord(e1, 0));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        // 8 chains x 16 FMA x iters per thread, 2 flops per FMA
        const double flops = 2.0 * 8 * 16 * (double)iters * 256.0 * blocks;
        if (r > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = best;
    return MPCF_OK;
}

int mpcf_time_run(mpcf_solver* s, int nsteps, double cfl, double dt_max, double* ms)
{
    Range nvtx("mpcf_time_run");
    if (!s || nsteps < 1 || !ms) return fail(MPCF_ERR_ARG, "bad arguments");
    DeviceGuard g(s->device);
    int rc = mpcf_run(s, 0, cfl, dt_max, 1, nullptr);   // builds the graphs
    if (rc) return rc;
    if (!s->sos_fresh && (rc = enqueue_sos(s))) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s->stream));
    for (int n = 0; n < nsteps; ++n)
    {
        CK(cudaGraphLaunch(s->graph[s->parity], s->stream));
        s->parity ^= 1;
    }
    s->sos_fresh = true;
    CK(cudaEventRecord(e1, s->stream));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->sums_valid = s->track_cons;
    *ms = t;
    return MPCF_OK;
}

int mpcf_update(mpcf_solver* s, double b)
{
    Range nvtx("mpcf_update");
    if (!s) return fail(MPCF_ERR_ARG, "null solver");
    DeviceGuard g(s->device);
    s->sos_fresh = false;                   // the state (or the accumulator) changes
    CK(launch_update(s->esz == 8, s->ddoms, s->ndom, s->parity, b, s->stream));
    s->parity ^= 1;
    s->sums_valid = false;
    CK(cudaStreamSynchronize(s->stream));
    return MPCF_OK;
}

int mpcf_device_info(int device, char* name, int name_len, long long* total_bytes, long long* free_bytes, int* sms)
{
    DeviceGuard g(device);
    cudaDeviceProp p;
    CK(cudaGetDeviceProperties(&p, device));
    if (name && name_len > 0) { strncpy(name, p.name, (size_t)name_len - 1); name[name_len - 1] = 0; }
    if (sms) *sms = p.multiProcessorCount;
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    if (total_bytes) *total_bytes = (long long)tot;
    if (free_bytes) *free_bytes = (long long)fr;
    return MPCF_OK;
}

int mpcf_device_synchronize(int device)
{
    DeviceGuard g(device);
    CK(cudaDeviceSynchronize());
    return MPCF_OK;
}

} // extern "C"
