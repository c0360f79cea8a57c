/*
 * mpcf_b200.h -- C ABI of libmpcf_b200, the B200 (sm_100a) implementation of
 * the CUBISM-MPCF per-step hot path: WENO5/HLLC convection in x/y/z, the
 * low-storage LSRK3 stage update and the maximum-speed-of-sound CFL
 * reduction, for the 7-field stiffened-gas two-phase system.
 *
 * Plain C: opaque handle, raw pointers and sizes, int status returns (0 on
 * success, a negative MPCF_ERR_* code otherwise; mpcf_last_error() gives
 * the message of the calling thread's last failure).  No allocation or CUDA
 * type appears in a signature.
 *
 * Data layout (reference: source/NodeBlock.h:26-36,110-117, Types.h:31):
 *   a state or register is 7 arrays (rho, rho*u, rho*v, rho*w, E,
 *   G = 1/(gamma-1), P = gamma*pc/(gamma-1)) of nx*ny*nz elements, cell
 *   (ix,iy,iz) at ix + nx*(iy + ny*iz).  Element type: float for the
 *   MPCF_PREC_FP32_REF, MPCF_PREC_FP32 and MPCF_PREC_MIXED precisions,
 *   double for MPCF_PREC_FP64 and MPCF_PREC_FP64_FAST.
 * Boundary conditions, per domain, 6 ints in the order
 *   x-left, x-right, y-left, y-right, z-left, z-right
 *   (MPCF_BC_ABSORBING / MPCF_BC_REFLECTING, BoundaryConditions.h:60-109;
 *   MPCF_BC_HALO on z faces of slabs, see the decomposition section).
 *
 * Threading: one host thread per solver at a time.  All work of a solver is
 * ordered on its own CUDA stream; calls that return host data synchronise it.
 */
#ifndef MPCF_B200_H
#define MPCF_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define MPCF_API_VERSION 1

typedef struct mpcf_solver mpcf_solver;

/* precisions */
#define MPCF_PREC_FP32_REF 0  /* FP32, rounding of the reference source (bit-exact to the CPU restatement) */
#define MPCF_PREC_FP32     1  /* FP32, fast weights / division, fused multiply-add */
#define MPCF_PREC_MIXED    2  /* fast FP32 + compensated (two-sum) FP32 pressure recovery + FP64 conservation sums */
#define MPCF_PREC_FP64     3  /* all FP64, rounding order of the reference source */
#define MPCF_PREC_FP64_FAST 4 /* all FP64 with the fast forms' factored algebra and refined reciprocals */

/* boundary conditions */
#define MPCF_BC_ABSORBING  0
#define MPCF_BC_REFLECTING 1
#define MPCF_BC_HALO       2   /* z faces only: ghost planes filled from a neighbouring slab */

/* status codes */
#define MPCF_OK            0
#define MPCF_ERR_ARG      -1   /* invalid argument */
#define MPCF_ERR_CUDA     -2   /* CUDA runtime error (message has the CUDA error string) */
#define MPCF_ERR_NOMEM    -3   /* device or host allocation failed */
#define MPCF_ERR_STATE    -4   /* call not valid in the solver's state */
#define MPCF_ERR_NUMERIC  -5   /* the device error word reports a non-physical state */

/* bits of the device error word */
#define MPCF_ERRBIT_NONPHYSICAL  1u  /* rho<=0, E<=0, G<=0 or non-finite after an update */
#define MPCF_ERRBIT_SOS          2u  /* maximum speed of sound not finite or not positive */
#define MPCF_ERRBIT_TMA_TIMEOUT  4u  /* a bulk tensor copy did not complete within the wait limit */
#define MPCF_ERRBIT_BOUNDS       8u  /* bounds-checking build (libmpcf_b200_check.so): a stage-kernel index
                                        left its buffer; it was clamped into it and the results are void */
#define MPCF_ERRBIT_TMA_INFLIGHT 16u /* after a bulk-copy wait ran out, a CTA's bounded wait for its own
                                       copies still in flight ran out as well */

/* stage-kernel tiling flags (mpcf_set_tiling / mpcf_get_tiling / mpcf_autotune) */
#define MPCF_TILE_PERSISTENT 1  /* one CTA per resident slot pulling tiles from a work counter */
#define MPCF_TILE_TMA        2  /* stage slabs with bulk tensor copies (domains with nx*elem % 16 == 0) */

/* Bubble-cloud initial condition (liquid with gas bubbles; indicator
 * alpha = 0.5*(1 - tanh(phi/(width*h))), phi = distance to the nearest
 * bubble surface; velocity noise uniform in [-noise, noise] from a
 * counter-based hash of (seed, cell, component)). */
typedef struct mpcf_ic_params
{
    double rho_l, p_l, gamma_l, pc_l;   /* liquid */
    double rho_g, p_g, gamma_g, pc_g;   /* gas */
    double noise;                       /* velocity noise amplitude */
    double width;                       /* interface width in cells */
    unsigned long long seed;
} mpcf_ic_params;

/* ---- version / errors --------------------------------------------------- */
int         mpcf_version(void);
const char* mpcf_last_error(void);
int         mpcf_elem_size(int precision);   /* 4 or 8, or MPCF_ERR_ARG */

/* ---- lifetime ----------------------------------------------------------- *
 * Replaces GPU::alloc / GPU::dealloc (source/GPU/GPU.h:48-49,
 * GPUhousehold.cu:81-254) and the GPUlab constructor's device set-up
 * (GPUlab.cpp:25-71).  ndomains >= 1 independent domains of sizes
 * dims[3*d..3*d+2] (each >= 5 in x and y, >= 3 in z, as the reference's
 * GPUkernels.cu:18-24 and BoundaryConditions.h mirrors require); bc may be
 * NULL (all absorbing).  h[d] = 1/max(nx,ny,nz) (NodeBlock.h:71).  The
 * solver owns all device memory: two state buffers (ping-pong), the
 * register and the per-domain scalars. */
int mpcf_create(mpcf_solver** out, int ndomains, const int* dims, const int* bc,
                int precision, int device);
int mpcf_destroy(mpcf_solver* s);
int mpcf_num_domains(const mpcf_solver* s);
int mpcf_precision(const mpcf_solver* s);

/* ---- state transfer ----------------------------------------------------- *
 * Replaces the per-stage PCIe staging of GPUlab (h2d_3DArray, h2d_tmp,
 * d2h_rhs, d2h_tmp: GPU.h:52-56, GPUhousehold.cu:260-334).  state7/reg7 are
 * 7 pointers each, host memory unless *_is_device is set; reg7 may be NULL
 * (set: register cleared; get: register not copied). */
int mpcf_set_state(mpcf_solver* s, int dom, const void* const* state7, const void* const* reg7, int src_is_device);
int mpcf_get_state(mpcf_solver* s, int dom, void* const* state7, void* const* reg7, int dst_is_device);
/* current device addresses of the state and register fields (valid until the
 * next stage, which swaps the state buffers) */
int mpcf_device_pointers(mpcf_solver* s, int dom, void** state7, void** reg7);

/* ---- the hot path --------------------------------------------------------- *
 * mpcf_max_sos: GPUlab::max_sos (GPUlab.cpp:647-700) + _maxSOS
 *   (GPUkernels.cu:1182-1222) / MaxSpeedOfSound_CUDA::compute
 *   (MaxSpeedOfSound_CUDA.cpp:13-18).  sos[d] per domain.
 * mpcf_stage: GPUlab::process_all(a, b, dtinvh) (GPUlab.cpp:703-793), i.e.
 *   ghosts/BCs + Convection_CUDA(a, dtinvh).compute + Update_CUDA(b).compute
 *   (Convection_CUDA.cpp:15-23, Update_CUDA.cpp:12-17): R <- a*R - dtinvh*L(U),
 *   U <- U + b*R.  dtinvh[d] per domain (NULL: use the device dt/h of the
 *   last mpcf_step / mpcf_compute_dt).
 * mpcf_compute_dt: max speed of sound and dt = min(cfl*h/sos, dt_max) on the
 *   device (LSRK3_IntegratorMPI.cpp:31-38), no host round trip.
 * mpcf_step: one LSRK3 step (LSRK3_IntegratorMPI.cpp:27-62): device dt, then
 *   the three stages (a,b) = (0,1/4), (-17/32,8/9), (-32/27,3/4).  dt_out[d]
 *   (optional) receives dt (synchronises).
 * mpcf_run: nsteps steps; use_graph replays a captured CUDA graph of the
 *   whole step.  time_out[d] (optional) receives the accumulated time. */
int mpcf_max_sos(mpcf_solver* s, double* sos);
int mpcf_stage(mpcf_solver* s, double a, double b, const double* dtinvh);
int mpcf_compute_dt(mpcf_solver* s, double cfl, double dt_max, double* dt_out);
int mpcf_step(mpcf_solver* s, double cfl, double dt_max, double* dt_out);
int mpcf_run(mpcf_solver* s, int nsteps, double cfl, double dt_max, int use_graph, double* time_out);
/* nsteps LSRK3 steps of a state that lives in host memory: the reference's
 * host-resident block streamed through the GPU (GPUlab::process_all's
 * chunked, double-buffered PCIe transfers on three streams,
 * GPUlab.cpp:202-372,703-793, under LSRK3_IntegratorMPI::operator(),
 * LSRK3_IntegratorMPI.cpp:27-62).  host7: the 7 fields of the single domain
 * (x fastest), read as every step's input and overwritten with every step's
 * result; page-locked memory lets the copies overlap the kernels.  Every
 * step uploads the state in z-chunks of whole tile layers on one copy
 * stream and runs the three stages as a wavefront over the chunks: a stage
 * of a chunk runs once the stage before it (stage 1: the upload) has
 * covered every chunk within 3 planes above, and each chunk of the new
 * state goes back on a second copy stream as soon as stage 3 has written
 * it; the next step's upload of a chunk follows its download (copies in
 * both directions overlap each other and the kernels).  The first step's dt
 * comes from the sound speed reduced chunk by chunk as the chunks land;
 * later steps take the sound speed that stage 3 accumulated over the state
 * it wrote (the values the host receives and sends back), as mpcf_run does.
 * nchunks: requested chunks (at most the tile layers, nz/dz; one layer per
 * chunk with the tiling's dz).  The register stays on the device (stage 1
 * multiplies it by a = 0).  Results are bit-identical to mpcf_run on the
 * same state.  Single-domain solvers without halo faces; conservation
 * tracking is not applied.  time_out (optional): the time. */
int mpcf_run_host(mpcf_solver* s, int nsteps, double cfl, double dt_max, void* const* host7, int nchunks,
                  double* time_out);
/* Windowed runs: a domain held in host memory that may be larger than the
 * device's, streamed through a few device slots in z-chunks of nslices
 * planes (the reference's GPUlab with nslices < sizeZ: chunks of nslices
 * planes with 3-plane overlaps streamed through the GPU every stage,
 * GPUlab.cpp:37-41 (nslices must divide sizeZ), 202-372, 703-793).
 * mpcf_create_window: a solver of min(nslots, nz/nslices) slots, each an
 *   nx*ny*nslices domain with 3 stored ghost planes on each z side (device
 *   memory of a slot: 3 buffers of nx*ny*(nslices+6) cells of 7 fields);
 *   bc6: the domain's faces (absorbing or reflecting; null: absorbing).
 *   nslices >= 3 must divide nz; nslots >= min(5, nz/nslices): a stage 3 of
 *   chunk c needs chunks c-1 .. c+3 resident.  Only mpcf_run_window advances
 *   it (the stepping calls and mpcf_link_z return MPCF_ERR_STATE);
 *   set_tiling applies to the slots.
 * mpcf_run_window: nsteps LSRK3 steps of host7 (7 fields of nx*ny*nz, x
 *   fastest; page-locked memory lets copies overlap), overwritten with each
 *   step's result.  The chunks of successive steps take the slots in turn
 *   (chunk c of step n: slot (n*chunks + c) % nslots): each chunk's upload, the
 *   three stages as a wavefront over the chunks (a stage of chunk c runs once
 *   the stage before it covers chunk c+1; before each stage a kernel fills
 *   the slot's ghost planes from the neighbouring slots, or by the boundary
 *   condition at the domain's z faces), and its download, on two copy
 *   streams and the solver's stream.  The first step's dt comes from a pass
 *   that streams every chunk through the slots, from the last down, and
 *   reduces its sound speed (the first step reuses the chunks it leaves);
 *   later steps take what stage 3 accumulated.  Results are bit-identical
 *   to mpcf_run of the whole domain on one device.  time_out (optional): the
 *   time.
 * mpcf_window_info: {nz, nslices, chunks, slots} of a windowed solver.
 * mpcf_window_plan: the operations of a windowed run in enqueue order (no
 *   device work): ops4[4 i .. 4 i + 3] = {kind (0 upload, 1 sound speed of
 *   the first step's input, 2 dt, 3 stage, 4 download), step (-1: the
 *   sound-speed pass), stage (0..2), chunk}, at most cap entries written;
 *   returns the number of operations, or MPCF_ERR_ARG when the slots are
 *   too few. */
int mpcf_create_window(mpcf_solver** out, int nx, int ny, int nz, int nslices, int nslots, int precision,
                       const int* bc6, int device);
int mpcf_run_window(mpcf_solver* s, int nsteps, double cfl, double dt_max, void* const* host7, double* time_out);
int mpcf_window_info(const mpcf_solver* s, int* info4);
/* One stage, or the maximum sound speed, of a windowed block whose state and
 * register both live in host memory: the reference's process_all and
 * max_sos over nslices chunks (GPUlab.cpp:647-700,703-793), for the shim's
 * GPUlab when the block does not fit on the device.
 * mpcf_window_stage: state7 and reg7 (7 fields of nx*ny*nz each) are read
 *   and overwritten chunk by chunk: rhs = a*R - dtinvh*L(U) into reg7,
 *   U + b*rhs into state7, bit-identical to mpcf_stage on the whole block.
 *   Each chunk's state and register go up, its ghost planes come from the
 *   neighbouring slots (or the z boundary condition), the stage runs once
 *   the chunk above is there, and both come back, on two copy streams.
 * mpcf_window_max_sos: the largest sound speed of state7 (streamed through
 *   the slots), NaN if any cell's is not real and finite.
 * mpcf_set_bc on a windowed solver (dom 0) sets the block's six faces. */
int mpcf_window_stage(mpcf_solver* s, double a, double b, double dtinvh, void* const* state7, void* const* reg7);
int mpcf_window_max_sos(mpcf_solver* s, const void* const* state7, double* sos);
int mpcf_window_plan(int nchunks, int nslots, int nsteps, int* ops4, int cap);
/* The operations of one mpcf_window_stage in enqueue order (no device
 * work), in mpcf_window_plan's format: kinds 0 upload (state and register),
 * 3 stage, 4 download; step and stage 0. */
int mpcf_window_stage_plan(int nchunks, int nslots, int* ops4, int cap);
int mpcf_synchronize(mpcf_solver* s);
/* Stream-ordered building blocks of a step, for a driver that orders its
 * own work with the solver's kernels: the reference's per-rank step with
 * its MPI MIN of dt (LSRK3_IntegratorMPI.cpp:27-62, :40) and its halo
 * exchange before every stage (GPUlab::load_ghosts, GPUlab.cpp:622-644),
 * run without host round trips (an NCCL all-reduce and point-to-point
 * copies on the solver's stream between these calls).  None of them
 * synchronises.
 * mpcf_stream: the solver's cudaStream_t (every kernel of the solver runs
 *   on it).
 * mpcf_sos_accumulator: device address of the per-domain sound-speed
 *   accumulator, ndom values of the state's type (float, or double for the
 *   FP64 forms); it holds non-negative values, so a caller may reduce it
 *   further in place (an all-reduce MAX over ranks) before mpcf_enqueue_dt.
 * mpcf_enqueue_sos: the maximum sound speed of every domain's current state
 *   into the accumulator (cleared first).
 * mpcf_enqueue_dt: dt = min(cfl h/sos, dt_max) and dt/h per domain on the
 *   device from the accumulator, which it clears.
 * mpcf_enqueue_stage: one stage with the device dt/h: mpcf_stage without
 *   its final synchronisation. */
int mpcf_stream(mpcf_solver* s, void** stream);
int mpcf_sos_accumulator(mpcf_solver* s, void** dev_ptr);
int mpcf_enqueue_sos(mpcf_solver* s);
int mpcf_enqueue_dt(mpcf_solver* s, double cfl, double dt_max);
int mpcf_enqueue_stage(mpcf_solver* s, double a, double b);
/* The state update alone, U <- U + b*R (Update_CUDA::compute ->
 * GPU::update -> _update, Update_CUDA.cpp:12-17, GPUkernels.cu:1142-1179),
 * for callers that split a stage into Convection_CUDA (mpcf_stage with
 * b = 0) and Update_CUDA; the pair is bit-identical to one mpcf_stage. */
int mpcf_update(mpcf_solver* s, double b);

/* FP64 sums of (rho, rho u, rho v, rho w, E) over each domain's current
 * state, out[5*d..5*d+4]; deterministic order. */
int mpcf_conserved_sums(mpcf_solver* s, double* out);
/* When on, stage 3 of every step accumulates the FP64 sums of the new
 * state inside the stage kernel (no extra pass); mpcf_conserved_sums then
 * returns them without another reduction. */
int mpcf_set_track_conservation(mpcf_solver* s, int on);

/* The same FP64 sums without allocating anything.  This entry point has no
 * counterpart in the reference.  It is for callers that may not allocate
 * device memory, directly or through a library: hosts that give a plug-in a
 * fixed device-memory budget at start-up and forbid cudaMalloc afterwards,
 * and tight loops that cannot afford cudaMalloc/cudaFree, which may
 * synchronise the whole device.  The caller passes device pointers to the 7
 * fields of a state of `ncells` cells (elem_size 4 or 8; only the first five
 * fields are read) and receives rho, rho u, rho v, rho w, E totals in out5,
 * host memory or, with out_is_device, device memory.  Work goes on `stream`
 * (a cudaStream_t, NULL for the default stream); a host output is ready when
 * the call returns.  The result is bit-identical to mpcf_conserved_sums on
 * the same state.
 * Limit: ncells <= 268435456 (8192 chunks of 32768 cells); larger inputs are
 * rejected with MPCF_ERR_ARG.  The partial sums live in a fixed 320 KB
 * device array of this library, which every GPU that loads it keeps until
 * the process exits.  The first call on a device looks up that array's
 * device address, with the device current; make that first call before any
 * stream capture.  The address is kept for the life of the process, so a
 * cudaDeviceReset of that device after the first call is not supported.
 * All calls share the array: calls that overlap on a GPU
 * (concurrent streams or threads) race and must be serialised by the
 * caller.  Every partial a call reads is written by that same call. */
int mpcf_conserved_sums_noalloc(const void* const* state7, long long ncells, int elem_size,
                                double* out5, int out_is_device, int device, void* stream);

/* device error word (MPCF_ERRBIT_*); clear != 0 resets it */
int mpcf_error_word(mpcf_solver* s, unsigned* word, int clear);

/* ---- boundary conditions / ghosts ---------------------------------------- *
 * mpcf_set_bc: change the 6 face conditions of a domain (the per-case
 *   GPUlab::_apply_bc overrides, e.g. Sim_SICCloudMPI.h:312-321).
 * mpcf_fill_ghosts: materialise the ghost layers the stage kernel
 *   synthesises, in the reference's halo layouts (GHOSTMAPX/GHOSTMAPY/ID3,
 *   Types.h:42-52): gx 2*7*3*ny*nz, gy 2*7*nx*3*nz, gz 2*7*nx*ny*3 elements,
 *   ordered [side][field][...]; side 0 = left (layer 0 outermost), side 1 =
 *   right (layer 0 innermost). */
int mpcf_set_bc(mpcf_solver* s, int dom, const int* bc6);
int mpcf_fill_ghosts(mpcf_solver* s, int dom, void* gx, void* gy, void* gz, int dst_is_device);

/* ---- z-slab domain decomposition ------------------------------------------ *
 * The reference spreads a global domain over MPI ranks (GridMPI.h:65-106),
 * refreshes 3-cell halos before every stage (GPUlab::load_ghosts,
 * GPUlab.cpp:622-644) and takes the minimum dt over ranks
 * (LSRK3_IntegratorMPI.cpp:40).  Here a global domain is cut into z-slabs.
 * A slab's z face towards a neighbouring slab is MPCF_BC_HALO (given to
 * mpcf_create; z faces only, fixed for the solver's life): its state buffers
 * then hold 3 ghost planes beyond that face, which the stage reads as stored
 * state.  mpcf_device_pointers returns the address of plane 0 of each field;
 * plane z of field q (-3 <= z < 0 below the slab, nz <= z < nz+3 above it)
 * is at state7[q] + z*nx*ny elements.  Before every stage the ghost planes
 * must hold the current state of the neighbour's boundary planes (planes
 * nz-3..nz-1 of the slab below, planes 0..2 of the slab above).
 *
 * mpcf_link_z: slabs in one solver (one GPU): domain `upper` sits on top of
 *   domain `lower` (same nx and ny, halo faces towards each other).  Every
 *   stage then first copies the boundary planes between linked slabs on the
 *   device (inside the captured step graph too), and linked slabs share one
 *   dt from the largest sound speed among them.  A chain of linked slabs
 *   advances bit-identically to the undivided domain.
 * mpcf_set_spacing: grid spacing h of a domain (default 1/max(nx,ny,nz),
 *   NodeBlock.h:71); a slab takes its global domain's 1/max(NX,NY,NZ).
 * mpcf_exchange_halos: the device copies between linked slabs, on demand
 *   (every stage does them anyway).
 * Slabs on different GPUs exchange through the caller (NCCL send/recv of
 *   the 3-plane blocks, e.g. the Python driver mpcf/decomp.py): per step,
 *   mpcf_max_sos, the maximum over ranks, dt = min(cfl*h/sos, dt_max), then
 *   per stage the exchange and mpcf_stage with dtinvh = dt/h. */
int mpcf_link_z(mpcf_solver* s, int lower, int upper);
int mpcf_set_spacing(mpcf_solver* s, int dom, double h);
int mpcf_exchange_halos(mpcf_solver* s);
/* The domain is the block of cells org3 .. org3 + dims - 1 of a global grid
 * of global3 cells (GridMPI's per-rank block offset): the initial-condition
 * generators (mpcf_ic_cloud, mpcf_ic_sic_cloud, mpcf_ic_steady, mpcf_ic_sod,
 * mpcf_ic_sbi) then write the global domain's values of these cells, so
 * slabs set up on their own GPUs equal the slices of the undivided domain's
 * initial condition.  Default: origin 0, global = the domain.  The spacing
 * is set separately (mpcf_set_spacing). */
int mpcf_set_origin(mpcf_solver* s, int dom, const int* org3, const int* global3);

/* ---- initial conditions --------------------------------------------------- */
/* device generator: state of domain dom from the cloud IC, register cleared */
int mpcf_ic_cloud(mpcf_solver* s, int dom, const mpcf_ic_params* p, int nbubbles, const double* bubbles4);
/* host generator of the same IC (elem_size 4 or 8): 7 host arrays */
int mpcf_ic_cloud_host(int nx, int ny, int nz, const mpcf_ic_params* p, int nbubbles,
                       const double* bubbles4, int elem_size, void* const* out7);
/* Seeded rejection sampling of non-overlapping spheres (std::mt19937_64):
 * centres uniform in [lo[i], hi[i]], radii uniform in [rmin, rmax], at least
 * `gap` apart surface to surface.  Writes up to n (x,y,z,r) quadruples and
 * returns how many were placed (>= 0) or an error code. */
int mpcf_bubbles(unsigned long long seed, int n, double rmin, double rmax,
                 const double* lo3, const double* hi3, double gap, int max_tries, double* out4);

/* ---- shock-induced cloud collapse ----------------------------------------- *
 * The reference's Sim_SICCloudMPI initial condition (replaces
 * Sim_SICCloudMPI::_ic, Sim_SICCloudMPI.cpp:43-132 and _ic_quad, :339-357):
 * a planar shock with Johnsen's post-shock liquid state behind it (the side
 * where n.(x - s) <= 0), a cloud of spheres of gas ahead of it, and every
 * cell set to the 3x3x3 Simpson average of the sampled mixture (samples at
 * the cell centre and its faces).  Fields use the state's precision with the
 * reference's rounding (FP32 bit-identical to the reference's
 * _FLOAT_PRECISION_ build); the register is cleared.  shapes4 holds
 * nshapes (x, y, z, radius) spheres, the lines of the reference's cloud.dat,
 * rounded once to the state's precision.  eps is SimTools::EPSILON: 0 (the
 * reference's SICCloud setting) gives a sharp interface, eps > 0 a cosine
 * ramp of half-width eps.  mpcf_sic_default_params gives the reference's
 * option defaults (Sim_SICCloudMPI.cpp:52-76); mpcf_sic_post_shock returns
 * rho1, u1, p1 and the shock Mach number as that precision computes them
 * (precision = MPCF_PREC_*). */
typedef struct
{
    double rho0, u0, p0;            /* pre-shock liquid        -rho0 -u0 -p0 */
    double rhoB, uB, pB;            /* bubble gas              -rhoB -uB -pB */
    double pressure_ratio;          /* p1/p0 across the shock  -pressureratio */
    double shock_n[3];              /* shock normal            -shockNx -shockNy -shockNz */
    double shock_s[3];              /* point on the shock      -shockSx -shockSy -shockSz */
    double g1, g2, pc1, pc2;        /* liquid / gas            -g1 -g2 -pc1 -pc2 */
    double eps;                     /* SimTools::EPSILON */
} mpcf_sic_params;
void mpcf_sic_default_params(mpcf_sic_params* p);
int mpcf_sic_post_shock(const mpcf_sic_params* p, int precision, double* post4);
int mpcf_ic_sic_cloud(mpcf_solver* s, int dom, const mpcf_sic_params* p, int nshapes, const double* shapes4);

/* ---- the reference's other cases ----------------------------------------- *
 * Initial conditions of Sim_SteadyStateMPI (a uniform state;
 * Sim_SteadyStateMPI.cpp:95-135), Sim_SodMPI (a two-state tube along `axis`;
 * Sim_SodMPI.cpp:20-95) and Sim_2DSBIMPI (a planar shock of Mach number
 * `mach` along axis0 hitting cylinders of gas with axes along the third
 * direction, positions in the axis0/axis1 plane, interface mollified over
 * mollfactor*sqrt(3)*h; Sim_2DSBIMPI.cpp:15-233), with the reference's
 * rounding (FP32 bit-identical to its _FLOAT_PRECISION_ build, except the
 * mollified 2DSBI interface, where CUDA's cosf may differ from the C
 * library's by one unit in the last place).  Axes: 0 = x, 1 = y, 2 = z; the
 * reference's -config strings map to (axis0, axis1) = "xy" (0,1), "xz" (0,2),
 * "yx" (1,0), "yz" (1,2), "zx" (2,0), "zy" (2,1).  bubbles4: (x, y, z, r) per
 * cylinder, the lines of the reference's <config>bubbles.dat.  The register is
 * cleared.  The boundary conditions of the cases' labs are: SteadyState
 * reflecting on all faces, Sod absorbing, 2DSBI reflecting on the axis1 faces
 * and absorbing on the others (GPUlab2DSBI_*reflect); set them with
 * mpcf_set_bc.  mpcf_case_default_params fills any non-NULL argument with the
 * reference's option defaults. */
typedef struct { double rho, u, v, w, p, g, pc; } mpcf_steady_params;      /* -rho -u -v -w -p -g -pc */
typedef struct
{
    double x0, rho1, rho2, u1, u2, p1, p2, g1, g2, pc1, pc2;   /* -x0 -rho1 -rho2 -u1 -u2 -p1 -p2 -g1 -g2 -pc1 -pc2 */
    int reverse, axis;                                          /* -reverse, -config x|y|z */
} mpcf_sod_params;
typedef struct
{
    double x0, mach, rho, rhobubble, u, p, pbubble, g1, g2, pc1, pc2;  /* -x0 -mach -rho -rhobubble -u -p -pbubble -g1 -g2 -pc1 -pc2 */
    int reverse, mollfactor, axis0, axis1;                             /* -reverse -mollfactor -config */
} mpcf_sbi_params;
void mpcf_case_default_params(mpcf_steady_params* steady, mpcf_sod_params* sod, mpcf_sbi_params* sbi);
int mpcf_ic_steady(mpcf_solver* s, int dom, const mpcf_steady_params* p);
int mpcf_ic_sod(mpcf_solver* s, int dom, const mpcf_sod_params* p);
int mpcf_ic_sbi(mpcf_solver* s, int dom, const mpcf_sbi_params* p, int nbubbles, const double* bubbles4);

/* ---- output and restart --------------------------------------------------- *
 * The arrays of the reference's dump and save (replaces
 * Sim_SteadyStateMPI::_dump/_save/_restart, Sim_SteadyStateMPI.cpp:138-180,
 * with DumpHDF5_MPI / ReadHDF5_MPI, IO/HDF5Dumper_MPI.h:30-260): one array of
 * nz x ny x nx cells x channels (channels fastest, then x, y, z) in the
 * state's precision, filled as the reference's streamers fill it
 * (Types.h:192-277):
 *   MPCF_DUMP_TENSOR  9 channels: rho, u, v, w, p, G, P, 0, 0 (_dump)
 *   MPCF_DUMP_SAVE    7 channels: the conserved fields (_save, restart)
 * mpcf_pack copies the array into host memory (for a caller's own writer,
 * e.g. HDF5); mpcf_unpack_save loads a MPCF_DUMP_SAVE array back into the
 * state (register cleared).
 * mpcf_dump writes <dir>/<name>.bin (the array, little-endian, no header) and
 * <dir>/<name>.xmf, the reference's XDMF description with the data item
 * pointing at the raw file (Format="Binary") where the reference points at
 * its HDF5 dataset; readers of XDMF (ParaView, VisIt) open it as is.
 * mpcf_save writes <dir>/save.info (t with 15 significant digits, step,
 * fcount: one per line, as _save does) and the MPCF_DUMP_SAVE array as
 * <dir>/save.data.{bin,xmf}.  mpcf_restart reads them back into the state,
 * sets the domain's time to t and returns 1, or returns 0 when there is no
 * <dir>/save.info (as _restart returns false).  The reference keeps save.info
 * in the working directory and the data under -fpath; here both are in dir.
 * mpcf_set_time / mpcf_get_time: the domain's accumulated time. */
#define MPCF_DUMP_TENSOR 0
#define MPCF_DUMP_SAVE   1
int mpcf_pack(mpcf_solver* s, int dom, int kind, void* host_out);
int mpcf_unpack_save(mpcf_solver* s, int dom, const void* host_in);
int mpcf_dump(mpcf_solver* s, int dom, int kind, const char* dir, const char* name, int step);
int mpcf_save(mpcf_solver* s, int dom, const char* dir, double t, int step, int fcount);
int mpcf_restart(mpcf_solver* s, int dom, const char* dir, double* t, int* step, int* fcount);
int mpcf_set_time(mpcf_solver* s, int dom, double t);
int mpcf_get_time(mpcf_solver* s, int dom, double* t);

/* ---- launch configuration ------------------------------------------------- *
 * tile = 32 x ty columns x dz slabs (ty 3, 7 or 8; 15 also for
 * MPCF_PREC_FP32_REF), one CTA per tile of 32*(ty+1) threads for ty = 3, 7,
 * 15 (a helper warp evaluates the tile's extra faces) and 32*ty for ty = 8;
 * flags = MPCF_TILE_PERSISTENT | MPCF_TILE_TMA.  With MPCF_TILE_TMA, domains
 * whose rows are multiples of 16 bytes stage their slabs with bulk tensor
 * copies (other domains keep ordinary loads).  mpcf_autotune times the
 * candidates on the solver's own state (which it leaves unchanged) and
 * keeps the fastest; best3 (optional) = {ty, dz, flags}, best_ms (optional)
 * = stage time. */
/* Reconstruction order of the stage: 5 (WENO5, the default) or 3, the
 * reference's compile-time WENO3 build (-D_WENO3_, GPUonly.cuh:102-137,
 * 141-176: two-stencil weights (1/3, 2/3) on the squared neighbour
 * differences, the same clipping).  WENO3 is provided for the two
 * reference-rounding forms, MPCF_PREC_FP32_REF (bit-identical to the
 * reference's WENO3 arithmetic) and MPCF_PREC_FP64; other forms are
 * rejected with MPCF_ERR_ARG.  mpcf_get_weno_order returns 5 or 3. */
int mpcf_set_weno_order(mpcf_solver* s, int order);
int mpcf_get_weno_order(const mpcf_solver* s);
int mpcf_set_tiling(mpcf_solver* s, int ty, int dz, int flags);
int mpcf_get_tiling(const mpcf_solver* s, int* ty, int* dz, int* flags);
int mpcf_autotune(mpcf_solver* s, int reps, int* best3, double* best_ms);

/* Failure-detection tests only.  It replaces no reference interface: the
 * reference ignores CUDA return codes (GPUhousehold.cu) and has no device
 * failure detection.  MPCF_TEST_DROP_LAST_COPY makes a
 * non-persistent stage launch with bulk-copy staging arm the mbarrier of the
 * last copy of each z-chunk without issuing the copy: the CTA's final bounded
 * wait runs out (2^18 polls, about 1.3 s), MPCF_ERRBIT_TMA_TIMEOUT is set, no copy is
 * left in flight and the context stays usable.  MPCF_TEST_DROP_MID_COPY drops
 * the chunk's first copy after the prologue instead: the wait runs out one
 * slab in, the CTA issues no further copy, waits (bounded) for the copy it
 * issued with the dropped one, and exits with none in flight (a drain wait
 * that also ran out would set MPCF_ERRBIT_TMA_INFLIGHT).  Persistent launches
 * ignore both.  0 (the default) turns them off. */
#define MPCF_TEST_DROP_LAST_COPY 1u
#define MPCF_TEST_DROP_MID_COPY  2u
int mpcf_set_test_flags(mpcf_solver* s, unsigned flags);
/* Failure-detection tests only: bulk copies the stage kernel issued while a
 * test flag was set (clear != 0 resets the count).  No reference
 * counterpart. */
int mpcf_test_copy_count(mpcf_solver* s, unsigned* count, int clear);

/* number of tiles one stage launch processes, and of stage-kernel CTAs */
int mpcf_launch_shape(const mpcf_solver* s, long long* ntiles, long long* grid, int* threads);

/* Time `reps` stage launches of the current configuration with CUDA events on
 * the solver's stream (state advances; use on throw-away data). */
int mpcf_time_stages(mpcf_solver* s, int reps, double dtinvh, double* ms_per_stage);

/* Replay nsteps captured step graphs back to back and return their device
 * time (CUDA events on the solver's stream), ms. */
int mpcf_time_run(mpcf_solver* s, int nsteps, double cfl, double dt_max, double* ms);

/* Device facts for host code that does not link the CUDA runtime itself
 * (GPU::tell_GPU / tell_memUsage_GPU of the reference, GPUhousehold.cu:390-418):
 * name (optional), total and free memory, SM count. */
int mpcf_device_info(int device, char* name, int name_len, long long* total_bytes, long long* free_bytes, int* sms);
/* Wait for all work on a device (GPU::syncGPU, GPUhousehold.cu:367-372). */
int mpcf_device_synchronize(int device);

/* Measured FP32 CUDA-core throughput of the device (FMA chains), TFLOP/s:
 * the denominator of the stage kernel's compute roofline. */
int mpcf_probe_fp32_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* MPCF_B200_H */
