"""z-slab decomposition of one global domain.

The reference spreads a domain over MPI ranks as a Cartesian grid of blocks
(source/GridMPI.h:65-106), refreshes 3-cell halos before every stage
(GPUlab::load_ghosts, source/GPUlab.cpp:622-644) and advances every rank with
the minimum dt over the ranks (MPI_Allreduce(MIN),
source/LSRK3_IntegratorMPI.cpp:40).  Here the domain is cut along z only:
a slab's z face towards a neighbouring slab is a halo face (BC_HALO) whose 3
ghost planes are stored state, refreshed from the neighbour before every
stage.  Two drivers share the plan:

Each slab carries its place in the global grid (mpcf_set_origin), so the
device initial-condition generators write the global domain's values of its
cells: a rank sets up its own slab without the global state.

* ``slab_solver``: all slabs in one Solver on one GPU.  The library links
  them (mpcf_link_z), copies the ghost planes on the device at the start of
  every stage and gives the linked slabs one dt; steps, runs and CUDA graphs
  work unchanged.
* ``SlabRank``: one slab per process and GPU.  Ghost planes travel with
  torch.distributed point-to-point operations (NCCL over NVLink between
  GPUs), dt comes from the maximum sound speed over the ranks.

Either way the slabs advance bit-identically to the undivided domain: every
cell sees the same stencil values and the same dt.

Global arrays are flat in the reference's order, x fastest then y then z
(cell (ix, iy, iz) at ix + NX*(iy + NY*iz)), so slab r is the contiguous
range of planes [z0, z0 + nz) of every field.
"""
import math

import numpy as np

from . import _lib
from ._lib import BC_ABSORBING, BC_HALO, MpcfError
from .solver import Solver, LSRK3

HALO = 3   # ghost planes of a halo face (the WENO5 stencil half-width)


def slab_extents(nz, nslabs):
    """(z0, nz_r) of each of `nslabs` contiguous z-slabs of `nz` planes; sizes
    differ by at most one (the larger slabs first) and are at least 3
    planes, so a slab can fill its neighbour's 3 ghost planes."""
    if nslabs < 1:
        raise ValueError("nslabs must be >= 1")
    base, extra = divmod(int(nz), int(nslabs))
    if base < HALO:
        raise ValueError(f"{nz} planes cannot make {nslabs} slabs of at least {HALO} planes")
    out, z0 = [], 0
    for r in range(nslabs):
        n = base + (1 if r < extra else 0)
        out.append((z0, n))
        z0 += n
    return out


def slab_bc(bc6, rank, nslabs):
    """Face conditions of slab `rank`: the global domain's x and y faces, its
    z faces where the slab touches the domain boundary, BC_HALO towards a
    neighbouring slab."""
    b = list(bc6 if bc6 is not None else (BC_ABSORBING,) * 6)
    if rank > 0:
        b[4] = BC_HALO
    if rank < nslabs - 1:
        b[5] = BC_HALO
    return tuple(b)


def global_spacing(global_dims):
    """Grid spacing of the global domain, 1/max(NX, NY, NZ) (NodeBlock.h:71)."""
    return 1.0 / max(int(v) for v in global_dims)


# ---------------------------------------------------------------------------
# all slabs on one GPU
# ---------------------------------------------------------------------------
def slab_solver(global_dims, nslabs, bc=None, precision="fp32_ref", device=0):
    """A Solver holding `nslabs` linked z-slabs of the domain `global_dims`
    (domain r = slab r, bottom to top); returns (solver, extents)."""
    NX, NY, NZ = (int(v) for v in global_dims)
    ext = slab_extents(NZ, nslabs)
    dims = [(NX, NY, n) for _, n in ext]
    bcs = [slab_bc(bc, r, nslabs) for r in range(nslabs)]
    s = Solver(dims, bc=bcs, precision=precision, device=device)
    try:
        h = global_spacing(global_dims)
        for r, (z0, _) in enumerate(ext):
            s.set_spacing(h, dom=r)
            s.set_origin((0, 0, z0), (NX, NY, NZ), dom=r)
        for r in range(nslabs - 1):
            s.link_z(r, r + 1)
    except Exception:
        s.close()
        raise
    return s, ext


def slab_of(field, global_dims, z0, nz):
    """Planes [z0, z0+nz) of a flat global field (a view)."""
    NX, NY, _ = global_dims
    plane = int(NX) * int(NY)
    return np.asarray(field).reshape(-1)[z0 * plane:(z0 + nz) * plane]


def scatter_state(solver, global_dims, ext, state, reg=None):
    """Upload a global state (and register) into the slabs of `solver`."""
    for r, (z0, n) in enumerate(ext):
        U = [np.ascontiguousarray(slab_of(f, global_dims, z0, n)) for f in state]
        R = None if reg is None else [np.ascontiguousarray(slab_of(f, global_dims, z0, n)) for f in reg]
        solver.set_state(U, R, dom=r)


def gather_state(solver, ext, with_reg=True):
    """The global state (and register) from the slabs of `solver`."""
    parts = [solver.get_state(dom=r, with_reg=with_reg) for r in range(len(ext))]
    if with_reg:
        U = [np.concatenate([p[0][q] for p in parts]) for q in range(7)]
        R = [np.concatenate([p[1][q] for p in parts]) for q in range(7)]
        return U, R
    return [np.concatenate([p[q] for p in parts]) for q in range(7)]


# ---------------------------------------------------------------------------
# one slab per rank
# ---------------------------------------------------------------------------
def exchange_planes(dist, rank, nranks, send_lo, send_hi, recv_lo, recv_hi, group=None):
    """Point-to-point exchange of 3-plane blocks with the z neighbours (the
    halo traffic of GPUlab::load_ghosts between ranks): `send_lo` (planes
    0..2) goes to rank-1, `send_hi` (planes nz-3..nz-1) to rank+1; `recv_lo`
    (ghost planes below) comes from rank-1, `recv_hi` (above) from rank+1.
    Each is a list of 7 tensors, one per field: device tensors for NCCL,
    host tensors for gloo.  Returns when every transfer has completed."""
    ops = []
    if rank > 0:
        ops += [dist.P2POp(dist.isend, t, rank - 1, group) for t in send_lo]
        ops += [dist.P2POp(dist.irecv, t, rank - 1, group) for t in recv_lo]
    if rank < nranks - 1:
        ops += [dist.P2POp(dist.isend, t, rank + 1, group) for t in send_hi]
        ops += [dist.P2POp(dist.irecv, t, rank + 1, group) for t in recv_hi]
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def global_dt(dist, sos_local, cfl, h, dt_max=1e30, device=None, group=None):
    """dt of every rank: min(cfl*h/sos, dt_max) with sos the maximum sound
    speed over the ranks, evaluated in the order of the device dt kernel (so
    one rank gives the dt of mpcf_step bit for bit).  The reference's minimum
    over ranks of cfl*h/sos_r is the same number."""
    import torch
    t = torch.tensor([float(sos_local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    sos = float(t.item())
    dt = cfl * h / sos if sos > 0 else float("nan")
    dt = dt_max if dt_max < dt else dt
    if not (sos > 0) or dt != dt or math.isinf(dt):
        raise MpcfError(_lib.ERR_NUMERIC, f"maximum sound speed {sos!r} gives no finite dt")
    return dt


class _DeviceBlock:
    """A raw device range seen by torch through __cuda_array_interface__."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


class SlabRank:
    """This process's z-slab of a global domain, on its own GPU.

    ``dist`` is torch.distributed with an initialised process group (NCCL
    for GPU ranks); rank r owns slab r of ``slab_extents(NZ, world_size)``.
    Each stage first exchanges the 3 boundary planes of the current state
    with the neighbours, then runs mpcf_stage; each step takes dt from the
    maximum sound speed over the ranks."""

    def __init__(self, global_dims, bc=None, precision="fp32_ref", dist=None, device=None, group=None,
                 rank=None, nranks=None):
        if device is None:
            # one GPU per rank: the device the rank made current (with
            # torch.cuda.set_device(LOCAL_RANK)) before joining the group
            import torch
            device = torch.cuda.current_device()
        self.global_dims = tuple(int(v) for v in global_dims)
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group) if rank is None else int(rank)
        self.nranks = dist.get_world_size(group) if nranks is None else int(nranks)
        NX, NY, NZ = self.global_dims
        self.ext = slab_extents(NZ, self.nranks)
        self.z0, self.nz = self.ext[self.rank]
        self.h = global_spacing(self.global_dims)
        self.solver = Solver([(NX, NY, self.nz)], bc=[slab_bc(bc, self.rank, self.nranks)],
                             precision=precision, device=device)
        self.solver.set_spacing(self.h)
        self.solver.set_origin((0, 0, self.z0), self.global_dims)
        self.device = device
        self.time = 0.0
        self._typestr = "<f8" if self.solver.dtype == np.float64 else "<f4"
        self._esz = 8 if self.solver.dtype == np.float64 else 4

    def close(self):
        self.solver.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # state of this slab from / into global arrays
    def set_global_state(self, state, reg=None):
        U = [np.ascontiguousarray(slab_of(f, self.global_dims, self.z0, self.nz)) for f in state]
        R = None if reg is None else [np.ascontiguousarray(slab_of(f, self.global_dims, self.z0, self.nz)) for f in reg]
        self.solver.set_state(U, R)

    def get_state(self, with_reg=True):
        return self.solver.get_state(with_reg=with_reg)

    def plane_blocks(self):
        """torch views of (send_lo, send_hi, recv_lo, recv_hi) of the current
        state buffer, 7 fields each (the buffer alternates every stage)."""
        import torch
        NX, NY, _ = self.global_dims
        plane = NX * NY
        n = HALO * plane
        st, _ = self.solver.device_pointers()
        dev = torch.device("cuda", self.device)

        def view(ptr, first_plane):
            return torch.as_tensor(_DeviceBlock(ptr + first_plane * plane * self._esz, n, self._typestr), device=dev)

        send_lo = [view(p, 0) for p in st]
        send_hi = [view(p, self.nz - HALO) for p in st]
        recv_lo = [view(p, -HALO) for p in st] if self.rank > 0 else []
        recv_hi = [view(p, self.nz) for p in st] if self.rank < self.nranks - 1 else []
        return send_lo, send_hi, recv_lo, recv_hi

    def exchange(self):
        """Refresh the ghost planes of the current state from the neighbours."""
        import torch
        if self.nranks == 1:
            return
        self.solver.synchronize()                 # the previous stage has written the planes
        exchange_planes(self.dist, self.rank, self.nranks, *self.plane_blocks(), group=self.group)
        torch.cuda.synchronize(self.device)       # the ghost planes have landed

    def step(self, cfl=0.3, dt_max=1e30):
        """One LSRK3 step of the global domain (LSRK3_IntegratorMPI.cpp:27-62);
        returns dt."""
        import torch
        sos = self.solver.max_sos()[0]
        dt = global_dt(self.dist, sos, cfl, self.h, dt_max, device=torch.device("cuda", self.device),
                       group=self.group)
        dtinvh = dt / self.h
        for a, b in LSRK3:
            self.exchange()
            self.solver.stage(a, b, [dtinvh])
        self.time += dt
        return dt

    def enqueue_step(self, cfl=0.3, dt_max=1e30):
        """One LSRK3 step ordered on the solver's stream, with no host round
        trip: the sound speed into the solver's device accumulator, an
        all-reduce MAX of it over the ranks, the device dt, and per stage the
        exchange of the ghost planes (NCCL point-to-point copies that start
        after the stage that wrote the planes; the next stage waits for them
        on the stream, not on the host) and the stage.  Bit-identical to
        step(), which synchronises four times per step.  A state without a
        real sound speed is flagged in the error word of the rank that holds
        it (the device dt kernel's check)."""
        import torch
        dev = torch.device("cuda", self.device)
        stream = torch.cuda.ExternalStream(self.solver.stream_handle(), device=dev)
        with torch.cuda.stream(stream):
            self.solver.enqueue_sos()
            acc = torch.as_tensor(_DeviceBlock(self.solver.sos_accumulator(), 1, self._typestr), device=dev)
            self.dist.all_reduce(acc, op=self.dist.ReduceOp.MAX, group=self.group)
            self.solver.enqueue_dt(cfl, dt_max)
            for a, b in LSRK3:
                if self.nranks > 1:
                    exchange_planes(self.dist, self.rank, self.nranks, *self.plane_blocks(), group=self.group)
                self.solver.enqueue_stage(a, b)

    def run(self, nsteps, cfl=0.3, dt_max=1e30, ordered=False):
        """nsteps steps; ordered: every step stream-ordered (enqueue_step),
        with one synchronisation at the end.  Returns the time."""
        if not ordered:
            for _ in range(int(nsteps)):
                self.step(cfl, dt_max)
            return self.time
        t0 = self.solver.get_time()
        for _ in range(int(nsteps)):
            self.enqueue_step(cfl, dt_max)
        self.solver.synchronize()
        self.time += self.solver.get_time() - t0
        return self.time
