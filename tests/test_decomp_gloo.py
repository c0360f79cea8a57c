"""z-slab decomposition on CPU: the host side of mpcf.decomp -- slab
extents, face conditions, the point-to-point exchange of the 3 boundary
planes and the dt reduction over ranks -- run by a world_size-2 (and 3)
gloo group.  Each rank advances its slab with the CPU oracle on the slab
extended by its ghost planes; the gathered result equals the oracle's run
of the undivided domain bit for bit (no GPU involved)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import mpcf.decomp as dc
from mpcf import BC_HALO

ABS, REF = 0, 1


def test_slab_extents_and_faces():
    assert dc.slab_extents(30, 3) == [(0, 10), (10, 10), (20, 10)]
    assert dc.slab_extents(31, 4) == [(0, 8), (8, 8), (16, 8), (24, 7)]
    assert dc.slab_extents(7, 1) == [(0, 7)]
    with pytest.raises(ValueError):
        dc.slab_extents(8, 3)                     # a slab of 2 planes cannot fill 3 ghost planes
    bc = (ABS, REF, REF, ABS, REF, ABS)
    assert dc.slab_bc(bc, 0, 3) == (ABS, REF, REF, ABS, REF, BC_HALO)
    assert dc.slab_bc(bc, 1, 3) == (ABS, REF, REF, ABS, BC_HALO, BC_HALO)
    assert dc.slab_bc(bc, 2, 3) == (ABS, REF, REF, ABS, BC_HALO, ABS)
    assert dc.slab_bc(bc, 0, 1) == bc
    assert dc.global_spacing((40, 24, 30)) == 1.0 / 40


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


DIMS = (24, 20, 18)
BC = (ABS, REF, ABS, ABS, REF, ABS)
STEPS = 2


def _initial_state():
    from conftest import cloud_state
    return [np.array(a) for a in cloud_state(DIMS, nb=3)]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import oracle_lib as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        NX, NY, NZ = DIMS
        plane = NX * NY
        ext = dc.slab_extents(NZ, world)
        z0, nz = ext[rank]
        lo = dc.HALO if rank > 0 else 0
        hi = dc.HALO if rank < world - 1 else 0
        U0 = _initial_state()
        # the slab with its ghost planes as one extended block of planes
        U = [np.ascontiguousarray(f[(z0 - lo) * plane:(z0 + nz + hi) * plane]) for f in U0]
        R = [np.zeros_like(f) for f in U]
        ext_dims = (NX, NY, nz + lo + hi)
        # faces of the extended block: the slab's own where it meets the
        # domain boundary; beyond ghost planes any condition will do, it only
        # reaches the ghost planes' own (discarded) results
        bc = tuple(ABS if c == BC_HALO else c for c in dc.slab_bc(BC, rank, world))
        h = dc.global_spacing(DIMS)
        t = torch.from_numpy

        def blocks():
            send_lo = [t(f[lo * plane:(lo + dc.HALO) * plane]) for f in U]
            send_hi = [t(f[(lo + nz - dc.HALO) * plane:(lo + nz) * plane]) for f in U]
            recv_lo = [t(f[:lo * plane]) for f in U] if lo else []
            recv_hi = [t(f[(lo + nz) * plane:]) for f in U] if hi else []
            return send_lo, send_hi, recv_lo, recv_hi

        dts = []
        for _ in range(STEPS):
            sos = O.max_sos([np.ascontiguousarray(f[lo * plane:(lo + nz) * plane]) for f in U])
            dt = dc.global_dt(dist, sos, 0.3, h)
            dts.append(dt)
            for a, b in ((0.0, 1.0 / 4), (-17.0 / 32, 8.0 / 9), (-32.0 / 27, 3.0 / 4)):
                dc.exchange_planes(dist, rank, world, *blocks())
                O.stage(ext_dims, bc, U, R, a, b, dt / h)
        out[rank] = (dts, [f[lo * plane:(lo + nz) * plane].copy() for f in U],
                     [f[lo * plane:(lo + nz) * plane].copy() for f in R])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_over_gloo_match_undivided_domain(world):
    import oracle_lib as O
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    U = _initial_state()
    R = [np.zeros_like(f) for f in U]
    dts = [O.step(DIMS, BC, U, R, cfl=0.3)[0] for _ in range(STEPS)]
    for r in range(world):
        assert out[r][0] == dts, (r, out[r][0], dts)
    for q in range(7):
        got_u = np.concatenate([out[r][1][q] for r in range(world)])
        got_r = np.concatenate([out[r][2][q] for r in range(world)])
        assert np.array_equal(got_u, U[q]), q
        assert np.array_equal(got_r, R[q]), q
