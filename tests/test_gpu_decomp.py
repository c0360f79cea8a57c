"""z-slab decomposition on the GPU: linked slabs of one solver (ghost planes
copied on the device inside every stage, one dt for the group) and the
per-rank driver's halo views, both bit-identical to the undivided domain."""
import numpy as np
import pytest

import mpcf.decomp as dc
from conftest import cloud_state
from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu

ABS, REF = 0, 1
DIMS = (40, 24, 30)
BC = (ABS, REF, ABS, ABS, REF, ABS)


def _state(prec, mpcf):
    dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    return [np.asarray(a, dtype=dt) for a in cloud_state(DIMS, nb=3)]


def _undivided(mpcf, prec, U0, steps, graph, tiling=None):
    with mpcf.Solver([DIMS], bc=[BC], precision=prec) as s:
        if tiling:
            s.set_tiling(*tiling)
        s.set_state(U0)
        t = s.run(steps, cfl=0.3, graph=graph)
        return t, s.get_state()


@pytest.mark.parametrize("prec", ["fp32_ref", "mixed", "fp64"])
@pytest.mark.parametrize("nslabs,graph", [(2, True), (3, False), (4, True)])
def test_linked_slabs_match_undivided_domain(mpcf, prec, nslabs, graph):
    U0 = _state(prec, mpcf)
    t_ref, (U_ref, R_ref) = _undivided(mpcf, prec, U0, 3, graph)
    s, ext = dc.slab_solver(DIMS, nslabs, bc=BC, precision=prec)
    with s:
        dc.scatter_state(s, DIMS, ext, U0)
        t = s.run(3, cfl=0.3, graph=graph)
        U, R = dc.gather_state(s, ext)
        assert s.error_word() == 0
    assert list(t) == [t_ref[0]] * nslabs, (t, t_ref)
    assert_bitwise(U, U_ref, f"state, {nslabs} slabs")
    assert_bitwise(R, R_ref, f"register, {nslabs} slabs")


@pytest.mark.parametrize("tiling", [(3, 4, False, False), (7, 64, True, True), (8, 5, True, True), (8, 64, False, False)])
def test_linked_slabs_every_tiling(mpcf, tiling):
    """Ghost planes are read by the bulk-copy staging and the ordinary loads
    alike (rows of 40 floats qualify for bulk copies), with chunks that
    start and end next to a ghost plane."""
    prec = "mixed"
    U0 = _state(prec, mpcf)
    t_ref, (U_ref, R_ref) = _undivided(mpcf, prec, U0, 2, True, tiling)
    s, ext = dc.slab_solver(DIMS, 3, bc=BC, precision=prec)
    with s:
        s.set_tiling(*tiling)
        dc.scatter_state(s, DIMS, ext, U0)
        s.run(2, cfl=0.3, graph=True)
        U, R = dc.gather_state(s, ext)
    assert_bitwise(U, U_ref, f"state, tiling {tiling}")
    assert_bitwise(R, R_ref, f"register, tiling {tiling}")


def test_halo_faces_are_validated(mpcf):
    with pytest.raises(mpcf.MpcfError):
        mpcf.Solver([(16, 16, 8)], bc=[(mpcf.BC_HALO, ABS, ABS, ABS, ABS, ABS)])   # x faces cannot be halos
    with mpcf.Solver([(16, 16, 8), (16, 16, 8), (16, 12, 8)],
                     bc=[(ABS,) * 5 + (mpcf.BC_HALO,), (ABS,) * 4 + (mpcf.BC_HALO, ABS),
                         (ABS,) * 4 + (mpcf.BC_HALO, ABS)]) as s:
        with pytest.raises(mpcf.MpcfError):
            s.link_z(1, 0)                  # domain 1's upper face is not a halo face
        with pytest.raises(mpcf.MpcfError):
            s.link_z(0, 2)                  # x-y sizes differ
        with pytest.raises(mpcf.MpcfError):
            s.set_bc((ABS,) * 6, dom=0)     # halo faces are fixed
        s.link_z(0, 1)
        with pytest.raises(mpcf.MpcfError):
            s.link_z(0, 1)                  # already linked
        with pytest.raises(mpcf.MpcfError):
            s.set_origin((0, 0, 9), (16, 16, 16), dom=0)     # planes 9..16 past the global extent
        with pytest.raises(mpcf.MpcfError):
            s.set_origin((0, -1, 0), (16, 16, 16), dom=0)    # negative origin
        with pytest.raises(mpcf.MpcfError):
            s.set_spacing(0.0, dom=0)                         # spacing must be positive
        s.set_origin((0, 0, 8), (16, 16, 16), dom=1)


def test_rank_driver_halo_views(mpcf):
    """Two SlabRank slabs in one process, their ghost planes filled through
    the driver's torch views of the device buffers (as NCCL would fill them),
    stage by stage with the undivided domain's dt: bit-identical."""
    import torch
    prec = "fp32_ref"
    U0 = _state(prec, mpcf)
    h = dc.global_spacing(DIMS)
    ranks = [dc.SlabRank(DIMS, bc=BC, precision=prec, rank=r, nranks=2) for r in range(2)]
    try:
        for r in ranks:
            r.set_global_state(U0)
        with mpcf.Solver([DIMS], bc=[BC], precision=prec) as ref:
            ref.set_state(U0)
            for _ in range(2):
                sos = max(r.solver.max_sos()[0] for r in ranks)
                assert sos == ref.max_sos()[0]
                dt = min(0.3 * h / sos, 1e30)
                for a, b in mpcf.LSRK3:
                    lo, hi = ranks[0].plane_blocks(), ranks[1].plane_blocks()
                    for q in range(7):
                        hi[2][q].copy_(lo[1][q])          # rank 1's lower ghosts <- rank 0's top planes
                        lo[3][q].copy_(hi[0][q])          # rank 0's upper ghosts <- rank 1's bottom planes
                    torch.cuda.synchronize()
                    for r in ranks:
                        r.solver.stage(a, b, [dt / h])
                    ref.stage(a, b, [dt / h])
            U_ref, R_ref = ref.get_state()
        parts = [r.get_state() for r in ranks]
        U = [np.concatenate([p[0][q] for p in parts]) for q in range(7)]
        R = [np.concatenate([p[1][q] for p in parts]) for q in range(7)]
        assert_bitwise(U, U_ref, "state")
        assert_bitwise(R, R_ref, "register")
    finally:
        for r in ranks:
            r.close()


def test_single_rank_driver_matches_step(mpcf):
    """The rank driver's host dt (maximum over a one-rank NCCL group) and
    per-stage calls reproduce mpcf_step bit for bit."""
    import datetime
    import os
    import socket
    import torch.distributed as dist
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        prec = "mixed"
        U0 = _state(prec, mpcf)
        with dc.SlabRank(DIMS, bc=BC, precision=prec, dist=dist) as r:
            r.set_global_state(U0)
            dts = [r.step(0.3) for _ in range(3)]
            U, R = r.get_state()
        with mpcf.Solver([DIMS], bc=[BC], precision=prec) as s:
            s.set_state(U0)
            dts_ref = [s.step(cfl=0.3)[0] for _ in range(3)]
            U_ref, R_ref = s.get_state()
        assert dts == dts_ref, (dts, dts_ref)
        assert_bitwise(U, U_ref, "state")
        assert_bitwise(R, R_ref, "register")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("prec", ["fp32_ref", "fp64"])
def test_single_rank_driver_stream_ordered_matches_step(mpcf, prec):
    """The stream-ordered rank driver (sound speed, its NCCL all-reduce, the
    device dt and the stages all on the solver's stream, no host round trip)
    reproduces mpcf_step bit for bit, the time included."""
    import datetime
    import os
    import socket
    import torch.distributed as dist
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        U0 = _state(prec, mpcf)
        with dc.SlabRank(DIMS, bc=BC, precision=prec, dist=dist) as r:
            r.set_global_state(U0)
            t = r.run(3, 0.3, ordered=True)
            U, R = r.get_state()
            assert r.solver.error_word() == 0
        with mpcf.Solver([DIMS], bc=[BC], precision=prec) as s:
            s.set_state(U0)
            t_ref = s.run(3, cfl=0.3, graph=False)[0]
            U_ref, R_ref = s.get_state()
        assert t == t_ref, (t, t_ref)
        assert_bitwise(U, U_ref, "state")
        assert_bitwise(R, R_ref, "register")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("prec", ["fp32_ref", "fp64"])
def test_slab_initial_conditions_match_undivided_domain(mpcf, prec):
    """Each slab carries its place in the global grid (mpcf_set_origin), so
    the device generators write the undivided domain's initial condition,
    slice by slice: the bubble cloud (noise streams included), the
    shock-induced cloud collapse, a Sod tube and a reversed 2DSBI set up
    across the slabs."""
    rng = np.random.default_rng(5)
    params, bub = mpcf.configs.small_cloud(DIMS, nb=3)
    h = dc.global_spacing(DIMS)
    shapes = np.column_stack([rng.uniform(0.2, 0.8, 8) * DIMS[0] * h,       # centres inside the domain
                              rng.uniform(0.2, 0.8, 8) * DIMS[1] * h,
                              rng.uniform(0.2, 0.8, 8) * DIMS[2] * h,
                              rng.uniform(0.03, 0.08, 8)])
    sic = mpcf.sic_params(eps=0.01, shock_n=(0.0, 0.0, 1.0), shock_s=(0.0, 0.0, 0.3))
    sbi_bub = np.array([[0.5, 0.3, 0.4, 0.1], [0.2, 0.4, 0.25, 0.08]])
    cases = {
        "cloud": lambda s, d: s.ic_cloud(params, bub, dom=d),
        "sic": lambda s, d: s.ic_sic_cloud(sic, shapes, dom=d),
        "sod": lambda s, d: s.ic_sod(dom=d, config="z", reverse=1),
        "sbi": lambda s, d: s.ic_sbi(sbi_bub, dom=d, config="xz", reverse=1, mollfactor=2),
    }
    for name, ic in cases.items():
        with mpcf.Solver([DIMS], bc=[BC], precision=prec) as s:
            ic(s, 0)
            want = s.get_state(with_reg=False)
        s, ext_ = dc.slab_solver(DIMS, 3, bc=BC, precision=prec)
        with s:
            for r in range(3):
                ic(s, r)
            got = dc.gather_state(s, ext_, with_reg=False)
        assert_bitwise(got, want, f"{name} initial condition over 3 slabs")


def test_linked_slabs_autotune_and_restart(mpcf, tmp_path):
    """The autotuner's trial stages on linked slabs exchange their ghost
    planes too and leave the state as it was; each slab saves and restarts
    like a domain; a run continued from the restarted slabs equals the
    undivided run bit for bit."""
    prec = "mixed"
    U0 = _state(prec, mpcf)
    t_ref, (U_ref, R_ref) = _undivided(mpcf, prec, U0, 4, True)
    s, ext = dc.slab_solver(DIMS, 3, bc=BC, precision=prec)
    with s:
        dc.scatter_state(s, DIMS, ext, U0)
        before = dc.gather_state(s, ext)
        s.autotune(reps=1)
        after = dc.gather_state(s, ext)
        assert_bitwise(after[0], before[0], "state after autotune")
        t2 = s.run(2, cfl=0.3, graph=True)
        for r in range(3):
            d = tmp_path / f"slab{r}"
            d.mkdir()
            s.save(d, t2[r], 2, dom=r)
    s2, _ = dc.slab_solver(DIMS, 3, bc=BC, precision=prec)
    with s2:
        for r in range(3):
            t, step, _ = s2.restart(tmp_path / f"slab{r}", dom=r)
            assert step == 2
        t4 = s2.run(2, cfl=0.3, graph=True)
        U, _ = dc.gather_state(s2, ext)
    assert t4 == pytest.approx([t_ref[0]] * 3, rel=1e-14)
    assert_bitwise(U, U_ref, "state after save, restart and two more steps")
