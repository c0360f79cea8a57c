"""Windowed runs (mpcf_create_window / mpcf_run_window): a domain held in
host memory streamed through a few device slots in z-chunks of nslices planes
(the reference's GPUlab with nslices < sizeZ, GPUlab.cpp:37-41,202-372,
703-793), so that a domain larger than device memory can be advanced.

Every step must be bit-identical to the same steps of the whole domain
resident on the device (mpcf_run): chunks of 3 planes (the stencil's reach)
up to several tile layers, the fewest slots the wavefront needs and more,
absorbing and reflecting z faces (ghost planes by the boundary condition),
every precision form, the reference's WENO3 build, and the 512^3 cloud of
the benchmark."""
import numpy as np
import pytest

from conftest import cloud_state
from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu

ABS, REF = 0, 1


def resident(mpcf, dims, bc, prec, U0, steps):
    with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
        s.set_state(U0)
        t = s.run(steps, cfl=0.3, graph=False)[0]
        return t, s.get_state(with_reg=False)


@pytest.mark.parametrize("prec,nslices,nslots,bc,tiling", [
    ("fp32_ref", 8, 5, (ABS,) * 6, None),              # 12 chunks through the fewest slots
    ("fp32_ref", 3, 6, (ABS, REF, REF, ABS, REF, REF), (7, 3, True, True)),   # chunks of the stencil's reach
    ("mixed", 16, 5, (REF,) * 6, (8, 16, True, True)),
    ("mixed", 32, 8, (ABS, ABS, ABS, ABS, REF, ABS), (8, 8, False, True)),    # more slots than chunks
    ("fp64", 12, 5, (ABS, REF, ABS, REF, ABS, REF), (3, 12, False, False)),
    ("fp32", 24, 4, (ABS,) * 6, None),                 # 4 chunks in 4 slots
    ("fp64_fast", 6, 7, (REF, ABS, ABS, REF, ABS, REF), None),
])
def test_window_run_equals_resident_run(mpcf, prec, nslices, nslots, bc, tiling):
    dims = (48, 40, 96)
    dtype = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    U0 = cloud_state(dims, nb=3, seed=17, dtype=dtype)
    t_res, U_res = resident(mpcf, dims, bc, prec, U0, 3)
    host = [np.ascontiguousarray(a, dtype=dtype).copy() for a in U0]
    with mpcf.WindowSolver(dims, nslices, nslots, bc=bc, precision=prec) as w:
        assert w.nchunks == dims[2] // nslices and w.nslots == min(nslots, w.nchunks)
        if tiling:
            w.set_tiling(*tiling)
        t = w.run(host, 3, cfl=0.3)
        assert w.error_word() == 0
    assert t == t_res, (t, t_res)
    assert_bitwise(host, U_res, f"windowed {prec}, {nslices}-plane chunks in {nslots} slots")


def test_window_run_in_two_calls(mpcf):
    """Two calls of 2 steps continue one run of 4 (the second call's first
    step reduces the sound speed of the host state again)."""
    dims = (40, 32, 60)
    bc = (ABS, REF, ABS, ABS, REF, ABS)
    U0 = cloud_state(dims, nb=2, seed=3)
    t_res, U_res = resident(mpcf, dims, bc, "fp32_ref", U0, 4)
    host = [np.array(a, dtype=np.float32) for a in U0]
    with mpcf.WindowSolver(dims, 5, 6, bc=bc, precision="fp32_ref") as w:
        w.run(host, 2)
        t = w.run(host, 2)
        assert w.error_word() == 0
    assert t == t_res
    assert_bitwise(host, U_res, "two windowed calls")


def test_window_rejects_what_it_cannot_run(mpcf):
    dims = (32, 16, 40)
    with pytest.raises(mpcf.MpcfError, match="divide"):
        mpcf.WindowSolver(dims, 7, 6)
    with pytest.raises(mpcf.MpcfError, match="at least 3"):
        mpcf.WindowSolver((32, 16, 40), 2, 6)
    with pytest.raises(mpcf.MpcfError, match="too few"):
        mpcf.WindowSolver(dims, 4, 4)
    with pytest.raises(mpcf.MpcfError, match="boundary condition"):
        mpcf.WindowSolver(dims, 8, 5, bc=(0, 0, 0, 0, 2, 0))
    with mpcf.WindowSolver(dims, 8, 5) as w:
        for call in (lambda: w.step(cfl=0.3), lambda: w.stage(0.0, 0.25, 0.01), lambda: mpcf.Solver.run(w, 1),
                     lambda: w.link_z(0, 1)):
            with pytest.raises(mpcf.MpcfError, match="windowed"):
                call()
        with pytest.raises(ValueError):
            w.run([np.zeros(10, np.float32)] * 7, 1)


def test_window_run_512cube(mpcf):
    """The benchmark's 512^3 cloud in 16 chunks of 32 planes through 6 slots
    (5.0 GB of slots on the device against 11.3 GB resident), three steps:
    bit-identical to the resident run."""
    import torch
    cfg = mpcf.configs.config("c3_512")
    dims = cfg["dims"][0]
    with mpcf.Solver([dims], precision="mixed") as s:
        s.set_tiling(8, 32, True, True)
        s.ic_cloud(cfg["params"], cfg["bubbles"][0])
        U0 = s.get_state(with_reg=False)
        t_res = s.run(3, cfl=0.3, graph=True)[0]
        U_res = s.get_state(with_reg=False)
    host = [torch.empty(U0[0].size, dtype=torch.float32, pin_memory=True) for _ in range(7)]
    for q in range(7):
        host[q].numpy()[:] = U0[q]
    del U0
    arrs = [h.numpy() for h in host]
    with mpcf.WindowSolver(dims, 32, 6, precision="mixed") as w:
        w.set_tiling(8, 32, True, True)
        t = w.run(arrs, 3, cfl=0.3)
        assert w.error_word() == 0
    assert t == t_res, (t, t_res)
    for q in range(7):
        assert np.array_equal(arrs[q], U_res[q]), q


def test_window_run_larger_than_device_memory(mpcf):
    """A 1344^3 FP32 cloud (2.43e9 cells): its two state buffers and the
    register would take 204 GB on the device, more than the B200's 192 GB;
    the windowed run streams it in 42 chunks of 32 planes through 6 slots
    (34.6 GB).  One step of the 200-bubble cloud (generated chunk by chunk
    in the global domain's coordinates); the planes of three z-windows (at
    the bottom face, across a chunk boundary in the middle, at the top face)
    are compared bit for bit with a resident run of each window and the 9
    planes beside it (a stage reads 3 planes beyond a cell), advanced with
    the windowed run's dt."""
    import psutil
    import torch
    n1 = 1344
    dims = (n1, n1, n1)
    N = n1 ** 3
    plane = n1 * n1
    if psutil.virtual_memory().available < 120e9:
        pytest.skip("needs 120 GB of free host memory")
    if 3 * 7 * 4 * N <= torch.cuda.mem_get_info()[1]:
        pytest.skip("the domain would fit on this device")
    cfg = mpcf.configs.config("c3_512")
    host = [torch.empty(N, dtype=torch.float32, pin_memory=True) for _ in range(7)]
    arrs = [h.numpy() for h in host]
    T = 32
    with mpcf.Solver([(n1, n1, T)], precision="mixed") as g:
        for z0 in range(0, n1, T):
            g.set_origin((0, 0, z0), dims)
            g.ic_cloud(cfg["params"], cfg["bubbles"][0])
            st = g.get_state(with_reg=False)
            for q in range(7):
                arrs[q][z0 * plane:(z0 + T) * plane] = st[q]
    margin = 9
    slabs = []
    for z0, z1 in ((0, 32), (656, 688), (n1 - 32, n1)):
        lo, hi = max(0, z0 - margin), min(n1, z1 + margin)
        slabs.append((z0, z1, lo, hi, [a[lo * plane:hi * plane].copy() for a in arrs]))
    with mpcf.WindowSolver(dims, T, 6, precision="mixed") as w:
        w.set_tiling(8, 32, True, True)
        t = w.run(arrs, 1, cfl=0.3)
        assert w.error_word() == 0
    dtinvh = float(np.float32(t / (1.0 / n1)))
    for z0, z1, lo, hi, U0 in slabs:
        with mpcf.Solver([(n1, n1, hi - lo)], precision="mixed") as s:
            s.set_tiling(8, 32, True, True)
            s.set_state(U0)
            for a, b in mpcf.LSRK3:
                s.stage(a, b, dtinvh)
            U = s.get_state(with_reg=False)
            assert s.error_word() == 0
        sl = slice((z0 - lo) * plane, (z1 - lo) * plane)
        for q in range(7):
            assert np.array_equal(U[q][sl], arrs[q][z0 * plane:z1 * plane]), (z0, q)


@pytest.mark.parametrize("prec,nslices,nslots", [("fp32_ref", 4, 3), ("mixed", 8, 6), ("fp64", 6, 4)])
def test_window_stage_and_sound_speed_equal_resident(mpcf, prec, nslices, nslots):
    """One stage of a block whose state and register live in host memory
    (mpcf_window_stage, the reference's chunked process_all) equals the
    resident stage with the same dt/h bit for bit, register included; the
    streamed sound speed equals the resident one."""
    dims = (40, 24, 48)
    bc = (ABS, REF, REF, ABS, REF, ABS)
    dtype = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    U0 = cloud_state(dims, nb=2, seed=41, dtype=dtype)
    R0 = [np.asarray(a, dtype=dtype) * dtype(1e-3) for a in cloud_state(dims, nb=1, seed=42, dtype=dtype)]
    a, b, dtinvh = -17.0 / 32, 8.0 / 9, 0.0371
    with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
        s.set_state(U0, R0)
        sos = s.max_sos()[0]
        s.stage(a, b, dtinvh)
        U_res, R_res = s.get_state()
    host = [np.array(x, dtype=dtype) for x in U0]
    reg = [np.array(x, dtype=dtype) for x in R0]
    with mpcf.WindowSolver(dims, nslices, max(nslots, 5), bc=bc, precision=prec) as w:
        assert w.max_sos_host(host) == sos
        w.stage_host(host, reg, a, b, dtinvh)
        assert w.error_word() == 0
    assert_bitwise(host, U_res, f"windowed stage {prec}")
    assert_bitwise(reg, R_res, f"windowed stage register {prec}")


@pytest.mark.parametrize("prec", ["fp32_ref", "fp64"])
def test_window_run_weno3_equals_resident(mpcf, prec):
    """The reference's compile-time WENO3 reconstruction (set on the windowed
    solver, every slot) streams like WENO5: two steps equal the resident run."""
    dims = (40, 24, 48)
    bc = (ABS, REF, ABS, ABS, REF, ABS)
    dtype = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    U0 = cloud_state(dims, nb=2, seed=23, dtype=dtype)
    with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
        s.set_weno_order(3)
        s.set_state(U0)
        t_res = s.run(2, cfl=0.3, graph=False)[0]
        U_res = s.get_state(with_reg=False)
    host = [np.array(a, dtype=dtype) for a in U0]
    with mpcf.WindowSolver(dims, 6, 5, bc=bc, precision=prec) as w:
        w.set_weno_order(3)
        t = w.run(host, 2, cfl=0.3)
        assert w.error_word() == 0
    assert t == t_res
    assert_bitwise(host, U_res, f"windowed WENO3 {prec}")
