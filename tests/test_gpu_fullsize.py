"""Full-size GPU checks (the benchmark configurations' sizes) through
size-independent properties: invariance of a uniform state, axis
permutations, conservation between reflecting walls, graph replay against
plain steps, ensembles against separate solvers, the host-resident streamed
run (the e2e path) against the device-resident run.  Parity against the CPU
oracle at these sizes and tilings is in test_gpu_parity_bench.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ABS, REF = 0, 1


def uniform(dims, vel=(0.0, 0.0, 0.0), dtype=np.float32):
    n = dims[0] * dims[1] * dims[2]
    rho, p, g, pc = 1000.0, 100.0, 6.59, 4096.0
    G, P = 1 / (g - 1), g * pc / (g - 1)
    E = G * p + P + 0.5 * rho * sum(v * v for v in vel)
    return [np.full(n, v, dtype) for v in (rho, rho * vel[0], rho * vel[1], rho * vel[2], E, G, P)]


@pytest.mark.parametrize("prec", ["fp32_ref", "mixed", "fp64", "fp64_fast"])
def test_uniform_state_invariant_256cube(mpcf, prec):
    dims = (256, 256, 256)
    dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    U0 = uniform(dims, vel=(0.3, -0.2, 0.1), dtype=dt)
    with mpcf.Solver([dims], precision=prec) as s:
        s.set_state(U0)
        s.run(2, cfl=0.3, graph=True)
        U, R = s.get_state()
        assert s.error_word() == 0
    for q in range(7):
        assert np.array_equal(U[q], U0[q]), q
        assert not np.any(R[q]), q


def permute(U, dims, axes):
    nx, ny, nz = dims
    out = []
    for a in U:
        arr = a.reshape(nz, ny, nx).transpose(2, 1, 0).transpose(axes)
        out.append(np.ascontiguousarray(arr.transpose(2, 1, 0)).ravel())
    m = [out[1], out[2], out[3]]
    out[1], out[2], out[3] = m[axes[0]], m[axes[1]], m[axes[2]]
    return out


def test_axis_permutation_at_scale(mpcf):
    """A tube problem along x, y or z gives permuted results (reference
    rounding, GPU only, 256x64x64): identical for x <-> y, equal to rounding
    for x <-> z."""
    dims = (256, 64, 64)
    U = uniform(dims)
    gas = uniform(dims)
    # gas column on the left half (ideal gas, gamma 1.4, p 0.0234, rho 1)
    n = dims[0] * dims[1] * dims[2]
    ix = np.arange(n) % dims[0]
    left = ix < dims[0] // 2
    Gg, rho_g, p_g = 1 / 0.4, 1.0, 0.0234
    vals = (rho_g, 0.0, 0.0, 0.0, Gg * p_g, Gg, 0.0)
    for q in range(7):
        gas[q][:] = vals[q]
        U[q] = np.where(left, gas[q], U[q]).astype(np.float32)
    res = {}
    for axes in ((0, 1, 2), (1, 0, 2), (2, 1, 0)):
        pd = tuple(dims[a] for a in axes)
        with mpcf.Solver([pd], precision="fp32_ref") as s:
            s.set_state(permute(U, dims, axes))
            s.run(2, cfl=0.3, graph=False)
            res[axes] = permute(s.get_state(with_reg=False), pd, tuple(np.argsort(axes)))
    # x <-> y: bit-identical.  x <-> z: the reference accumulates the G/P
    # extra-term sums x, then y, then z ((X + Y) + Z, GPUkernels.cu:35-62,
    # 422-444,795-817), and floating-point addition does not reassociate, so
    # a permutation that moves the varying term from first to last place
    # changes the last bit of sumG/sumP; equal to rounding.
    for q in range(7):
        assert np.array_equal(res[(1, 0, 2)][q], res[(0, 1, 2)][q]), ((1, 0, 2), q)
        a, b = res[(2, 1, 0)][q], res[(0, 1, 2)][q]
        assert np.abs(a.astype(np.float64) - b).max() <= 1e-6 * max(np.abs(b).max(), 1.0), ((2, 1, 0), q)


def test_fp64_conservation_reflecting_256cube(mpcf):
    dims = (256, 256, 256)
    cfg = mpcf.configs.config("c2_256")
    with mpcf.Solver([dims], bc=[(REF,) * 6], precision="fp64") as s:
        s.ic_cloud(cfg["params"], cfg["bubbles"][0])
        s0 = s.conserved_sums()[0]
        s.track_conservation(True)
        s.run(5, cfl=0.3, graph=True)
        s1 = s.conserved_sums()[0]
        assert s.error_word() == 0
    assert abs(s1[0] - s0[0]) <= 1e-12 * abs(s0[0])
    assert abs(s1[4] - s0[4]) <= 1e-12 * abs(s0[4])


def test_config2_256cube_100_steps_stays_physical(mpcf):
    """Configuration 2: 256^3, 50 bubbles, 100 steps at CFL 0.3, FP32,
    fully device resident: no non-physical state, time advances."""
    cfg = mpcf.configs.config("c2_256")
    with mpcf.Solver(cfg["dims"], precision="fp32") as s:
        s.ic_cloud(cfg["params"], cfg["bubbles"][0])
        t = s.run(100, cfl=0.3, graph=True)[0]
        assert s.error_word() == 0
        U = s.get_state(with_reg=False)
    assert t > 0 and np.isfinite(t)
    assert np.isfinite(U[0]).all() and U[0].min() > 0


def test_ensemble_equals_separate_solvers(mpcf):
    """Configuration 4's ensemble (64 uneven domains, one persistent launch
    per stage, CUDA graph) advances every domain exactly as a solver of that
    domain alone would (reference rounding, per-domain dt)."""
    cfg = mpcf.configs.config("c4_ensemble")
    dims = cfg["dims"]
    with mpcf.Solver(dims, precision="fp32_ref") as s:
        s.set_tiling(3, 32, True)
        for d, bub in enumerate(cfg["bubbles"]):
            s.ic_cloud(cfg["params"], bub, dom=d)
        t_ens = s.run(3, cfl=0.3, graph=True)
        ens = [s.get_state(dom=d, with_reg=False) for d in range(len(dims))]
    for d in (0, 17, 63):
        with mpcf.Solver([dims[d]], precision="fp32_ref") as s1:
            s1.ic_cloud(cfg["params"], cfg["bubbles"][d])
            t1 = s1.run(3, cfl=0.3, graph=False)[0]
            one = s1.get_state(with_reg=False)
        assert t1 == t_ens[d], d
        for q in range(7):
            assert np.array_equal(one[q], ens[d][q]), (d, q)


def test_graph_replay_equals_plain_steps_512cube(mpcf):
    cfg = mpcf.configs.config("c3_512")
    out = []
    for graph in (True, False):
        with mpcf.Solver(cfg["dims"], precision="mixed") as s:
            s.ic_cloud(cfg["params"], cfg["bubbles"][0])
            t = s.run(2, cfl=0.3, graph=graph)[0]
            st = s.get_state(with_reg=False)
            out.append((t, st[0][::997].copy(), st[4][::997].copy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])


def test_streamed_run_equals_resident_run_512cube(mpcf):
    """The e2e path at the bench's size and settings: configuration 3's
    cloud held in page-locked host memory and streamed through the GPU in 16
    z-chunks (32 x 8 tiles, 32-plane layers, persistent, bulk-copy staging),
    three steps, against the same steps of the device-resident run: the
    host state and the time bit for bit."""
    import torch
    cfg = mpcf.configs.config("c3_512")
    dims = cfg["dims"][0]
    tiling = (8, 32, True, True)
    with mpcf.Solver([dims], precision="mixed") as s:
        s.set_tiling(*tiling)
        s.ic_cloud(cfg["params"], cfg["bubbles"][0])
        U0 = s.get_state(with_reg=False)
        t_res = s.run(3, cfl=0.3, graph=True)[0]
        U_res = s.get_state(with_reg=False)
    host = [torch.empty(U0[0].size, dtype=torch.float32, pin_memory=True) for _ in range(7)]
    for q in range(7):
        host[q].numpy()[:] = U0[q]
    del U0
    arrs = [h.numpy() for h in host]
    with mpcf.Solver([dims], precision="mixed") as s:
        s.set_tiling(*tiling)
        t = s.run_host(arrs, 3, cfl=0.3, nchunks=16)
        assert s.error_word() == 0
    assert t == t_res, (t, t_res)
    for q in range(7):
        assert np.array_equal(arrs[q], U_res[q]), q
