"""GPU generator of the reference's shock-induced cloud-collapse IC
(mpcf_ic_sic_cloud; Sim_SICCloudMPI.cpp:43-357) against the reference's own
fields (golden) and the oracle restatement, through the C ABI."""
import os

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_sic_ic.npz")
KEYS = ("rho0", "u0", "p0", "rhoB", "uB", "pB", "pressure_ratio")


def params(mpcf, prm, eps):
    kw = {k: float(prm[i]) for i, k in enumerate(KEYS)}
    kw.update(shock_n=prm[7:10], shock_s=prm[10:13], g1=prm[13], g2=prm[14], pc1=prm[15], pc2=prm[16], eps=eps)
    return mpcf.sic_params(**kw)


def gpu_ic(mpcf, dims, prm, shapes, eps, precision="fp32_ref"):
    with mpcf.Solver([dims], precision=precision) as s:
        s.ic_sic_cloud(params(mpcf, prm, eps), shapes)
        U, R = s.get_state()
    for q in range(7):
        assert not np.any(R[q])
    return U


def test_sic_ic_equals_reference_fields():
    """FP32 reference rounding: bit-identical to the reference's own IC code
    on every golden case (sharp and cosine-ramp interfaces, oblique shock)."""
    import mpcf
    g = np.load(GOLD)
    i = 0
    while f"dims{i}" in g.files:
        dims = tuple(int(v) for v in g[f"dims{i}"])
        U = gpu_ic(mpcf, dims, g[f"prm{i}"], g[f"shapes{i}"], float(g[f"eps{i}"]))
        for q in range(7):
            assert np.array_equal(U[q], g[f"U{i}"][q]), (i, q)
        i += 1
    assert i >= 3


@pytest.mark.parametrize("dims,eps", [((40, 33, 20), 0.0), ((17, 48, 9), 0.0), ((32, 32, 32), 0.04)])
def test_sic_ic_equals_oracle(mpcf, dims, eps):
    rng = np.random.default_rng(sum(dims))
    prm = list(O.SIC_DEFAULTS)
    prm[2], prm[10] = 50.0, 0.25
    prm[7:10] = [1.0, 0.4, -0.3]
    k = 25
    sh = np.column_stack([rng.uniform(0.2, 1.0, k), rng.uniform(0.0, 1.0, k), rng.uniform(0.0, 0.6, k),
                          rng.uniform(0.01, 0.1, k)])
    U = gpu_ic(mpcf, dims, prm, sh, eps)
    W, _ = O.sic_cloud(dims, prm, sh, eps)
    for q in range(7):
        if eps == 0:
            assert np.array_equal(U[q], W[q]), q
        else:
            # the cosine ramp: CUDA's and the C library's cos may differ in
            # the last bit of a double
            assert np.abs(U[q].astype(np.float64) - W[q]).max() <= 1e-6 * np.abs(W[q]).max(), q


def test_sic_ic_many_shapes_in_one_tile(mpcf):
    """More spheres within reach of one tile than its shared-memory list holds
    (1024): that tile reads every sphere, with the same result."""
    rng = np.random.default_rng(5)
    dims = (24, 24, 16)
    k = 1500
    sh = np.column_stack([rng.uniform(0.30, 0.45, k), rng.uniform(0.30, 0.45, k), rng.uniform(0.2, 0.35, k),
                          rng.uniform(0.002, 0.02, k)])
    prm = list(O.SIC_DEFAULTS)
    U = gpu_ic(mpcf, dims, prm, sh, 0.0)
    W, _ = O.sic_cloud(dims, prm, sh, 0.0)
    for q in range(7):
        assert np.array_equal(U[q], W[q]), q


def test_sic_ic_fp64(mpcf):
    rng = np.random.default_rng(9)
    dims = (30, 26, 22)
    k = 12
    sh = np.column_stack([rng.uniform(0.3, 0.9, k), rng.uniform(0.1, 0.8, k), rng.uniform(0.1, 0.6, k),
                          rng.uniform(0.03, 0.12, k)])
    prm = list(O.SIC_DEFAULTS)
    prm[2] = 100.0
    U = gpu_ic(mpcf, dims, prm, sh, 0.0, precision="fp64")
    W, post = O.sic_cloud(dims, prm, sh, 0.0, dtype=np.float64)
    for q in range(7):
        assert np.array_equal(U[q], W[q]), q
    assert mpcf.sic_post_shock(params(mpcf, prm, 0.0), "fp64") == post


def test_sic_ic_then_lsrk3_step(mpcf):
    """The shocked cloud through one full LSRK3 step: GPU (reference rounding)
    against the oracle, bit for bit, and the state stays physical."""
    dims = (24, 20, 16)
    g = np.load(GOLD)
    prm, sh = g["prm0"], g["shapes0"]
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.ic_sic_cloud(params(mpcf, prm, 0.0), sh)
        U0, R0 = s.get_state()
        s.run(1, cfl=0.3, graph=False)
        Ug, Rg = s.get_state()
        assert s.error_word() == 0
    U, R = [a.copy() for a in U0], [a.copy() for a in R0]
    O.step(dims, (0,) * 6, U, R, cfl=0.3)
    for q in range(7):
        assert np.array_equal(Ug[q], U[q]), q
        assert np.array_equal(Rg[q], R[q]), q
    assert Ug[0].min() > 0 and Ug[4].min() > 0
