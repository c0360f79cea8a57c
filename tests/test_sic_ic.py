"""The reference's shock-induced cloud-collapse initial condition
(source/Sim/Sim_SICCloudMPI.cpp:43-357), on the CPU:

1. the oracle restatement (oracle/oracle_ic.h) against golden fields the
   reference's own IC code produced (tests/golden/ref_sic_ic.npz, made by
   tests/golden/make_golden.py from oracle/_ref/libref_sic_ic.so);
2. the same live against the reference where oracle/_ref was built here;
3. the library's post-shock state (a host function of the C ABI) against
   the reference's, bit for bit.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_sic_ic.npz")


def golden_cases():
    g = np.load(GOLD)
    i = 0
    while f"dims{i}" in g.files:
        yield (tuple(int(v) for v in g[f"dims{i}"]), g[f"prm{i}"], g[f"shapes{i}"], float(g[f"eps{i}"]),
               g[f"U{i}"], tuple(g[f"post{i}"]))
        i += 1


def test_golden_sic_ic_bitexact():
    n = 0
    for dims, prm, shapes, eps, U, post in golden_cases():
        out, opost = O.sic_cloud(dims, prm, shapes, eps)
        assert opost == post
        for q in range(7):
            assert np.array_equal(out[q], U[q]), (n, q, np.abs(out[q].astype(np.float64) - U[q]).max())
        n += 1
    assert n >= 3


def test_sic_ic_physical_and_mixed():
    """Liquid, gas and shocked liquid all appear, and the mixture is physical."""
    dims, prm, shapes, eps, U, post = next(golden_cases())
    rho, E, G, P = U[0], U[4], U[5], U[6]
    assert rho.min() > 0 and E.min() > 0 and G.min() > 0 and P.min() > 0
    assert np.isclose(rho.max(), post[0], rtol=1e-6)        # post-shock liquid present
    assert rho.min() < 2                                     # gas present
    # the shocked region moves at u1 (momentum rho*u1)
    shocked = np.isclose(rho, np.float32(post[0]))
    assert np.allclose(U[1][shocked], np.float32(post[0]) * np.float32(post[1]), rtol=1e-6)


@pytest.fixture(scope="module")
def refsic():
    L = O.ref_lib("libref_sic_ic")
    if L is None:
        pytest.skip("oracle/_ref not built (the reference tree is absent)")
    return L


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_live_sic_ic_random_clouds(refsic, seed):
    # option values are non-negative: the reference's parser takes any token
    # starting with '-' as an option name (ArgumentParser.h:104-121)
    rng = np.random.default_rng(seed)
    prm = list(O.SIC_DEFAULTS)
    prm[2] = float(rng.uniform(1, 200))                              # p0
    prm[6] = float(rng.uniform(5, 60))                               # pressure ratio
    prm[7:10] = [float(v) for v in np.abs(rng.normal(0, 1, 3)) + np.array([1.0, 0, 0])]   # >= 0 (above)
    prm[10:13] = [float(v) for v in rng.uniform(0, 0.3, 3)]
    k = int(rng.integers(1, 20))
    sh = np.column_stack([rng.uniform(-0.1, 1.1, k), rng.uniform(-0.1, 0.9, k), rng.uniform(-0.1, 0.75, k),
                          rng.uniform(0.01, 0.2, k)]).astype(np.float32).astype(np.float64)
    eps = [0.0, 0.02, 0.05][seed % 3]
    with tempfile.TemporaryDirectory() as w:
        dims, ref, rpost = O.ref_sic_cloud(refsic, prm, sh, eps, w)
    out, opost = O.sic_cloud(dims, prm, sh, eps)
    assert opost == rpost
    for q in range(7):
        assert np.array_equal(out[q], ref[q]), (q, np.abs(out[q].astype(np.float64) - ref[q]).max())


def test_sic_post_shock_c_abi_matches_reference(mpcf):
    """mpcf_sic_post_shock (library host code, no GPU) equals the reference's
    post-shock state for every golden case, in FP32 reference rounding."""
    keys = ("rho0", "u0", "p0", "rhoB", "uB", "pB", "pressure_ratio")
    for dims, prm, shapes, eps, U, post in golden_cases():
        kw = {k: prm[i] for i, k in enumerate(keys)}
        kw.update(shock_n=prm[7:10], shock_s=prm[10:13], g1=prm[13], g2=prm[14], pc1=prm[15], pc2=prm[16], eps=eps)
        p = mpcf.sic_params(**kw)
        assert mpcf.sic_post_shock(p, "fp32_ref") == post
    # the library's defaults are the reference's option defaults
    d = mpcf.sic_params()
    got = (d.rho0, d.u0, d.p0, d.rhoB, d.uB, d.pB, d.pressure_ratio, *d.shock_n, *d.shock_s, d.g1, d.g2, d.pc1, d.pc2)
    assert got == O.SIC_DEFAULTS and d.eps == 0.0


def test_sic_params_rejected(mpcf):
    with pytest.raises(mpcf.MpcfError):
        mpcf.sic_post_shock(mpcf.sic_params(shock_n=(0, 0, 0)))
    with pytest.raises(mpcf.MpcfError):
        mpcf.sic_post_shock(mpcf.sic_params(g1=1.0))
