"""The precision report of bench.py (CPU only): `precision_error` is the
relative L1 and L-inf of rho, p and G of a form's state against the FP64
run, accumulated in chunks of cells so that a 1024^3 comparison fits in host
memory.  Checked against a direct whole-array computation, with chunks that
do not divide the cell count, on an FP32 state and an FP64 reference."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def cloud_like(n, seed, dtype):
    """A stiffened-gas state with liquid-like magnitudes: rho ~ 1e3, E ~ P."""
    rng = np.random.default_rng(seed)
    rho = 1000.0 + rng.normal(0, 5, n)
    vel = rng.normal(0, 1e-3, (3, n))
    G = 1.0 / 5.59 + rng.normal(0, 1e-4, n)
    P = 6.59 * 4096.0 / 5.59 + rng.normal(0, 1, n)
    p = 100.0 + rng.normal(0, 1, n)
    E = G * p + P + 0.5 * rho * (vel ** 2).sum(0)
    return [a.astype(dtype) for a in (rho, rho * vel[0], rho * vel[1], rho * vel[2], E, G, P)]


def direct(st, ref64):
    rho = st[0].astype(np.float64)
    ke = sum(st[q].astype(np.float64) ** 2 for q in (1, 2, 3))
    G = st[5].astype(np.float64)
    p = (st[4].astype(np.float64) - 0.5 * ke / rho - st[6].astype(np.float64)) / G
    out = {}
    for name, v, r in (("rho", rho, ref64[0]), ("p", p, ref64[1]), ("G", G, ref64[2])):
        out["L1_" + name] = np.abs(v - r).sum() / np.abs(r).sum()
        out["Linf_" + name] = np.abs(v - r).max() / np.abs(r).max()
    return out


@pytest.mark.parametrize("chunk", [1 << 24, 1000, 4093])
def test_precision_error_matches_direct_computation(monkeypatch, chunk):
    monkeypatch.setattr(bench, "CHUNK", chunk)
    n = 20011
    st64 = cloud_like(n, 1, np.float64)
    st32 = [a.astype(np.float32) for a in st64]
    ref = bench.derived_fields(st64)
    got = bench.errors_against(st32, ref)
    want = direct(st32, ref)
    assert set(got) == set(want)
    for k in want:
        assert got[k] == pytest.approx(want[k], rel=1e-9), k
    # FP32 storage of the same state: rho and G round to ~3e-8, the
    # pressure carries the cancellation of E against P
    assert got["L1_rho"] < 1e-7 and got["L1_G"] < 1e-7
    assert got["L1_p"] > got["L1_rho"]


def test_identical_states_have_zero_error():
    st = cloud_like(5000, 2, np.float64)
    err = bench.errors_against(st, bench.derived_fields(st))
    assert all(v == 0.0 for v in err.values())
