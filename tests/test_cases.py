"""The reference's SteadyState, Sod and 2DSBI initial conditions on the CPU:
the restatement oracle_lib.case_ic against the reference's own case code
(golden record tests/golden/ref_cases.npz, and live where oracle/_ref was
built here), bit for bit."""
import os
import tempfile

import numpy as np
import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cases.npz")


def golden_cases():
    g = np.load(GOLD)
    i = 0
    while f"case{i}" in g.files:
        case = str(g[f"case{i}"])
        opts = [tuple(x.split("=", 1)) for x in g[f"opts{i}"]]
        opts = [(k, v if k == "-config" else float(v)) for k, v in opts]
        bub = g[f"bubbles{i}"]
        yield (case, O.case_prm(case, opts), tuple(int(v) for v in g[f"dims{i}"]),
               bub if len(bub) else None, list(g[f"U{i}"]))
        i += 1


def test_golden_cases_bitexact():
    seen = set()
    for case, prm, dims, bub, U in golden_cases():
        out = O.case_ic(case, dims, prm, bub)
        for q in range(7):
            assert np.array_equal(out[q], U[q]), (case, q)
        seen.add(case)
    assert seen == {"steady", "sod", "sbi"}


@pytest.mark.parametrize("seed", [1, 2])
def test_live_cases_random_options(seed):
    L = O.ref_lib("libref_cases")
    if L is None:
        pytest.skip("oracle/_ref not built (the reference tree is absent)")
    rng = np.random.default_rng(seed)
    config = ["xy", "xz", "yx", "yz", "zx", "zy"][int(rng.integers(6))]
    sod_cfg = "xyz"[int(rng.integers(3))]
    runs = [
        ("steady", [("-rho", float(rng.uniform(0.5, 1000))), ("-u", float(rng.uniform(0, 5))),
                    ("-p", float(rng.uniform(0.1, 100))), ("-g", float(rng.uniform(1.1, 7))),
                    ("-pc", float(rng.uniform(0, 5000)))], None, "xy"),
        ("sod", [("-config", sod_cfg), ("-x0", float(rng.uniform(0.2, 0.8))), ("-reverse", int(rng.integers(2))),
                 ("-rho2", float(rng.uniform(0.1, 1))), ("-u1", float(rng.uniform(0, 2)))], None, sod_cfg),
        ("sbi", [("-config", config), ("-mach", float(rng.uniform(1.05, 2.5))), ("-reverse", int(rng.integers(2))),
                 ("-mollfactor", int(rng.integers(1, 4))), ("-x0", float(rng.uniform(0.05, 0.3)))],
         [tuple(float(np.float32(v)) for v in (rng.uniform(0.2, 0.8), rng.uniform(0.2, 0.8), rng.uniform(0.2, 0.8),
                                               rng.uniform(0.05, 0.15))) for _ in range(3)], config),
    ]
    for case, opts, bub, cfg in runs:
        with tempfile.TemporaryDirectory() as w:
            dims, ref = O.ref_case(L, case, opts, w, bubbles=bub, config=cfg)
        out = O.case_ic(case, dims, O.case_prm(case, opts), bub)
        for q in range(7):
            assert np.array_equal(out[q], ref[q]), (case, opts, q)
