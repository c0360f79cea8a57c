"""The arrays of the reference's dump and save (the output streamers of
source/Types.h:192-277, as DumpHDF5_MPI lays them out), on the CPU: the
restatement in oracle_lib.pack against the reference's own streamers,
through the golden record (tests/golden/ref_dump.npz) and live where
oracle/_ref was built here."""
import os

import numpy as np
import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_dump.npz")


@pytest.mark.parametrize("kind", ["tensor", "save"])
def test_golden_dump_arrays(kind):
    g = np.load(GOLD)
    U = list(g["U"])
    got = O.pack(U, (12, 10, 8), kind)
    assert got.shape == g[kind].shape
    assert np.array_equal(got, g[kind])


def test_live_dump_arrays():
    L = O.ref_lib("libref_dump_12x10x8")
    if L is None:
        pytest.skip("oracle/_ref not built (the reference tree is absent)")
    rng = np.random.default_rng(3)
    n = 12 * 10 * 8
    rho = rng.uniform(0.5, 1200, n).astype(np.float32)
    U = [rho] + [(rho * rng.uniform(-20, 20, n)).astype(np.float32) for _ in range(3)]
    G = rng.uniform(0.15, 2.5, n).astype(np.float32)
    P = rng.uniform(0, 5000, n).astype(np.float32)
    ke = 0.5 * (U[1].astype(np.float64) ** 2 + U[2] ** 2 + U[3] ** 2) / rho
    E = (G * rng.uniform(0.01, 1000, n) + P + ke).astype(np.float32)
    U += [E, G, P]
    for kind in ("tensor", "save"):
        assert np.array_equal(O.pack(U, (12, 10, 8), kind), O.ref_pack(L, kind, U)), kind
    # the restart direction is the identity on the save array
    back = [np.zeros(n, np.float32) for _ in range(7)]
    arr = np.ascontiguousarray(O.ref_pack(L, "save", U)).reshape(-1)
    L.ref_unpack_save(arr.ctypes.data_as(O._PF), O.fptrs(back))
    for q in range(7):
        assert np.array_equal(back[q], U[q])
