"""CPU tests of the C-ABI library: it loads without a GPU, exports every
symbol include/mpcf_b200.h declares, and its host-only entry points (IC
generator, bubble sampler, argument validation) behave."""
import ctypes
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(REPO, "include", f) for f in sorted(os.listdir(os.path.join(REPO, "include")))
           if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(mpcf_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("mpcf_create", "mpcf_stage", "mpcf_step", "mpcf_max_sos", "mpcf_run", "mpcf_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol(mpcf):
    L = mpcf.lib()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_header(mpcf):
    from mpcf import _lib
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_version_and_elem_size(mpcf):
    L = mpcf.lib()
    assert L.mpcf_version() == 1
    assert L.mpcf_elem_size(mpcf.PREC_FP64) == 8
    assert L.mpcf_elem_size(mpcf.PREC_MIXED) == 4
    assert L.mpcf_elem_size(7) == -1
    assert b"precision" in L.mpcf_last_error()


def test_create_rejects_bad_arguments(mpcf):
    L = mpcf.lib()
    h = ctypes.c_void_p()
    dims = (ctypes.c_int * 3)(4, 8, 8)     # nx below the reference minimum 5
    assert L.mpcf_create(ctypes.byref(h), 1, dims, None, 0, 0) == -1
    assert b"minimum" in L.mpcf_last_error()
    dims = (ctypes.c_int * 3)(8, 8, 8)
    bc = (ctypes.c_int * 6)(0, 0, 0, 0, 0, 5)
    assert L.mpcf_create(ctypes.byref(h), 1, dims, bc, 0, 0) == -1
    assert L.mpcf_create(ctypes.byref(h), 0, dims, None, 0, 0) == -1
    assert L.mpcf_create(ctypes.byref(h), 1, dims, None, 9, 0) == -1
    bc = (ctypes.c_int * 6)(mpcf.BC_HALO, 0, 0, 0, 0, 0)     # halo faces are z faces only
    assert L.mpcf_create(ctypes.byref(h), 1, dims, bc, 0, 0) == -1
    assert b"halo faces are z faces" in L.mpcf_last_error()


def test_bubbles_are_seeded_and_disjoint(mpcf):
    a = mpcf.bubbles(42, 50, 0.02, 0.06)
    b = mpcf.bubbles(42, 50, 0.02, 0.06)
    assert a.shape == (50, 4) and np.array_equal(a, b)
    assert (a[:, :3] >= 0.2).all() and (a[:, :3] <= 0.8).all()
    assert (a[:, 3] >= 0.02).all() and (a[:, 3] <= 0.06).all()
    d = np.sqrt(((a[:, None, :3] - a[None, :, :3]) ** 2).sum(-1))
    rr = a[:, None, 3] + a[None, :, 3]
    iu = np.triu_indices(len(a), 1)
    assert (d[iu] >= rr[iu]).all()
    c = mpcf.bubbles(43, 50, 0.02, 0.06)
    assert not np.array_equal(a, c)


def test_host_ic_cloud_properties(mpcf):
    dims = (32, 24, 16)
    params = mpcf.configs.ic_params(100.0, seed=9)
    bub = np.array([[0.5, 0.35, 0.25, 0.12]])
    U = mpcf.ic_cloud_host(dims, params, bub, np.float32)
    rho, ru, rv, rw, E, G, P = [a.reshape(dims[::-1]) for a in U]
    h = 1.0 / 32
    ic = (int(0.5 / h), int(0.35 / h), int(0.25 / h))          # (x, y, z) near the centre
    # centre cell: phi ~ -0.096, alpha = 0.5*(1 - tanh(phi/(1.5h))) ~ 0.983
    phi = np.sqrt((16.5 * h - 0.5) ** 2 + (11.5 * h - 0.35) ** 2 + (8.5 * h - 0.25) ** 2) - 0.12
    alpha = 0.5 * (1 - np.tanh(phi / (1.5 * h)))
    assert abs(rho[ic[2], ic[1], ic[0]] - (alpha + (1 - alpha) * 1000.0)) < 1e-3
    assert abs(rho[0, 0, 0] - 1000.0) < 1e-3                       # liquid far away
    assert abs(G[0, 0, 0] - 1 / 5.59) < 1e-6
    assert abs(G[ic[2], ic[1], ic[0]] - (alpha * 2.5 + (1 - alpha) / 5.59)) < 1e-5
    u = ru / rho
    assert np.abs(u).max() <= 1e-3 * (1 + 1e-6)
    p = (E - 0.5 * (ru * ru + rv * rv + rw * rw) / rho - P) / G
    assert abs(p[0, 0, 0] - 100.0) < 5e-2
    # the counter-based noise does not depend on the domain: same seed, same cell index
    U2 = mpcf.ic_cloud_host(dims, params, bub, np.float64)
    assert np.allclose(U2[1], U[1], rtol=1e-6, atol=1e-9)


def test_configs_build(mpcf):
    c1 = mpcf.configs.config("c1_64")
    assert c1["dims"] == [(64, 64, 64)] and c1["bubbles"][0].shape == (1, 4)
    c2 = mpcf.configs.config("c2_256")
    assert c2["bubbles"][0].shape == (50, 4)
    c4 = mpcf.configs.config("c4_ensemble")
    assert len(c4["dims"]) == 64
    assert all(e in (32, 48, 64, 96, 128) for d in c4["dims"] for e in d)
    assert all(1 <= len(b) <= 8 for b in c4["bubbles"])


def test_dropin_driver_library_loads():
    """The reference integrator + shim driver (oracle/_ref, built where the
    reference tree is present) resolves all its symbols against
    libmpcf_b200 without a GPU."""
    p = os.path.join(REPO, "oracle", "_ref", "libref_lsrk3_driver.so")
    if not os.path.exists(p):
        pytest.skip("oracle/_ref not built")
    L = ctypes.CDLL(p)
    d = (ctypes.c_int * 3)()
    L.drv_dims(d)
    assert (d[0], d[1], d[2]) == (32, 24, 16)
