"""GPU parity at the benchmark configurations' own sizes and tilings.

The bench advances 256^3 and 512^3 bubble clouds with whole-column
persistent tilings and the autotuner's choice, and the 64-domain ensemble in
one launch.  Here one full LSRK3 step of each, from the oracle's own
initial condition (the oracle's restatement of the cloud set-up, uploaded
as is), is compared with the CPU oracle:

* FP32 reference rounding at 256^3 (configuration 2's cloud): bit for bit
  against the oracle's whole-domain step, on the autotuned tiling, on
  32x15 tiles with 32-slab chunks and on 32x8 tiles over whole columns,
  all persistent with bulk-copy staging.
* FP32 reference rounding at 512^3 (configuration 3's cloud) with the
  bench's tilings: bit for bit on three z-windows of the domain (its first
  32, middle 64 and last 32 planes).  The oracle advances each window from
  the initial planes within 9 of it (3 per stage; planes outside the
  domain are the domain's own boundary) with the whole domain's time step,
  so the window's planes are exact: a stage reads 3 planes beyond a cell.
* The fast FP32 and mixed forms at 256^3 against the FP64 oracle's step:
  every stored field at least as close to it as the reference rounding is,
  in relative L-inf and L1.
* The 64-domain ensemble of configuration 4 (reference rounding, one
  persistent launch per stage, per-domain time steps): every domain bit
  for bit against the oracle's step of that domain alone.
"""
import numpy as np
import pytest

import oracle_lib as O
from test_gpu_parity import assert_bitwise, rel_linf

pytestmark = pytest.mark.gpu

CFL = 0.3
# LSRK3_IntegratorMPI.cpp:46,51,56
LSRK3 = ((0.0, 1.0 / 4), (-17.0 / 32, 8.0 / 9), (-32.0 / 27, 3.0 / 4))
ABS6 = (0,) * 6


def oracle_cfg(mpcf, name):
    return mpcf.configs.config(name, placer=O.bubbles)


def gpu_step(mpcf, dims, prec, U0, tiling):
    """One LSRK3 step on the GPU from U0 (register zero); tiling (ty, dz,
    persistent, tma) or "auto" (the autotuner on this state).  Returns (dt,
    U, R, tiling used)."""
    dtype = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    with mpcf.Solver([dims], precision=prec) as s:
        s.set_state([np.asarray(a, dtype) for a in U0], [np.zeros(a.size, dtype) for a in U0])
        if tiling == "auto":
            s.set_tiling(*s.autotune(reps=1)[0])
        else:
            s.set_tiling(*tiling)
        dt = s.step(cfl=CFL)[0]
        U, R = s.get_state()
        assert s.error_word() == 0
        return dt, U, R, s.tiling()


@pytest.fixture(scope="module")
def c2_ref(mpcf):
    """Configuration 2's initial state and the oracle's FP32 step of it."""
    cfg = oracle_cfg(mpcf, "c2_256")
    dims = cfg["dims"][0]
    U0 = O.ic_cloud(dims, cfg["params"], cfg["bubbles"][0], np.float32)
    U = [a.copy() for a in U0]
    R = [np.zeros_like(a) for a in U0]
    dt, _ = O.step(dims, ABS6, U, R, cfl=CFL)
    return dims, U0, dt, U, R


@pytest.mark.parametrize("tiling", ["auto", (15, 32, True, True), (8, 256, True, True)])
def test_config2_256cube_reference_rounding_bit_exact(mpcf, c2_ref, tiling):
    dims, U0, dt_o, Uo, Ro = c2_ref
    dt, U, R, used = gpu_step(mpcf, dims, "fp32_ref", U0, tiling)
    assert dt == dt_o, (used, dt, dt_o)
    assert_bitwise(U, Uo, f"state, tiling {used}")
    assert_bitwise(R, Ro, f"register, tiling {used}")


def window_step(dims, U0, z0, z1, dtinvh, margin=9):
    """The oracle's FP32 step of planes z0..z1-1 of a domain (absorbing
    boundaries): it advances the planes within `margin` of the window and
    returns the window's planes of the state and the register."""
    nx, ny, nz = dims
    lo, hi = max(0, z0 - margin), min(nz, z1 + margin)
    n = nx * ny
    U = [a[lo * n:hi * n].copy() for a in U0]
    R = [np.zeros_like(a) for a in U]
    wd = (nx, ny, hi - lo)
    for a, b in LSRK3:
        O.stage(wd, ABS6, U, R, a, b, dtinvh)
    s = slice((z0 - lo) * n, (z1 - lo) * n)
    return [a[s] for a in U], [a[s] for a in R]


@pytest.fixture(scope="module")
def c3_ref(mpcf):
    cfg = oracle_cfg(mpcf, "c3_512")
    dims = cfg["dims"][0]
    U0 = O.ic_cloud(dims, cfg["params"], cfg["bubbles"][0], np.float32)
    # the whole domain's time step, as the GPU step computes it
    # (LSRK3_IntegratorMPI.cpp:27-62 with the CUDA sound speed)
    sos = np.float32(O.max_sos(U0))
    h = 1.0 / max(dims)
    dt = CFL * h / float(sos)
    return dims, U0, dt, h


@pytest.mark.parametrize("tiling", [(15, 32, True, True), (8, 512, True, True)])
def test_config3_512cube_reference_rounding_bit_exact_on_windows(mpcf, c3_ref, tiling):
    dims, U0, dt_o, h = c3_ref
    dt, U, R, used = gpu_step(mpcf, dims, "fp32_ref", U0, tiling)
    assert dt == dt_o, (used, dt, dt_o)
    n = dims[0] * dims[1]
    nz = dims[2]
    for z0, z1 in ((0, 32), (nz // 2 - 32, nz // 2 + 32), (nz - 32, nz)):
        Uw, Rw = window_step(dims, U0, z0, z1, float(np.float32(dt / h)))
        s = slice(z0 * n, z1 * n)
        assert_bitwise([a[s] for a in U], Uw, f"state planes {z0}-{z1 - 1}, tiling {used}")
        assert_bitwise([a[s] for a in R], Rw, f"register planes {z0}-{z1 - 1}, tiling {used}")


@pytest.fixture(scope="module")
def c2_fp64(mpcf, c2_ref):
    dims, U0 = c2_ref[0], c2_ref[1]
    U = [a.astype(np.float64) for a in U0]
    R = [np.zeros_like(a) for a in U]
    dt, _ = O.step(dims, ABS6, U, R, cfl=CFL)
    return dt, U, R


def rel_l1(a, b):
    return float(np.abs(a.astype(np.float64) - b).mean() / max(np.abs(b).mean(), 1e-300))


@pytest.mark.parametrize("prec", ["mixed", "fp32"])
def test_config2_256cube_fast_forms_track_fp64_oracle(mpcf, c2_ref, c2_fp64, prec):
    """One step from the same FP32 state: every stored field of the fast form
    is at least as close to the FP64 oracle's step as the reference's own
    FP32 rounding is (the oracle's FP32 step, which the GPU reproduces bit
    for bit), in relative L-inf and in relative L1, and within 1e-3 relative
    L-inf; the register within 1e-2.  (Reference rounding against FP64 after
    this step: momenta 8e-4 L-inf / 1.8e-4 L1, rho and E 6e-7, G and P 2e-7.)"""
    dims, U0, _, Uref, Rref = c2_ref
    dt64, U64, R64 = c2_fp64
    dt, U, R, used = gpu_step(mpcf, dims, prec, U0, "auto")
    assert abs(dt - dt64) <= 1e-6 * dt64, (dt, dt64)
    for q in range(7):
        e_inf, e_ref = rel_linf(U[q], U64[q]), rel_linf(Uref[q], U64[q])
        e_l1, e_l1ref = rel_l1(U[q], U64[q]), rel_l1(Uref[q], U64[q])
        assert e_inf <= e_ref and e_inf <= 1e-3, (used, q, e_inf, e_ref)
        assert e_l1 <= e_l1ref, (used, q, e_l1, e_l1ref)
        assert rel_linf(R[q], R64[q]) <= 1e-2, (used, q, rel_linf(R[q], R64[q]))


def test_config2_256cube_fast_fp64_matches_fp64_oracle(mpcf, c2_ref, c2_fp64):
    """The fast FP64 form (factored algebra, refined reciprocals) against the
    FP64 oracle (the reference's expanded algebra in double) after one step
    of configuration 2: within 1e-8 of each field's maximum (the oracle's
    expanded indicators cancel to ~1e-12 absolute against epsilon 1e-6)."""
    dims, U0 = c2_ref[0], c2_ref[1]
    dt64, U64, R64 = c2_fp64
    dt, U, R, used = gpu_step(mpcf, dims, "fp64_fast", [a.astype(np.float64) for a in U0], "auto")
    assert abs(dt - dt64) <= 1e-14 * dt64, (dt, dt64)
    for q in range(7):
        assert rel_linf(U[q], U64[q]) <= 1e-8, (used, q, rel_linf(U[q], U64[q]))
        assert rel_linf(R[q], R64[q]) <= 1e-5, (used, q, rel_linf(R[q], R64[q]))


def test_config4_ensemble_one_step_bit_exact(mpcf):
    cfg = oracle_cfg(mpcf, "c4_ensemble")
    dims = cfg["dims"]
    U0 = [O.ic_cloud(d, cfg["params"], b, np.float32) for d, b in zip(dims, cfg["bubbles"])]
    with mpcf.Solver(dims, precision="fp32_ref") as s:
        for d in range(len(dims)):
            s.set_state(U0[d], [np.zeros_like(a) for a in U0[d]], dom=d)
        s.set_tiling(*s.autotune(reps=1)[0])
        dts = s.step(cfl=CFL)
        got = [s.get_state(dom=d) for d in range(len(dims))]
        assert s.error_word() == 0
        used = s.tiling()
    for d in range(len(dims)):
        U = [a.copy() for a in U0[d]]
        R = [np.zeros_like(a) for a in U]
        dt_o, _ = O.step(dims[d], ABS6, U, R, cfl=CFL)
        assert dts[d] == dt_o, (d, dts[d], dt_o)
        assert_bitwise(got[d][0], U, f"domain {d} {dims[d]} state, tiling {used}")
        assert_bitwise(got[d][1], R, f"domain {d} {dims[d]} register, tiling {used}")
