"""GPU generators of the reference's SteadyState, Sod and 2DSBI initial
conditions (mpcf_ic_steady / mpcf_ic_sod / mpcf_ic_sbi) against the
reference's own fields (golden) and the restatement, through the C ABI."""
import os

import numpy as np
import pytest

import oracle_lib as O
from test_cases import golden_cases

pytestmark = pytest.mark.gpu


def gpu_case(mpcf, case, dims, prm, bub, precision="fp32_ref"):
    kw = {k: v for k, v in prm.items()}
    with mpcf.Solver([dims], precision=precision) as s:
        if case == "steady":
            s.ic_steady(**kw)
        elif case == "sod":
            s.ic_sod(**kw)
        else:
            s.ic_sbi(bub if bub is not None else np.zeros((0, 4)), **kw)
        U, R = s.get_state()
    for q in range(7):
        assert not np.any(R[q])
    return U


def assert_case_equal(case, got, want, what):
    for q in range(7):
        if case == "sbi":
            # the mollified interface passes through cosf, which may differ
            # from the C library's in the last place; a last-place change of
            # the indicator (in [0, 1]) moves a mixed field by up to that
            # times the jump across the interface.  Only interface cells may
            # differ, and only by that much.
            d = np.abs(got[q].astype(np.float64) - want[q])
            assert d.max() <= 2.5e-7 * max(np.abs(want[q]).max(), 1e-30), (what, q, float(d.max()))
            assert np.count_nonzero(d) <= 0.05 * d.size, (what, q, int(np.count_nonzero(d)))
        else:
            assert np.array_equal(got[q], want[q]), (what, q)


def test_cases_equal_reference_fields(mpcf):
    for case, prm, dims, bub, U in golden_cases():
        assert_case_equal(case, gpu_case(mpcf, case, dims, prm, bub), U, (case, prm))


@pytest.mark.parametrize("dims", [(25, 21, 15), (9, 40, 17)])
def test_cases_odd_sizes_against_restatement(mpcf, dims):
    """Odd extents, including the unswapped middle plane of a reversed 2DSBI."""
    bub = np.array([[0.5, 0.4, 0.3, 0.12], [0.3, 0.7, 0.6, 0.1]])
    for case, opts in [("steady", [("-rho", 3.0), ("-w", 2.0), ("-pc", 7.0)]),
                       ("sod", [("-config", "z"), ("-reverse", 1)]),
                       ("sbi", [("-config", "xz"), ("-reverse", 1), ("-mollfactor", 2)]),
                       ("sbi", [("-config", "zy"), ("-mach", 1.8)])]:
        prm = O.case_prm(case, opts)
        want = O.case_ic(case, dims, prm, bub if case == "sbi" else None)
        assert_case_equal(case, gpu_case(mpcf, case, dims, prm, bub), want, (case, opts))


def test_cases_fp64(mpcf):
    dims = (20, 18, 12)
    bub = np.array([[0.5, 0.4, 0.3, 0.12]])
    for case, opts in [("steady", [("-rho", 2.0), ("-u", 0.5)]), ("sod", [("-config", "y")]),
                       ("sbi", [("-config", "yx"), ("-reverse", 1)])]:
        prm = O.case_prm(case, opts)
        want = O.case_ic(case, dims, prm, bub if case == "sbi" else None, dtype=np.float64)
        got = gpu_case(mpcf, case, dims, prm, bub, precision="fp64")
        for q in range(7):
            assert np.abs(got[q] - want[q]).max() <= 1e-14 * max(np.abs(want[q]).max(), 1.0), (case, q)


def test_steady_state_with_its_lab_is_invariant(mpcf):
    """Sim_SteadyStateMPI's state with its lab's reflecting walls stays
    bit-identical over LSRK3 steps (known-answer test 1)."""
    dims = (24, 20, 16)
    with mpcf.Solver([dims], bc=[mpcf.case_bc("steady")], precision="fp32_ref") as s:
        s.ic_steady(rho=2.0, p=3.0, g=6.59, pc=4096.0)
        U0 = s.get_state(with_reg=False)
        s.run(3, cfl=0.3, graph=False)
        U = s.get_state(with_reg=False)
    for q in range(7):
        assert np.array_equal(U[q], U0[q]), q


def test_sod_tube_is_symmetric_across_axes(mpcf):
    """The Sod tube along x and along y (transposed domain) evolve
    identically (known-answer test 2, with the case's own IC and lab)."""
    res = {}
    for cfg, dims in (("x", (40, 8, 6)), ("y", (8, 40, 6))):
        with mpcf.Solver([dims], bc=[mpcf.case_bc("sod")], precision="fp32_ref") as s:
            s.ic_sod(config=cfg)
            s.run(4, cfl=0.3, graph=False)
            U = s.get_state(with_reg=False)
        nx, ny, nz = dims
        arr = [a.reshape(nz, ny, nx) for a in U]
        if cfg == "y":
            arr = [a.transpose(0, 2, 1) for a in arr]
            arr[1], arr[2] = arr[2], arr[1]
        res[cfg] = arr
    for q in range(7):
        assert np.array_equal(res["x"][q], res["y"][q]), q


def test_long_runs_stay_physical(mpcf):
    """300 steps of 2DSBI (Mach 1.22, reflecting walls) and 100 steps of the
    steady state: no error bits; the steady state is invariant bit for bit,
    and the mixed form stays within 1e-6 (L1 of rho) of the FP64 run."""
    dims = (192, 96, 8)
    bub = np.array([[0.4, 0.25, 0.02, 0.1], [0.7, 0.2, 0.02, 0.08]])
    rho = {}
    for prec in ("fp64", "mixed"):
        with mpcf.Solver([dims], bc=[mpcf.case_bc("sbi", "xy")], precision=prec) as s:
            s.ic_sbi(bub, config="xy", mollfactor=1)
            s.run(300, cfl=0.3, graph=True)
            assert s.error_word() == 0, prec
            rho[prec] = np.asarray(s.get_state(with_reg=False)[0], np.float64)
    l1 = np.abs(rho["mixed"] - rho["fp64"]).mean() / np.abs(rho["fp64"]).mean()
    assert l1 < 1e-6, l1
    for prec in ("fp32_ref", "mixed", "fp64"):
        with mpcf.Solver([(48, 40, 32)], bc=[mpcf.case_bc("steady")], precision=prec) as s:
            s.ic_steady(rho=2.0, p=3.0)
            U0 = s.get_state(with_reg=False)
            s.run(100, cfl=0.3, graph=True)
            assert s.error_word() == 0, prec
            for a, b in zip(U0, s.get_state(with_reg=False)):
                assert np.array_equal(a, b), prec
