"""The reference's compile-time WENO3 build (-D_WENO3_, GPUonly.cuh:102-176)
on the GPU: mpcf_set_weno_order(s, 3) for the two reference-rounding forms.

The FP32 form is compared bit for bit with the oracle's WENO3 (the oracle's
restatement is pinned to the reference's own WENO3 functions, compiled from
GPUonly.cuh with -D_WENO3_), on several shapes, boundary mixes and tilings;
the FP64 form within FP64 rounding of the FP64 oracle."""
import numpy as np
import pytest

import oracle_lib as O
from conftest import cloud_state
from test_gpu_parity import assert_bitwise, rel_linf

pytestmark = pytest.mark.gpu

ABS, REF = 0, 1


@pytest.mark.parametrize("dims,bc,tiling", [
    ((40, 24, 16), (ABS,) * 6, (7, 8, False, True)),
    ((37, 13, 11), (ABS, REF, REF, ABS, ABS, REF), (3, 4, True, False)),
    ((64, 48, 20), (REF, ABS, ABS, REF, REF, ABS), (15, 20, True, True)),
    ((64, 64, 24), (ABS,) * 6, (8, 24, True, True)),
])
def test_weno3_reference_rounding_step_bit_exact(mpcf, dims, bc, tiling):
    U0 = cloud_state(dims, nb=2, seed=31)
    U = [a.copy() for a in U0]
    R = [np.zeros_like(a) for a in U0]
    with mpcf.Solver([dims], bc=[bc], precision="fp32_ref") as s:
        s.set_weno_order(3)
        assert s.weno_order() == 3
        s.set_tiling(*tiling)
        s.set_state(U0, R)
        dt = s.step(cfl=0.3)[0]
        Ug, Rg = s.get_state()
        assert s.error_word() == 0
    with O.weno3():
        dt_o, _ = O.step(dims, bc, U, R, cfl=0.3)
    assert dt == dt_o
    assert_bitwise(Ug, U, f"WENO3 state, tiling {tiling}")
    assert_bitwise(Rg, R, f"WENO3 register, tiling {tiling}")


def test_weno3_differs_from_weno5_and_graphs_follow_the_order(mpcf):
    dims = (48, 32, 24)
    U0 = cloud_state(dims, nb=2, seed=8)
    out = {}
    for order, graph in ((5, True), (3, True), (3, False)):
        with mpcf.Solver([dims], precision="fp32_ref") as s:
            s.set_state(U0)
            s.run(1, graph=True)              # a graph of the WENO5 step exists
            s.set_weno_order(order)
            s.set_state(U0)
            s.run(2, graph=graph)
            out[(order, graph)] = s.get_state(with_reg=False)
    assert_bitwise(out[(3, True)], out[(3, False)], "WENO3 graph against plain steps")
    assert not np.array_equal(out[(3, True)][0], out[(5, True)][0])


def test_weno3_fp64_matches_fp64_oracle(mpcf):
    dims = (30, 22, 14)
    bc = (ABS, REF, ABS, ABS, REF, ABS)
    U0 = cloud_state(dims, nb=2, dtype=np.float64)
    U = [np.array(a) for a in U0]
    R = [np.zeros_like(a) for a in U]
    with mpcf.Solver([dims], bc=[bc], precision="fp64") as s:
        s.set_weno_order(3)
        s.set_state(U, R)
        dt = s.step(cfl=0.3)[0]
        Ug, Rg = s.get_state()
    with O.weno3():
        dt_o, _ = O.step(dims, bc, U, R, cfl=0.3)
    assert abs(dt - dt_o) <= 1e-14 * dt_o
    # the FP64 kernels contract multiply-adds, the oracle does not
    for q in range(7):
        assert rel_linf(Ug[q], U[q]) <= 1e-8, (q, rel_linf(Ug[q], U[q]))
        assert rel_linf(Rg[q], R[q]) <= 1e-5, (q, rel_linf(Rg[q], R[q]))


def test_weno3_only_for_the_reference_rounding_forms(mpcf):
    for prec in ("fp32", "mixed", "fp64_fast"):
        with mpcf.Solver([(32, 16, 16)], precision=prec) as s:
            with pytest.raises(mpcf.MpcfError, match="WENO3"):
                s.set_weno_order(3)
            assert s.weno_order() == 5
    with mpcf.Solver([(32, 16, 16)], precision="fp32_ref") as s:
        with pytest.raises(mpcf.MpcfError):
            s.set_weno_order(4)
