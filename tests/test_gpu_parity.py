"""GPU parity: the sm_100a kernels through the C ABI against the CPU oracle.

MPCF_PREC_FP32_REF is compared bit for bit (rounding of the reference
source, FP32 with its double-promoted sub-expressions); the fast FP32 and
mixed forms within the stated tolerances; FP64 against the FP64 oracle.
Metric for the tolerance tests (the reference's parity metric): per stored
field and register, max|x_gpu - x_oracle| / max|x_oracle|.
"""
import numpy as np
import pytest

import oracle_lib as O
from conftest import cloud_state

pytestmark = pytest.mark.gpu

ABS, REF = 0, 1


def rel_linf(a, b):
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max() / den)


def assert_bitwise(got, want, what):
    for q in range(7):
        g, w = got[q], want[q]
        bad = ~((g == w) | (np.isnan(g) & np.isnan(w)))
        if bad.any():
            i = int(np.flatnonzero(bad)[0])
            raise AssertionError(f"{what} field {q}: {int(bad.sum())} cells differ; first at {i}: "
                                 f"gpu={g[i]!r} oracle={w[i]!r} (rel linf {rel_linf(g, w):.3e})")


def run_pair(mpcf, dims, bc, prec, U0, R0=None, stages=((0.0, 0.25, 0.05),), tiling=None):
    """Run stages on GPU and oracle from the same inputs; return (gpu, oracle)."""
    dtype = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    U = [np.array(a, dtype=dtype) for a in U0]
    R = [np.zeros_like(a) for a in U] if R0 is None else [np.array(a, dtype=dtype) for a in R0]
    with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
        if tiling:
            s.set_tiling(*tiling)
        s.set_state(U, R)
        for a, b, dtinvh in stages:
            s.stage(a, b, dtinvh)
        Ug, Rg = s.get_state()
        assert s.error_word() == 0
    for a, b, dtinvh in stages:
        O.stage(dims, bc, U, R, a, b, dtinvh)
    return (Ug, Rg), (U, R)


# ---------------------------------------------------------------------------
# bit-exact reference-rounding path
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dims,bc", [
    ((8, 7, 6), (ABS,) * 6),
    ((8, 7, 6), (REF,) * 6),
    ((37, 13, 11), (ABS, REF, REF, ABS, ABS, REF)),
    ((5, 5, 3), (REF, ABS, ABS, REF, REF, ABS)),
    ((64, 9, 20), (ABS,) * 6),
])
def test_ref32_stage_bitexact(mpcf, dims, bc):
    U0 = cloud_state(dims, nb=2)
    R0 = [np.asarray(a) * np.float32(1e-3) for a in cloud_state(dims, nb=1, seed=5)]
    stages = [(0.0, 0.25, 0.057), (-17.0 / 32, 8.0 / 9, 0.057), (-32.0 / 27, 0.75, 0.057)]
    (Ug, Rg), (Uo, Ro) = run_pair(mpcf, dims, bc, "fp32_ref", U0, R0, stages)
    assert_bitwise(Ug, Uo, "state")
    assert_bitwise(Rg, Ro, "register")


@pytest.mark.parametrize("tiling", [(3, 3, False, False), (3, 64, False, True), (7, 5, True, True), (15, 7, False, True),
                                    (3, 1, True, True), (7, 9, True, False), (15, 2, True, True), (8, 4, True, True),
                                    (8, 64, False, False), (3, 5, False, True)])
@pytest.mark.parametrize("dims", [(45, 19, 14), (44, 19, 14)])
def test_ref32_tiling_invariant(mpcf, tiling, dims):
    # rows of 45 floats are not 16-byte multiples (ordinary loads even with
    # the TMA flag); rows of 44 are, so TMA tilings stage with bulk copies,
    # including partial tiles in x and y and reflecting edges
    bc = (ABS, REF, ABS, ABS, REF, ABS)
    U0 = cloud_state(dims, nb=3)
    (Ug, Rg), (Uo, Ro) = run_pair(mpcf, dims, bc, "fp32_ref", U0, tiling=tiling)
    assert_bitwise(Ug, Uo, f"state tiling={tiling}")
    assert_bitwise(Rg, Ro, f"register tiling={tiling}")


def test_ref32_lsrk3_step_64cube(mpcf):
    """Configuration 1: 64^3, one bubble, one LSRK3 step at CFL 0.3, absorbing."""
    cfg = mpcf.configs.config("c1_64")
    dims = cfg["dims"][0]
    bc = (ABS,) * 6
    U = mpcf.ic_cloud_host(dims, cfg["params"], cfg["bubbles"][0], np.float32)
    R = [np.zeros_like(a) for a in U]
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(U, R)
        dt_gpu = s.step(cfl=0.3)[0]
        Ug, Rg = s.get_state()
        assert s.error_word() == 0
    dt_o, sos_o = O.step(dims, bc, U, R, cfl=0.3)
    assert dt_gpu == dt_o
    assert_bitwise(Ug, U, "state")
    assert_bitwise(Rg, R, "register")
    for q in range(7):   # the stated parity metric, trivially met when bit-exact
        assert rel_linf(Ug[q], U[q]) <= 1e-5


def test_ref32_drop_in_lab_driver(mpcf):
    """LSRK3_IntegratorMPI::operator() shape driving the GPUlab mirror."""
    dims = (24, 20, 16)
    U = cloud_state(dims, nb=2)
    R = [np.zeros_like(a) for a in U]
    host_U = [a.copy() for a in U]
    host_R = [a.copy() for a in R]
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(U, R)
        lab = mpcf.GPUlab(s, nslices=dims[2], host_state=host_U, host_reg=host_R, sync_host=True)
        dt = mpcf.lsrk3_step(lab, 1.0 / max(dims), 0.3)
    dt_o, _ = O.step(dims, (ABS,) * 6, U, R, cfl=0.3)
    assert dt == dt_o
    assert_bitwise(host_U, U, "state")
    assert_bitwise(host_R, R, "register")


def test_sos_matches_oracle(mpcf):
    dims = (33, 17, 9)
    U = cloud_state(dims, nb=2)
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(U)
        sos = s.max_sos()[0]
    assert np.float32(sos) == np.float32(O.max_sos([np.asarray(a) for a in U]))


def test_ghost_fill_matches_oracle(mpcf):
    dims = (11, 9, 7)
    U = cloud_state(dims, nb=1)
    for bc in [(ABS,) * 6, (REF,) * 6, (ABS, REF, REF, ABS, REF, ABS)]:
        with mpcf.Solver([dims], bc=[bc], precision="fp32_ref") as s:
            s.set_state(U)
            gx, gy, gz = s.fill_ghosts()
        ox, oy, oz = O.fill_ghosts(dims, bc, [np.asarray(a) for a in U])
        assert np.array_equal(gx, ox) and np.array_equal(gy, oy) and np.array_equal(gz, oz)


def test_graph_and_plain_steps_agree(mpcf):
    dims = (40, 24, 18)
    U = cloud_state(dims, nb=2)
    outs = []
    for graph in (False, True):
        with mpcf.Solver([dims], precision="fp32_ref") as s:
            s.set_state(U)
            t = s.run(4, cfl=0.3, graph=graph)
            outs.append((t, s.get_state()))
    assert outs[0][0] == outs[1][0]
    assert_bitwise(outs[0][1][0], outs[1][1][0], "graph vs plain state")


def test_ensemble_matches_single_domains(mpcf):
    dims = [(32, 16, 8), (21, 30, 12), (48, 8, 10)]
    bcs = [(ABS,) * 6, (REF,) * 6, (ABS, REF, ABS, REF, ABS, REF)]
    states = [cloud_state(d, nb=2, seed=3 + i) for i, d in enumerate(dims)]
    with mpcf.Solver(dims, bc=bcs, precision="fp32_ref") as s:
        s.set_tiling(3, 8, True)
        for i, U in enumerate(states):
            s.set_state(U, dom=i)
        dts = s.step(cfl=0.3)
        got = [s.get_state(dom=i) for i in range(len(dims))]
    for i, d in enumerate(dims):
        U = [np.array(a) for a in states[i]]
        R = [np.zeros_like(a) for a in U]
        dt_o, _ = O.step(d, bcs[i], U, R, cfl=0.3)
        assert dts[i] == dt_o
        assert_bitwise(got[i][0], U, f"domain {i} state")
        assert_bitwise(got[i][1], R, f"domain {i} register")


# ---------------------------------------------------------------------------
# fast FP32, mixed and FP64
# ---------------------------------------------------------------------------
FAST_TILINGS = [(3, 3, False, False), (3, 64, False, True), (7, 5, True, True), (7, 9, True, False),
                (7, 64, False, True), (8, 4, True, True), (8, 64, False, False), (8, 7, True, True), (8, 4, False, True)]


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
@pytest.mark.parametrize("dims", [(45, 19, 14), (44, 19, 14)])
def test_fast_forms_every_tiling_tracks_fp64_oracle(mpcf, prec, dims):
    """The fast forms reconstruct both edge values of a cell at once and
    evaluate the faces in a second pass; the tile's edge cells (ghost rows and
    columns) come from other warps than its interior.  One stage on every
    tiling -- partial tiles, 44 (bulk copies) and 45 (ordinary loads) wide
    rows, reflecting edges -- stays within FP32 rounding of the FP64 oracle,
    and the tilings agree with one another bit for bit (every cell and face
    of a direction goes through the same code whichever warp evaluates it)."""
    bc = (ABS, REF, ABS, ABS, REF, ABS)
    U64 = [np.asarray(a, dtype=np.float64) for a in cloud_state(dims, nb=3)]
    U = [a.copy() for a in U64]
    R = [np.zeros_like(a) for a in U]
    stage = (0.0, 0.25, 0.05)
    O.stage(dims, bc, U, R, *stage)
    U32 = [a.astype(np.float32) for a in U64]
    first = None
    for tiling in FAST_TILINGS:
        with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
            s.set_tiling(*tiling)
            s.set_state(U32)
            s.stage(*stage)
            Ug, Rg = s.get_state()
            assert s.error_word() == 0
        # FP32 pressure recovery cancels on liquid cells (p ~ 1e2 against
        # E, P ~ 1e4): the fast FP32 form's state is ~1e-4 off FP64 there,
        # below the reference rounding's own ~3e-4; the mixed form recovers
        # the pressure in compensated FP32 and stays at FP32 rounding
        tol_u = 2e-4 if prec == "fp32" else 2e-6
        for q in range(7):
            assert rel_linf(Ug[q], U[q]) <= tol_u, (tiling, q, rel_linf(Ug[q], U[q]))
            assert rel_linf(Rg[q], R[q]) <= 2e-3, (tiling, q, rel_linf(Rg[q], R[q]))
        if first is None:
            first = (Ug, Rg)
        else:
            assert_bitwise(Ug, first[0], f"state, tiling {tiling} vs {FAST_TILINGS[0]}")
            assert_bitwise(Rg, first[1], f"register, tiling {tiling} vs {FAST_TILINGS[0]}")


@pytest.mark.parametrize("prec", ["fp64", "fp64_fast"])
def test_fp64_matches_fp64_oracle(mpcf, prec):
    """Both FP64 forms: the reference-rounding one and the fast one (the fast
    forms' factored algebra in double, refined reciprocals)."""
    dims = (30, 22, 14)
    bc = (ABS, REF, ABS, ABS, REF, ABS)
    U0 = cloud_state(dims, nb=2, dtype=np.float64)
    U = [np.array(a) for a in U0]
    R = [np.zeros_like(a) for a in U]
    with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
        s.set_state(U, R)
        dt = s.step(cfl=0.3)[0]
        Ug, Rg = s.get_state()
    dt_o, _ = O.step(dims, bc, U, R, cfl=0.3)
    assert abs(dt - dt_o) <= 1e-14 * dt_o
    # FP64 tolerance: the GPU contracts multiply-adds, the oracle does not.
    # WENO weights 1/(10(beta+1e-6)^2) amplify last-bit differences of the
    # smoothness indicators where beta ~ 1e-6, so 1e-16 rounding shows up at
    # ~1e-12 of the field maximum after one step.
    # Even in FP64 the reference's expanded smoothness indicators lose ~1e-12
    # absolute to cancellation on liquid stencils, against epsilon = 1e-6, so
    # contraction differences reach ~1e-9 of a field's maximum after a step.
    # The register holds the last stage's increment (~1e-4 of the state), so
    # its bound is looser by that factor.
    for q in range(7):
        assert rel_linf(Ug[q], U[q]) <= 1e-8, (q, rel_linf(Ug[q], U[q]))
        assert rel_linf(Rg[q], R[q]) <= 1e-5, (q, rel_linf(Rg[q], R[q]))


def rel_l1(a, b):
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).mean() / max(np.abs(b).mean(), 1e-300))


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_fast_forms_at_least_as_accurate_as_reference_rounding(mpcf, prec):
    """The fast FP32 and mixed forms are not bit-exact to the reference by
    design (factored smoothness indicators, single-precision weights, fused
    multiply-adds, compensated pressure in the mixed form).  The reference's own
    FP32 indicators cancel ~1e4-sized products down to ~epsilon on smooth
    liquid stencils, so its results carry rounding noise of O(local
    variation); the right yardstick is the FP64 oracle.  After one LSRK3
    step from the same inputs the fast forms are at least as close to it
    as the reference rounding (L1 of each stored field), and within 1e-3
    pointwise of the reference-rounding result."""
    dims = (40, 26, 18)
    U64 = [np.asarray(a) for a in cloud_state(dims, nb=2, dtype=np.float64)]
    U = [a.copy() for a in U64]
    R = [np.zeros_like(a) for a in U]
    O.step(dims, (ABS,) * 6, U, R, cfl=0.3)               # FP64 truth
    U32 = [a.astype(np.float32) for a in U64]
    got = {}
    for p in ("fp32_ref", prec):
        with mpcf.Solver([dims], precision=p) as s:
            s.set_state(U32)
            s.step(cfl=0.3)
            got[p] = s.get_state(with_reg=False)
    for q in range(7):
        e_ref = rel_l1(got["fp32_ref"][q], U[q])
        e_fast = rel_l1(got[prec][q], U[q])
        assert e_fast <= 1.5 * e_ref + 1e-9, (q, e_fast, e_ref)
        assert rel_linf(got[prec][q], got["fp32_ref"][q]) <= 1e-3, q


def test_fast_forms_track_fp64(mpcf):
    """Accuracy against the all-FP64 run after 3 steps of a bubble cloud:
    the mixed form's L1 error of rho is at most 1e-6 and not worse than the
    reference-rounding FP32 path's."""
    dims = (48, 40, 32)
    U64 = cloud_state(dims, nb=3, dtype=np.float64)
    res = {}
    for prec in ("fp64", "fp32_ref", "mixed"):
        dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
        with mpcf.Solver([dims], precision=prec) as s:
            s.set_state([a.astype(dt) for a in U64])
            s.run(3, cfl=0.3, graph=True)
            res[prec] = s.get_state(with_reg=False)
    e_ref = rel_l1(res["fp32_ref"][0], res["fp64"][0])
    e_mix = rel_l1(res["mixed"][0], res["fp64"][0])
    assert e_mix <= 1e-6, e_mix
    assert e_mix <= 1.5 * e_ref + 1e-9, (e_mix, e_ref)


def test_fast_forms_track_fp64_over_many_steps(mpcf):
    """A longer run (40 steps, the bubbles start to collapse): the fast forms
    stay physical and within 1e-5 of the all-FP64 run in L1 of every
    conserved field relative to its mean magnitude, and the mixed form stays
    at least as close as the reference rounding in rho."""
    dims = (64, 48, 40)
    U64 = cloud_state(dims, nb=4, dtype=np.float64, p_liquid=1000.0)
    res, t = {}, {}
    for prec in ("fp64", "fp32_ref", "fp32", "mixed"):
        dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
        with mpcf.Solver([dims], precision=prec) as s:
            s.set_state([a.astype(dt) for a in U64])
            t[prec] = s.run(40, cfl=0.3, graph=True)[0]
            res[prec] = s.get_state(with_reg=False)
            assert s.error_word() == 0, prec
    for prec in ("fp32", "mixed"):
        assert abs(t[prec] - t["fp64"]) <= 1e-5 * t["fp64"], (prec, t[prec], t["fp64"])
        for q in (0, 4, 5, 6):
            e = rel_l1(res[prec][q], res["fp64"][q])
            assert e <= 1e-5, (prec, q, e)
    assert rel_l1(res["mixed"][0], res["fp64"][0]) <= 1.5 * rel_l1(res["fp32_ref"][0], res["fp64"][0]) + 1e-9


def test_convection_then_update_equals_fused_stage(mpcf):
    """Convection_CUDA (stage with b = 0) followed by Update_CUDA (mpcf_update)
    is bit-identical to one fused stage, like the reference's two kernels."""
    dims = (36, 20, 12)
    U0 = cloud_state(dims, nb=2)
    R0 = [np.asarray(a) * np.float32(1e-3) for a in cloud_state(dims, nb=1, seed=5)]
    a, b, dtinvh = -17.0 / 32, 8.0 / 9, 0.05
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(U0, R0)
        s.stage(a, 0.0, dtinvh)
        s.update(b)
        Us, Rs = s.get_state()
    (Uf, Rf), _ = run_pair(mpcf, dims, (ABS,) * 6, "fp32_ref", U0, R0, stages=[(a, b, dtinvh)])
    assert_bitwise(Us, Uf, "state")
    assert_bitwise(Rs, Rf, "register")


def test_error_word_flags_nonphysical(mpcf):
    """A state with negative density raises the device error bit, no fault."""
    dims = (16, 8, 6)
    U = cloud_state(dims, nb=1)
    U[0][5] = -1.0
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(U)
        s.stage(0.0, 0.25, 0.05)
        w = s.error_word(clear=True)
        assert w & mpcf._lib.ERRBIT_NONPHYSICAL
        assert s.error_word() == 0


@pytest.mark.parametrize("prec", ["fp32_ref", "fp32", "mixed", "fp64", "fp64_fast"])
def test_pure_gas_round_off_is_not_flagged(mpcf, prec):
    """A bubble deep enough to hold pure gas (P = 0 exactly, as at the
    centre of the 512^3 cloud's larger bubbles) is a physical state after
    an update, where P there may be left at round-off below zero: the error
    word stays clear and p + pc stays positive everywhere."""
    dims = (96, 96, 96)
    params = mpcf.configs.ic_params(1000.0)
    bub = np.array([[0.5, 0.5, 0.5, 0.35], [0.15, 0.2, 0.8, 0.1]])
    with mpcf.Solver([dims], precision=prec) as s:
        s.ic_cloud(params, bub)
        assert np.count_nonzero(s.get_state(with_reg=False)[6] == 0) > 0     # pure gas
        s.run(3, cfl=0.3, graph=True)
        w = s.error_word()
        r, ru, rv, rw, E, G, P = [np.asarray(a, np.float64) for a in s.get_state(with_reg=False)]
    assert w == 0, (hex(w), int(np.count_nonzero(P < 0)), P.min())
    p = (E - 0.5 * (ru * ru + rv * rv + rw * rw) / r - P) / G
    assert (p + P / (1 + G)).min() > 0


def test_error_word_flags_a_state_without_sound_speed(mpcf):
    """One liquid cell with p = -2 pc has positive rho, E and G but no real
    sound speed: the sound-speed bit is raised, without a fault."""
    dims = (16, 8, 6)
    n = dims[0] * dims[1] * dims[2]
    g, pc = 6.59, 4096.0
    G, P = 1.0 / (g - 1.0), g * pc / (g - 1.0)
    U = [np.full(n, 1000.0, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32),
         np.zeros(n, np.float32), np.full(n, G * 100.0 + P, np.float32), np.full(n, G, np.float32),
         np.full(n, P, np.float32)]
    U[4][77] = G * (-2.0 * pc) + P          # E > 0, p + pc = -pc
    assert U[4][77] > 0
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(U)
        s.step(cfl=0.3)
        w = s.error_word(clear=True)
        assert w & mpcf._lib.ERRBIT_SOS, hex(w)
        assert s.error_word() == 0


@pytest.mark.parametrize("prec", ["fp32_ref", "mixed"])
@pytest.mark.parametrize("tiling", [(3, 64, False, True), (7, 64, True, True), (7, 5, False, False),
                                    (8, 64, True, True), (8, 5, False, False)])
def test_fused_sound_speed_every_tiling(mpcf, prec, tiling):
    """Steps 2 and 3 take dt from the sound speed that the previous step's
    last stage accumulated; a solver whose state is set again before every
    step measures it with the stand-alone reduction instead.  Both give the
    same dt and state bit for bit on tiles with and without a helper warp."""
    dims = (40, 24, 16)
    U = cloud_state(dims, nb=3)
    with mpcf.Solver([dims], precision=prec) as s:
        s.set_tiling(*tiling)
        s.set_state(U)
        dts = [s.step(cfl=0.3)[0] for _ in range(3)]
        Uf, Rf = s.get_state()
    dts1 = []
    with mpcf.Solver([dims], precision=prec) as s1:
        s1.set_tiling(*tiling)
        s1.set_state(U)
        for _ in range(3):
            dts1.append(s1.step(cfl=0.3)[0])
            st, reg = s1.get_state()
            s1.set_state(st, reg)
        U1, R1 = s1.get_state()
    assert dts == dts1, (dts, dts1)
    assert_bitwise(Uf, U1, f"fused vs stand-alone sound speed, tiling={tiling}")
    assert_bitwise(Rf, R1, f"fused vs stand-alone sound speed, tiling={tiling}")


def test_fused_sound_speed_follows_state_changes(mpcf):
    """The last stage of a step accumulates the next step's sound speed; a
    state replaced between steps must be re-measured (the stand-alone
    reduction), in graph and plain runs alike."""
    dims = (40, 24, 16)
    U = cloud_state(dims, nb=3)
    U2 = cloud_state(dims, nb=1, seed=99, p_liquid=1000.0)
    for graph in (True, False):
        with mpcf.Solver([dims], precision="fp32_ref") as s:
            s.set_state(U)
            s.run(2, cfl=0.3, graph=graph)
            s.set_state(U2)
            s.run(2, cfl=0.3, graph=graph)
            Ug = s.get_state(with_reg=False)
        with mpcf.Solver([dims], precision="fp32_ref") as s1:
            s1.set_state(U2)
            s1.run(2, cfl=0.3, graph=not graph)
            U1 = s1.get_state(with_reg=False)
        Uo, Ro = [a.copy() for a in U2], [np.zeros_like(a) for a in U2]
        for _ in range(2):
            O.step(dims, (ABS,) * 6, Uo, Ro, cfl=0.3)
        assert_bitwise(Ug, U1, f"graph={graph} vs fresh solver")
        assert_bitwise(Ug, Uo, f"graph={graph} vs oracle")


def test_autotune_leaves_the_state_and_picks_shallow_chunks_on_small_domains(mpcf):
    """The autotuner times its candidates on the solver's own state and
    leaves it unchanged.  On a 64^3 domain, whose 16-deep chunks fill less
    than one wave of resident CTAs, it also tries shallower chunks, and
    one of those wins."""
    dims = (64, 64, 64)
    U0 = cloud_state(dims, nb=1)
    with mpcf.Solver([dims], precision="mixed") as s:
        s.set_state(U0)
        best, ms = s.autotune(reps=2)
        U, R = s.get_state()
    assert_bitwise(U, [np.asarray(a, np.float32) for a in U0], "state after autotune")
    assert best[1] < 16, best
    assert ms > 0
