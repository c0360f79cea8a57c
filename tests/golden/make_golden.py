"""Generate the golden vectors that pin the oracle to the reference.

Run where the reference tree is present, after `make -C oracle ref`:

    python tests/golden/make_golden.py

It calls the reference's own code compiled from its sources (oracle/_ref):
  * source/GPU/GPUonly.cuh device math (WENO5 +/- with clipping, Einfeldt,
    Batten s*, HLLC rho/vel/pvel/e, extra-term velocity, stencil reads),
    and its WENO3 reconstruction (the -D_WENO3_ build),
  * source/GPU/GPUkernels.cu stage kernels (flux assembly, extra terms,
    divergence, update), run on the host in the WENO5 and WENO3 builds,
  * source/BoundaryConditions.h absorbing/reflecting ghost fills,
  * source/MaxSpeedOfSound.cpp (MaxSpeedOfSound_CPP::compute),
  * source/Sim/Sim_SICCloudMPI.cpp (the shock-induced cloud-collapse IC,
    Sim_SICCloudMPI::_ic run on a 24x20x16 block),
  * source/Types.h output streamers (the arrays of the dump and the save),
  * source/Sim/Sim_SteadyStateMPI.cpp, Sim_SodMPI.cpp, Sim_2DSBIMPI.cpp (the
    other cases' initial conditions, run on a 24x20x16 block),
on seeded inputs, and stores inputs and outputs as .npz fixtures next to
this script.  The reference has no golden vectors or known-answer tests of
its own; these fixtures are its outputs, recorded here.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as O  # noqa: E402

F = ctypes.c_float


def weno_inputs(rng, n):
    """Stencils of 6 values: smooth, jumps, flat, tiny, large, mixed signs."""
    out = []
    for k in range(n):
        kind = k % 6
        if kind == 0:
            base = rng.uniform(-10, 10)
            v = base + np.cumsum(rng.normal(0, 0.1, 6))
        elif kind == 1:
            lo, hi = rng.uniform(0.5, 2.0), rng.uniform(500, 1000)
            cut = rng.integers(1, 6)
            v = np.where(np.arange(6) < cut, lo, hi) * (1 + rng.normal(0, 1e-3, 6))
        elif kind == 2:
            v = np.full(6, rng.uniform(-100, 100))
        elif kind == 3:
            v = rng.normal(0, 1e-3, 6)
        elif kind == 4:
            v = rng.uniform(4000, 5000, 6)
        else:
            v = rng.normal(0, 1, 6) * 10 ** rng.uniform(-4, 3)
        out.append(v.astype(np.float32))
    return np.array(out, np.float32)


def states(rng, n):
    """Left/right face states: rho, u, v, w, p, G, P on both sides."""
    liquid = rng.random(n) < 0.5
    rm = np.where(liquid, rng.uniform(900, 1000, n), rng.uniform(0.5, 20, n))
    rp = np.where(rng.random(n) < 0.5, rm * (1 + rng.normal(0, 1e-3, n)), rng.uniform(0.5, 1000, n))
    vel = rng.normal(0, 1, (6, n)) * 10 ** rng.uniform(-4, 0.5, (6, n))
    pm = rng.uniform(0.02, 2000, n)
    pp = np.where(rng.random(n) < 0.3, pm, rng.uniform(0.02, 2000, n))
    Gm = rng.uniform(0.1789, 2.5, n)
    Gp = rng.uniform(0.1789, 2.5, n)
    Pm = rng.uniform(0, 4829, n)
    Pp = rng.uniform(0, 4829, n)
    return np.array([rm, rp, *vel, pm, pp, Gm, Gp, Pm, Pp], np.float32).T


def make_devmath(L, rng):
    W = weno_inputs(rng, 3000)
    wm = np.array([L.ref_weno_minus_clipped(*map(float, w[:5])) for w in W], np.float32)
    wp = np.array([L.ref_weno_pluss_clipped(*map(float, w[1:])) for w in W], np.float32)
    wmu = np.array([L.ref_weno_minus(*map(float, w[:5])) for w in W], np.float32)
    wpu = np.array([L.ref_weno_pluss(*map(float, w[1:])) for w in W], np.float32)

    S = states(rng, 3000)
    out2 = (F * 2)()
    sm = np.empty(len(S), np.float32)
    sp = np.empty(len(S), np.float32)
    ss = np.empty(len(S), np.float32)
    hr, hv, hpv, he, hx = (np.empty(len(S), np.float32) for _ in range(5))
    for i, st in enumerate(S):
        rm, rp, um, up, vm, vp, wm_, wp_, pm, pp, Gm, Gp, Pm, Pp = map(float, st)
        L.ref_char_vel_einfeldt(rm, rp, um, up, pm, pp, Gm, Gp, Pm, Pp, out2)
        sm[i], sp[i] = out2[0], out2[1]
        s_ = L.ref_char_vel_star(rm, rp, um, up, pm, pp, float(sm[i]), float(sp[i]))
        if i % 7 == 0:
            s_ = 0.0     # exercise the sign_star == 0 branch
        ss[i] = s_
        a = (float(sm[i]), float(sp[i]), float(ss[i]))
        hr[i] = L.ref_hllc_rho(rm, rp, um, up, *a)
        hv[i] = L.ref_hllc_vel(rm, rp, vm, vp, um, up, *a)
        hpv[i] = L.ref_hllc_pvel(rm, rp, um, up, pm, pp, *a)
        he[i] = L.ref_hllc_e(rm, rp, um, up, vm, vp, wm_, wp_, pm, pp, Gm, Gp, Pm, Pp, *a)
        hx[i] = L.ref_extraterm_hllc_vel(um, up, Gm, Gp, Pm, Pp, *a)
    np.savez_compressed(os.path.join(HERE, "ref_devmath.npz"), weno_in=W, weno_minus_clipped=wm,
                        weno_pluss_clipped=wp, weno_minus=wmu, weno_pluss=wpu, states=S, sm=sm, sp=sp,
                        ss=ss, hllc_rho=hr, hllc_vel=hv, hllc_pvel=hpv, hllc_e=he, extraterm=hx)


def make_devmath_w3(rng):
    """The reference's compile-time WENO3 build (-D_WENO3_) of the same
    reconstruction functions."""
    L = O.ref_lib("libref_devmath_w3_8x7x6")
    W = weno_inputs(rng, 3000)
    wm = np.array([L.ref_weno_minus_clipped(*map(float, w[:5])) for w in W], np.float32)
    wp = np.array([L.ref_weno_pluss_clipped(*map(float, w[1:])) for w in W], np.float32)
    np.savez_compressed(os.path.join(HERE, "ref_devmath_w3.npz"), weno_in=W, weno_minus_clipped=wm,
                        weno_pluss_clipped=wp)


STAGE_CASES = (   # (reconstruction order, boundary conditions, stages (a, b, dt/h))
    (5, (0, 0, 0, 0, 0, 0), ((0.0, 0.25, 0.05),)),
    (5, (0, 1, 1, 0, 0, 1), ((0.0, 0.25, 0.04), (-17.0 / 32, 8.0 / 9, 0.04), (-32.0 / 27, 0.75, 0.04))),
    (5, (1, 1, 1, 1, 1, 1), ((-17.0 / 32, 8.0 / 9, 0.06),)),
    (3, (1, 0, 0, 1, 1, 0), ((0.0, 0.25, 0.05), (-17.0 / 32, 8.0 / 9, 0.05), (-32.0 / 27, 0.75, 0.05))),
)


def make_stage():
    """The reference's own stage kernels (GPUkernels.cu:35-1179, run on the
    host by oracle/ref_kernels.cpp) on seeded states: the SHA-256 of the
    state and register after the stages, and the first cells of rho."""
    rec = {}
    for i, (order, bc, stages) in enumerate(STAGE_CASES):
        L = O.ref_kernels(order)
        dims = O.ref_kernels_dims(L)
        U, R = O.stage_input(dims, 40 + i)
        gxyz = None
        for a, b, dtinvh in stages:
            gxyz = O.fill_ghosts(dims, bc, U)
            O.ref_kernels_stage(L, U, R, gxyz, a, b, dtinvh)
        rec[f"order{i}"] = np.array(order)
        rec[f"bc{i}"] = np.array(bc)
        rec[f"stages{i}"] = np.array(stages, np.float64)
        rec[f"dims{i}"] = np.array(dims)
        rec[f"digest{i}"] = np.array(O.state_digest(U, R))
        rec[f"rho{i}"] = U[0][:64].copy()
    np.savez_compressed(os.path.join(HERE, "ref_stage.npz"), **rec)


def cloud(dims, seed):
    import mpcf
    params, bub = mpcf.configs.small_cloud(dims, nb=2, seed=seed)
    return [np.ascontiguousarray(a) for a in mpcf.ic_cloud_host(dims, params, bub, np.float32)]


def make_bc(rng):
    combos = [(0,) * 6, (1,) * 6, (0, 1, 1, 0, 1, 0), (1, 0, 0, 1, 0, 1)]
    rec = {}
    for name in ("libref_bc_8x7x6", "libref_bc_16x16x16"):
        L = O.ref_lib(name)
        d = (ctypes.c_int * 3)()
        L.ref_bc_dims(d)
        dims = (d[0], d[1], d[2])
        U = cloud(dims, 5)
        for ci, bc in enumerate(combos):
            nx, ny, nz = dims
            gx = np.zeros(2 * 7 * 3 * ny * nz, np.float32)
            gy = np.zeros(2 * 7 * nx * 3 * nz, np.float32)
            gz = np.zeros(2 * 7 * nx * ny * 3, np.float32)
            L.ref_fill_ghosts(O.bc_arr(bc), O.fptrs(U), gx.ctypes.data_as(ctypes.POINTER(F)),
                              gy.ctypes.data_as(ctypes.POINTER(F)), gz.ctypes.data_as(ctypes.POINTER(F)))
            key = f"{dims[0]}x{dims[1]}x{dims[2]}_{ci}"
            rec[key + "_dims"] = np.array(dims)
            rec[key + "_bc"] = np.array(bc)
            rec[key + "_U"] = np.array(U)
            rec[key + "_gx"], rec[key + "_gy"], rec[key + "_gz"] = gx, gy, gz
    np.savez_compressed(os.path.join(HERE, "ref_bc.npz"), **rec)


def make_sos():
    L = O.ref_lib("libref_sos")
    rec = {}
    for i, dims in enumerate([(24, 20, 16), (40, 33, 7)]):
        U = cloud(dims, 21 + i)
        rec[f"U{i}"] = np.array(U)
        rec[f"sos{i}"] = np.float32(L.ref_max_sos_cpp(U[0].size, O.fptrs(U)))
    np.savez_compressed(os.path.join(HERE, "ref_sos.npz"), **rec)


def sic_cases(rng):
    """Parameter sets and clouds of the SICCloud IC cases: shock along x with a
    sharp interface; an oblique shock with a cosine ramp; the reference's
    option defaults with spheres cut by the domain edges."""
    cases = []
    prm = list(O.SIC_DEFAULTS)
    prm[2], prm[10] = 100.0, 0.2                          # p0, shock point x
    sh = [(0.5, 0.4, 0.3, 0.12), (0.75, 0.3, 0.35, 0.07), (0.62, 0.62, 0.45, 0.09)]
    cases.append((prm, sh, 0.0))
    prm = list(O.SIC_DEFAULTS)
    prm[2], prm[6] = 10.0, 25.0                           # p0, pressure ratio
    prm[7], prm[8], prm[9] = 1.0, 0.35, 0.2               # oblique normal
    prm[10], prm[11], prm[12] = 0.15, 0.1, 0.3
    sh = [tuple(v) for v in np.column_stack([rng.uniform(0.35, 0.95, 12), rng.uniform(0.1, 0.75, 12),
                                             rng.uniform(0.1, 0.6, 12), rng.uniform(0.02, 0.08, 12)])]
    cases.append((prm, sh, 0.03))
    prm = list(O.SIC_DEFAULTS)
    sh = [(0.98, 0.05, 0.3, 0.1), (0.4, 0.8, 0.64, 0.15), (0.3, 0.3, 0.0, 0.2)]
    cases.append((prm, sh, 0.0))
    # shapes as float32 values (the reference reads cloud.dat into Real)
    return [(p, [tuple(float(np.float32(x)) for x in c) for c in sh], e) for p, sh, e in cases]


def make_sic(rng):
    import tempfile
    L = O.ref_lib("libref_sic_ic")
    rec = {}
    for i, (prm, sh, eps) in enumerate(sic_cases(rng)):
        with tempfile.TemporaryDirectory() as w:
            dims, out, post = O.ref_sic_cloud(L, prm, sh, eps, w)
        rec[f"dims{i}"] = np.array(dims)
        rec[f"prm{i}"] = np.array(prm, np.float64)
        rec[f"shapes{i}"] = np.array(sh, np.float64)
        rec[f"eps{i}"] = np.float64(eps)
        rec[f"U{i}"] = np.array(out)
        rec[f"post{i}"] = np.array(post, np.float64)
    np.savez_compressed(os.path.join(HERE, "ref_sic_ic.npz"), **rec)


def make_dump():
    """The reference's dump and save arrays (myTensorialStreamer,
    mySaveStreamer) of a 12x10x8 cloud state with a velocity field."""
    L = O.ref_lib("libref_dump_12x10x8")
    U = cloud((12, 10, 8), 41)
    rng = np.random.default_rng(41)
    for q in (1, 2, 3):                          # momenta of |u| up to ~5
        U[q] = (U[0] * rng.uniform(-5, 5, U[0].size)).astype(np.float32)
    rec = {"U": np.array(U), "tensor": O.ref_pack(L, "tensor", U), "save": O.ref_pack(L, "save", U)}
    np.savez_compressed(os.path.join(HERE, "ref_dump.npz"), **rec)


CASE_SETS = [
    ("steady", [], None, "xy"),
    ("steady", [("-rho", 2.0), ("-u", 0.5), ("-v", 0.25), ("-w", 0.125), ("-p", 3.0), ("-g", 6.59), ("-pc", 4096.0)], None, "xy"),
    ("steady", [("-rho", 1000.0), ("-u", 7.0), ("-p", 100.0), ("-g", 1.4), ("-pc", 0.5)], None, "xy"),
    ("sod", [], None, "x"),
    ("sod", [("-config", "y"), ("-reverse", 1), ("-x0", 0.3)], None, "y"),
    ("sod", [("-config", "z"), ("-rho1", 1000.0), ("-p1", 1000.0), ("-g1", 6.59), ("-pc1", 4096.0), ("-u2", 3.0),
             ("-rho2", 1.0), ("-p2", 1.0), ("-g2", 1.4), ("-pc2", 0.0)], None, "z"),
    ("sbi", [("-config", "xy")], [(0.5, 0.45, 0.3, 0.15), (0.8, 0.2, 0.3, 0.08), (0.3, 0.7, 0.3, 0.1)], "xy"),
    ("sbi", [("-config", "zx"), ("-reverse", 1), ("-mollfactor", 2), ("-x0", 0.2)],
     [(0.4, 0.3, 0.35, 0.12), (0.7, 0.5, 0.5, 0.09)], "zx"),
    ("sbi", [("-config", "yz"), ("-mach", 1.5), ("-rhobubble", 5.0), ("-pbubble", 1.0), ("-g2", 1.1)],
     [(0.4, 0.45, 0.3, 0.13), (0.2, 0.6, 0.5, 0.11)], "yz"),
]


def make_cases():
    """The reference's SteadyState, Sod and 2DSBI initial conditions
    (Sim_*MPI::_ic run by oracle/ref_cases_harness.cpp on a 24x20x16 block)."""
    import tempfile
    L = O.ref_lib("libref_cases")
    rec = {}
    for i, (case, opts, bub, config) in enumerate(CASE_SETS):
        if bub is not None:
            bub = [tuple(float(np.float32(v)) for v in b) for b in bub]
        with tempfile.TemporaryDirectory() as w:
            dims, out = O.ref_case(L, case, opts, w, bubbles=bub, config=config)
        rec[f"case{i}"] = np.array(case)
        rec[f"opts{i}"] = np.array([f"{k}={v}" for k, v in opts])
        rec[f"bubbles{i}"] = np.array(bub if bub is not None else np.zeros((0, 4)), np.float64)
        rec[f"config{i}"] = np.array(config)
        rec[f"dims{i}"] = np.array(dims)
        rec[f"U{i}"] = np.array(out)
    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **rec)


def main():
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "cubism-jr-gpu-mpcf_b200"))
    L = O.ref_lib("libref_devmath_8x7x6")
    if L is None:
        raise SystemExit("oracle/_ref not built (needs the reference tree): make -C oracle ref")
    rng = np.random.default_rng(20261203)
    make_devmath(L, rng)
    make_bc(rng)
    make_sos()
    make_sic(np.random.default_rng(20261204))
    make_dump()
    make_cases()
    make_devmath_w3(np.random.default_rng(20261205))
    make_stage()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
