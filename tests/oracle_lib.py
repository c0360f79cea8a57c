"""ctypes access to the CPU parity oracle (oracle/liboracle.so) and to the
reference pieces compiled from their own sources (oracle/_ref/*.so).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this module.
"""
import ctypes
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

_c = ctypes
_F = _c.c_float
_D = _c.c_double
_I = _c.c_int
_PF = _c.POINTER(_c.c_float)
_PD = _c.POINTER(_c.c_double)
_PPF = _c.POINTER(_PF)
_PPD = _c.POINTER(_PD)
_PI = _c.POINTER(_c.c_int)

_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise OSError("oracle not built: run `make -C oracle`")
        L = _c.CDLL(ORACLE_SO)
        L.oracle_stage_f32.argtypes = [_I, _I, _I, _PI, _PPF, _PPF, _F, _F, _F]
        L.oracle_stage_f64.argtypes = [_I, _I, _I, _PI, _PPD, _PPD, _D, _D, _D]
        L.oracle_max_sos_f32.restype = _F
        L.oracle_max_sos_f32.argtypes = [_c.c_longlong, _PPF]
        L.oracle_max_sos_f64.restype = _D
        L.oracle_max_sos_f64.argtypes = [_c.c_longlong, _PPD]
        L.oracle_max_sos_cpp_f32.restype = _F
        L.oracle_max_sos_cpp_f32.argtypes = [_c.c_longlong, _PPF]
        L.oracle_step_f32.restype = _D
        L.oracle_step_f32.argtypes = [_I, _I, _I, _PI, _PPF, _PPF, _D, _D, _D, _PD]
        L.oracle_step_f64.restype = _D
        L.oracle_step_f64.argtypes = [_I, _I, _I, _PI, _PPD, _PPD, _D, _D, _D, _PD]
        L.oracle_fill_ghosts_f32.argtypes = [_I, _I, _I, _PI, _PPF, _PF, _PF, _PF]
        L.oracle_face_flux_f32.argtypes = [_PF, _I, _PF]
        for n in ("oracle_weno_minus_clipped_f32", "oracle_weno_pluss_clipped_f32"):
            getattr(L, n).restype = _F
            getattr(L, n).argtypes = [_F] * 5
        L.oracle_char_vel_einfeldt_f32.argtypes = [_F] * 10 + [_PF]
        L.oracle_char_vel_star_f32.restype = _F
        L.oracle_char_vel_star_f32.argtypes = [_F] * 8
        L.oracle_hllc_rho_f32.restype = _F
        L.oracle_hllc_rho_f32.argtypes = [_F] * 7
        L.oracle_hllc_vel_f32.restype = _F
        L.oracle_hllc_vel_f32.argtypes = [_F] * 9
        L.oracle_hllc_pvel_f32.restype = _F
        L.oracle_hllc_pvel_f32.argtypes = [_F] * 9
        L.oracle_hllc_e_f32.restype = _F
        L.oracle_hllc_e_f32.argtypes = [_F] * 17
        L.oracle_extraterm_hllc_vel_f32.restype = _F
        L.oracle_extraterm_hllc_vel_f32.argtypes = [_F] * 9
        L.oracle_stencil_f32.argtypes = [_I, _I, _I, _PPF, _PF, _PF, _PF, _I, _I, _I, _I, _I, _PF]
        L.oracle_sic_cloud_f32.argtypes = [_I, _I, _I, _PD, _I, _PD, _D, _PPF, _PD]
        L.oracle_sic_cloud_f64.argtypes = [_I, _I, _I, _PD, _I, _PD, _D, _PPD, _PD]
        L.oracle_set_weno3.argtypes = [_I]
        L.oracle_bubbles.restype = _I
        L.oracle_bubbles.argtypes = [_c.c_ulonglong, _I, _D, _D, _PD, _PD, _D, _I, _PD]
        L.oracle_ic_cloud_f32.argtypes = [_I, _I, _I, _PI, _PI, _PD, _c.c_ulonglong, _I, _PD, _PPF]
        L.oracle_ic_cloud_f64.argtypes = [_I, _I, _I, _PI, _PI, _PD, _c.c_ulonglong, _I, _PD, _PPD]
        _oracle = L
    return _oracle


def contracted():
    """oracle/liboracle_contracted.so: the oracle's stage source built with
    fused multiply-add contraction, or None when it is not built or this CPU
    has no FMA instructions."""
    p = os.path.join(ORACLE_DIR, "liboracle_contracted.so")
    try:
        with open("/proc/cpuinfo") as f:
            has_fma = " fma " in f.read()
    except OSError:
        has_fma = False
    if not (has_fma and os.path.exists(p)):
        return None
    L = _c.CDLL(p)
    L.oracle_step_f32.restype = _D
    L.oracle_step_f32.argtypes = [_I, _I, _I, _PI, _PPF, _PPF, _D, _D, _D, _PD]
    return L


def ref_lib(name):
    """Load oracle/_ref/<name>.so or return None when it was not built."""
    p = os.path.join(REF_DIR, name + ".so")
    if not os.path.exists(p):
        return None
    L = _c.CDLL(p)
    if name == "libref_sos":
        L.ref_max_sos_cpp.restype = _F
        L.ref_max_sos_cpp.argtypes = [_c.c_longlong, _PPF]
    if name.startswith("libref_bc"):
        L.ref_fill_ghosts.argtypes = [_PI, _PPF, _PF, _PF, _PF]
        L.ref_bc_dims.argtypes = [_PI]
    if name.startswith("libref_dump"):
        L.ref_dump_dims.argtypes = [_PI]
        L.ref_pack.argtypes = [_I, _PPF, _PF]
        L.ref_unpack_save.argtypes = [_PF, _PPF]
    if name == "libref_cases":
        L.ref_cases_dims.argtypes = [_PI]
        L.ref_case_ic.argtypes = [_I, _c.c_char_p, _I, _c.POINTER(_c.c_char_p), _PPF]
    if name == "libref_sic_ic":
        L.ref_sic_dims.argtypes = [_PI]
        L.ref_sic_ic.argtypes = [_c.c_char_p, _I, _c.POINTER(_c.c_char_p), _D, _PPF, _PD]
    if name.startswith("libref_devmath"):   # the WENO5 and the WENO3 build
        L.ref_devmath_dims.argtypes = [_PI]
        for n in ("ref_weno_pluss", "ref_weno_minus", "ref_weno_pluss_clipped", "ref_weno_minus_clipped"):
            getattr(L, n).restype = _F
            getattr(L, n).argtypes = [_F] * 5
        L.ref_char_vel_einfeldt.argtypes = [_F] * 10 + [_PF]
        L.ref_char_vel_star.restype = _F
        L.ref_char_vel_star.argtypes = [_F] * 8
        L.ref_hllc_rho.restype = _F
        L.ref_hllc_rho.argtypes = [_F] * 7
        L.ref_hllc_vel.restype = _F
        L.ref_hllc_vel.argtypes = [_F] * 9
        L.ref_hllc_pvel.restype = _F
        L.ref_hllc_pvel.argtypes = [_F] * 9
        L.ref_hllc_e.restype = _F
        L.ref_hllc_e.argtypes = [_F] * 17
        L.ref_extraterm_hllc_vel.restype = _F
        L.ref_extraterm_hllc_vel.argtypes = [_F] * 9
        L.ref_read_stencil.argtypes = [_I, _PF, _I, _PF, _PF, _c.c_uint, _c.c_uint, _c.c_uint, _PF]
    return L


def fptrs(arrs):
    t = _PD if arrs[0].dtype == np.float64 else _PF
    return (t * len(arrs))(*[a.ctypes.data_as(t) for a in arrs])


def bc_arr(bc):
    return (_c.c_int * 6)(*bc)


def stage(dims, bc, U, R, a, b, dtinvh):
    """In-place oracle stage on lists of 7 contiguous arrays."""
    nx, ny, nz = dims
    L = oracle()
    if U[0].dtype == np.float64:
        rc = L.oracle_stage_f64(nx, ny, nz, bc_arr(bc), fptrs(U), fptrs(R), a, b, dtinvh)
    else:
        rc = L.oracle_stage_f32(nx, ny, nz, bc_arr(bc), fptrs(U), fptrs(R),
                                float(np.float32(a)), float(np.float32(b)), float(np.float32(dtinvh)))
    assert rc == 0


def step(dims, bc, U, R, cfl=0.3, dt_max=1e30):
    """In-place oracle LSRK3 step; returns (dt, sos)."""
    nx, ny, nz = dims
    h = 1.0 / max(dims)
    sos = _c.c_double()
    L = oracle()
    f = L.oracle_step_f64 if U[0].dtype == np.float64 else L.oracle_step_f32
    dt = f(nx, ny, nz, bc_arr(bc), fptrs(U), fptrs(R), cfl, dt_max, h, _c.byref(sos))
    assert dt >= 0
    return dt, sos.value


def max_sos(U):
    L = oracle()
    if U[0].dtype == np.float64:
        return L.oracle_max_sos_f64(U[0].size, fptrs(U))
    return L.oracle_max_sos_f32(U[0].size, fptrs(U))


def fill_ghosts(dims, bc, U):
    nx, ny, nz = dims
    gx = np.empty(2 * 7 * 3 * ny * nz, np.float32)
    gy = np.empty(2 * 7 * nx * 3 * nz, np.float32)
    gz = np.empty(2 * 7 * nx * ny * 3, np.float32)
    oracle().oracle_fill_ghosts_f32(nx, ny, nz, bc_arr(bc), fptrs(U),
                                    gx.ctypes.data_as(_PF), gy.ctypes.data_as(_PF), gz.ctypes.data_as(_PF))
    return gx, gy, gz


# --- shock-induced cloud-collapse IC ------------------------------------------
# Parameter vector order of oracle_sic_cloud_* (and of mpcf_sic_params):
SIC_KEYS = ("rho0", "u0", "p0", "rhoB", "uB", "pB", "pressure_ratio",
            "nx", "ny", "nz", "Sx", "Sy", "Sz", "g1", "g2", "pc1", "pc2")
# the reference's command-line option of each (Sim_SICCloudMPI.cpp:52-76)
SIC_OPTS = ("-rho0", "-u0", "-p0", "-rhoB", "-uB", "-pB", "-pressureratio",
            "-shockNx", "-shockNy", "-shockNz", "-shockSx", "-shockSy", "-shockSz",
            "-g1", "-g2", "-pc1", "-pc2")
SIC_DEFAULTS = (1000.0, 0.0, 1.0, 1.0, 0.0, 0.0234, 40.0, 1.0, 0.0, 0.0, 0.05, 0.0, 0.0, 6.59, 1.4, 4096.0, 1.0)


def sic_cloud(dims, prm, shapes, eps, dtype=np.float32):
    """Oracle restatement of the SICCloud IC: (7 fields, (rho1, u1, p1, mach))."""
    nx, ny, nz = dims
    out = [np.zeros(nx * ny * nz, dtype) for _ in range(7)]
    p = np.ascontiguousarray(prm, np.float64)
    sh = np.ascontiguousarray(shapes, np.float64).reshape(-1)
    post = (_D * 4)()
    f = oracle().oracle_sic_cloud_f64 if dtype == np.float64 else oracle().oracle_sic_cloud_f32
    f(nx, ny, nz, p.ctypes.data_as(_PD), sh.size // 4, sh.ctypes.data_as(_PD) if sh.size else None,
      float(eps), fptrs(out), post)
    return out, tuple(post)


def ref_sic_cloud(L, prm, shapes, eps, workdir):
    """The reference's own Sim_SICCloudMPI::_ic() (oracle/_ref/libref_sic_ic.so)
    on its compile-time block: writes cloud_config.dat and cloud.dat into
    workdir (shapes as 9-significant-digit text, exact for float32 values)."""
    if any(float(v) < 0 for v in prm):
        # ArgumentParser.h:104-121 takes every token that starts with '-' as
        # an option name, so "-shockNz -0.2" would set shockNz = 1: the
        # reference's command line cannot carry negative values
        raise ValueError("negative option values cannot reach the reference's parser")
    d = (_c.c_int * 3)()
    L.ref_sic_dims(d)
    n = d[0] * d[1] * d[2]
    with open(os.path.join(workdir, "cloud_config.dat"), "w") as f:
        f.write(f"{len(shapes)} 0\n0.01 0.5\n0 0 0\n1 1 1\n")
    with open(os.path.join(workdir, "cloud.dat"), "w") as f:
        for i, c in enumerate(shapes):
            f.write(f"{i} {c[0]:.9g} {c[1]:.9g} {c[2]:.9g} {c[3]:.9g}\n")
    args = [b"sic"]
    for opt, v in zip(SIC_OPTS, prm):
        args += [opt.encode(), repr(float(v)).encode()]
    argv = (_c.c_char_p * len(args))(*args)
    out = [np.zeros(n, np.float32) for _ in range(7)]
    post = (_D * 4)()
    rc = L.ref_sic_ic(workdir.encode(), len(args), argv, float(eps), fptrs(out), post)
    if rc != 0:
        raise RuntimeError(f"ref_sic_ic failed: {rc}")
    return (d[0], d[1], d[2]), out, tuple(post)


# --- dump / save arrays -------------------------------------------------------
def pack(U, dims, kind):
    """The interleaved (nz, ny, nx, channels) array the reference's streamers
    fill (Types.h:192-277): kind "tensor" = rho, u, v, w, p, G, P, 0, 0 with
    p = (E - 0.5*(ru^2+rv^2+rw^2)/rho - P)/G (the 0.5 literal makes that part
    double; the squares are summed in the state's type); kind "save" = the
    7 conserved fields."""
    nx, ny, nz = dims
    r, mu, mv, mw, e, G, P = [np.asarray(a).reshape(nz, ny, nx) for a in U]
    if kind == "save":
        return np.stack([r, mu, mv, mw, e, G, P], axis=-1)
    T = r.dtype.type
    sq = (mu * mu + mv * mv) + mw * mw
    f = np.float64
    p = ((e.astype(f) - 0.5 * sq.astype(f) / r.astype(f)) - P.astype(f)) / G.astype(f)
    z = np.zeros_like(r)
    return np.stack([r, mu / r, mv / r, mw / r, p.astype(T), G, P, z, z], axis=-1)


def ref_pack(L, kind, U):
    """The reference's own streamers (oracle/_ref/libref_dump_*.so)."""
    d = (_c.c_int * 3)()
    L.ref_dump_dims(d)
    nch = 9 if kind == "tensor" else 7
    out = np.zeros(d[0] * d[1] * d[2] * nch, np.float32)
    L.ref_pack(0 if kind == "tensor" else 1, fptrs([np.ascontiguousarray(a, np.float32) for a in U]), out.ctypes.data_as(_PF))
    return out.reshape(d[2], d[1], d[0], nch)


# --- SteadyState / Sod / 2DSBI cases ----------------------------------------------
CASES = {"steady": 0, "sod": 1, "sbi": 2}


def ref_case(L, case, opts, workdir, bubbles=None, config="xy"):
    """The reference's own case set-up (oracle/_ref/libref_cases.so) on its
    compile-time block: opts is a list of (option, value) pairs; for "sbi"
    the bubbles are written to <config>bubbles.dat in workdir."""
    d = (_c.c_int * 3)()
    L.ref_cases_dims(d)
    n = d[0] * d[1] * d[2]
    if bubbles is not None:
        with open(os.path.join(workdir, f"{config}bubbles.dat"), "w") as f:
            f.write(f"{len(bubbles)}\n")
            for b in bubbles:
                f.write(f"{b[0]:.9g} {b[1]:.9g} {b[2]:.9g} {b[3]:.9g}\n")
    args = [b"case", b"-dryrun", b"1", b"-verb", b"0"]
    for k, v in opts:
        if isinstance(v, (int, float)) and float(v) < 0:
            raise ValueError("negative option values cannot reach the reference's parser")
        args += [k.encode(), str(v).encode()]
    argv = (_c.c_char_p * len(args))(*args)
    out = [np.zeros(n, np.float32) for _ in range(7)]
    rc = L.ref_case_ic(CASES[case], workdir.encode(), len(args), argv, fptrs(out))
    if rc != 0:
        raise RuntimeError(f"ref_case_ic failed: {rc}")
    return (d[0], d[1], d[2]), out


_libm = None


def _m():
    global _libm
    if _libm is None:
        _libm = _c.CDLL("libm.so.6")
        _libm.powf.restype = _F
        _libm.powf.argtypes = [_F, _F]
        _libm.cosf.restype = _F
        _libm.cosf.argtypes = [_F]
    return _libm


def _cell_positions(dims):
    nx, ny, nz = dims
    h = 1.0 / max(dims)
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return h, [h * (ix.ravel() + 0.5), h * (iy.ravel() + 0.5), h * (iz.ravel() + 0.5)], [ix.ravel(), iy.ravel(), iz.ravel()]


def case_ic(case, dims, prm, bubbles=None, dtype=np.float32):
    """Restatement of the reference's case initial conditions:
      "steady": Sim_SteadyStateMPI::_ic (Sim_SteadyStateMPI.cpp:103-134)
      "sod":    Sim_SodMPI::_ic (Sim_SodMPI.cpp:27-91)
      "sbi":    Sim_2DSBIMPI::_ic (Sim_2DSBIMPI.cpp:83-229; Real = dtype)
    prm: dict of the mpcf_*_params fields.  Returns 7 flat fields."""
    n = dims[0] * dims[1] * dims[2]
    f = np.float64
    if case == "steady":
        r, u, v, w, p, g, pc = (prm[k] for k in ("rho", "u", "v", "w", "p", "g", "pc"))
        G = 1.0 / (g - 1.0)
        P = g * pc * G
        e = G * p + P + 0.5 * r * (u * u + v * v + w * w)
        return [np.full(n, val, dtype) for val in (r, r * u, r * v, r * w, e, G, P)]
    h, pos, idx = _cell_positions(dims)
    if case == "sod":
        a = prm["axis"]
        x = pos[a] > prm["x0"] if prm["reverse"] else pos[a] < prm["x0"]
        xf, nf = x.astype(f), (~x).astype(f)
        g1, g2 = prm["g1"], prm["g2"]
        r = xf * prm["rho1"] + nf * prm["rho2"]
        p = xf * prm["p1"] + nf * prm["p2"]
        u = xf * prm["rho1"] * prm["u1"] + nf * prm["rho2"] * prm["u2"]
        G = xf * 1. / (g1 - 1.) + nf * 1. / (g2 - 1.)
        P = xf * prm["pc1"] * g1 / (g1 - 1.) + nf * prm["pc2"] * g2 / (g2 - 1.)
        mom = [u if a == d else np.zeros(n) for d in range(3)]
        return [a_.astype(dtype) for a_ in (r, mom[0], mom[1], mom[2], G * p + P + 0.5 * u * u / r, G, P)]
    # 2DSBI, Real = dtype
    T = np.dtype(dtype).type
    L = _m()
    pre = [T(prm["rho"]), T(prm["u"]), T(prm["p"])]
    mach, gamma, pc = T(prm["mach"]), T(prm["g1"]), T(prm["pc1"])
    m2 = T(L.powf(mach, T(2.))) if T is np.float32 else T(mach ** 2.0)
    mpost = np.sqrt((f(m2) * (f(gamma) - 1.) + 2.) / (2. * f(gamma) * f(m2) - (f(gamma) - 1.)))
    post0 = T((f(gamma) + 1.) * f(m2) / ((f(gamma) - 1.) * f(m2) + 2.) * f(pre[0]))
    post2 = T(1. / (f(gamma) + 1.) * (2. * f(gamma) * f(m2) - (f(gamma) - 1.)) * f(pre[2]))
    u_pre = f(mach * np.sqrt(gamma * (pc + pre[2]) / pre[0]))
    u_post = mpost * f(np.sqrt(gamma * (pc + post2) / post0))
    post1 = T(u_pre - u_post)
    rho1, u1, p1 = f(post0), f(post1), f(post2)
    G1, G2 = prm["g1"] - 1, prm["g2"] - 1
    F1, F2 = prm["g1"] * prm["pc1"], prm["g2"] * prm["pc2"]
    eps = f(T(prm["mollfactor"])) * np.sqrt(3.) * h
    a0, a1 = prm["axis0"], prm["axis1"]
    n3 = list(dims)
    src = [i.copy() for i in idx]
    flip = np.zeros(n, bool)
    if prm["reverse"]:
        mid = (idx[a0] == n3[a0] // 2) if n3[a0] % 2 else np.zeros(n, bool)
        flip = ~mid
        for d in range(3):
            src[d] = np.where(flip, n3[d] - 1 - idx[d], idx[d])
    P_ = [h * (src[d] + 0.5) for d in range(3)]
    shock = np.where((P_[a0] - prm["x0"]).astype(T) > 0, T(0), T(1)).astype(T)
    bubble = np.zeros(n, T)
    done = np.zeros(n, bool)
    cosf = np.vectorize(lambda x: L.cosf(x) if T is np.float32 else np.cos(x))
    for b in (bubbles if bubbles is not None else []):
        dx = P_[a0] - f(T(b[a0]))
        dy = P_[a1] - f(T(b[a1]))
        r = np.sqrt(dx * dx + dy * dy).astype(T)
        phi = (r - T(b[3])).astype(T)
        x = 0.5 * (phi.astype(f) + eps) / eps
        mx = np.where(0. < x, x, 0.)
        mn = np.where(mx < 1., mx, 1.)
        alpha = (np.pi * mn).astype(T)
        c = np.array(cosf(alpha), dtype=T) if alpha.size else alpha
        bi = (0.5 + 0.5 * c.astype(f)).astype(T)
        take = ~done
        bubble = np.where(take, bi, bubble).astype(T)
        done = done | (take & (bi > 0))
    s, bb = shock.astype(f), bubble.astype(f)
    one_s, one_b = (T(1) - shock).astype(f), (T(1) - bubble).astype(f)
    rho = (s * rho1 + one_s * (prm["rhobubble"] * bb + prm["rho"] * one_b)).astype(T)
    mom = ((s * u1 + one_s * prm["u"]) * rho.astype(f)).astype(T)
    G = (1. / G1 * one_b + 1. / G2 * bb).astype(T)
    P = (F1 / G1 * one_b + F2 / G2 * bb).astype(T)
    pressure = (s * p1 + one_s * (prm["pbubble"] * bb + prm["p"] * one_b)).astype(T)
    m = mom.astype(f)
    ke = (0.5 * (m * m + 0. + 0.) / rho.astype(f)).astype(T)
    E = (pressure * G + P + ke).astype(T)
    mom = np.where(flip, -mom, mom).astype(T)
    zero = np.zeros(n, T)
    moms = [mom if a0 == d else zero for d in range(3)]
    return [rho, moms[0], moms[1], moms[2], E, G, P]


def case_prm(case, opts, config=None):
    """mpcf_*_params fields (reference defaults) from a list of the
    reference's (option, value) pairs."""
    defaults = {
        "steady": dict(rho=1.0, u=0.0, v=0.0, w=0.0, p=1.0, g=1.4, pc=0.0),
        "sod": dict(x0=0.5, rho1=1.0, rho2=0.125, u1=0.0, u2=0.0, p1=1.0, p2=0.1, g1=1.4, g2=1.4, pc1=0.0,
                    pc2=0.0, reverse=0, axis=0),
        "sbi": dict(x0=0.1, mach=1.22, rho=1.0, rhobubble=0.138, u=0.0, p=1.0, pbubble=1.0, g1=1.4, g2=1.67,
                    pc1=0.0, pc2=0.0, reverse=0, mollfactor=1, axis0=0, axis1=1),
    }
    prm = dict(defaults[case])
    axes = {"xy": (0, 1), "xz": (0, 2), "yx": (1, 0), "yz": (1, 2), "zx": (2, 0), "zy": (2, 1)}
    for k, v in opts:
        k = k.lstrip("-")
        if k == "config":
            if case == "sod":
                prm["axis"] = "xyz".index(v)
            else:
                prm["axis0"], prm["axis1"] = axes[v]
        else:
            prm[k] = type(prm[k])(v)
    return prm


def bubbles(seed, n, rmin, rmax, lo=(0.2, 0.2, 0.2), hi=(0.8, 0.8, 0.8), gap=0.0, max_tries=200000):
    """Seeded non-overlapping spheres (x, y, z, r), shape (placed, 4): the
    oracle's restatement of the workloads' bubble placement."""
    out = np.zeros((max(n, 1), 4), np.float64)
    lo3 = (_D * 3)(*lo)
    hi3 = (_D * 3)(*hi)
    k = oracle().oracle_bubbles(_c.c_ulonglong(seed), int(n), float(rmin), float(rmax), lo3, hi3,
                                float(gap), int(max_tries), out.ctypes.data_as(_PD))
    return out[:k]


def cloud_prm(params):
    """The cloud parameters (an object with the mpcf_ic_params fields) as
    the oracle's array, and the noise seed."""
    names = ("rho_l", "p_l", "gamma_l", "pc_l", "rho_g", "p_g", "gamma_g", "pc_g", "noise", "width")
    return np.array([float(getattr(params, n)) for n in names], np.float64), int(params.seed)


def ic_cloud(dims, params, bub, dtype=np.float32, origin=None, glob=None):
    """Bubble-cloud state of an nx*ny*nz block (7 flat arrays); the block's
    cell (0,0,0) is global cell `origin` of a `glob`-sized domain (default:
    the block is the domain)."""
    nx, ny, nz = dims
    out = [np.empty(nx * ny * nz, dtype) for _ in range(7)]
    prm, seed = cloud_prm(params)
    b = np.ascontiguousarray(bub, dtype=np.float64).ravel()
    o3 = (_I * 3)(*origin) if origin is not None else None
    g3 = (_I * 3)(*glob) if glob is not None else None
    f = oracle().oracle_ic_cloud_f64 if dtype == np.float64 else oracle().oracle_ic_cloud_f32
    f(nx, ny, nz, o3, g3, prm.ctypes.data_as(_PD), _c.c_ulonglong(seed), b.size // 4,
      b.ctypes.data_as(_PD) if b.size else None, fptrs(out))
    return out


class weno3:
    """Context manager: the oracle's reconstruction is the reference's
    compile-time WENO3 build while inside (GPUonly.cuh:102,141)."""

    def __enter__(self):
        oracle().oracle_set_weno3(1)
        return self

    def __exit__(self, *exc):
        oracle().oracle_set_weno3(0)
        return False


def ref_kernels(order=5):
    """oracle/_ref/libref_kernels[_w3]_20x16x12.so: the reference's own stage
    kernels run on the host (WENO5 or the -D_WENO3_ build), or None."""
    L = ref_lib("libref_kernels_20x16x12" if order == 5 else "libref_kernels_w3_20x16x12")
    if L is not None:
        L.ref_kernels_dims.argtypes = [_PI]
        L.ref_kernels_stage.argtypes = [_PPF, _PPF, _PF, _PF, _PF, _F, _F, _F]
    return L


def ref_kernels_dims(L):
    d = (_I * 3)()
    L.ref_kernels_dims(d)
    return d[0], d[1], d[2]


def ref_kernels_stage(L, U, R, ghosts, a, b, dtinvh):
    """One stage of the reference's kernels, in place on U and R (FP32)."""
    gx, gy, gz = ghosts
    L.ref_kernels_stage(fptrs(U), fptrs(R), gx.ctypes.data_as(_PF), gy.ctypes.data_as(_PF), gz.ctypes.data_as(_PF),
                        float(np.float32(a)), float(np.float32(b)), float(np.float32(dtinvh)))


def stage_input(dims, seed):
    """The state (the oracle's cloud set-up with its seeded placement: two
    bubbles) and a seeded register of a stage case of the reference-kernel
    checks."""
    from mpcf import configs
    params = configs.ic_params(100.0, seed)
    ext = configs.extents(dims)
    edge = min(ext)
    bub = bubbles(seed, 2, 0.08 * edge, 0.2 * edge, tuple(0.2 * e for e in ext), tuple(0.8 * e for e in ext))
    U = ic_cloud(dims, params, bub, np.float32)
    rng = np.random.default_rng(seed)
    R = [rng.normal(0, 1e-2, U[0].size).astype(np.float32) for _ in range(7)]
    return U, R


def state_digest(U, R):
    """SHA-256 of the FP32 bytes of the 7 state and 7 register fields."""
    import hashlib
    h = hashlib.sha256()
    for a in list(U) + list(R):
        h.update(np.ascontiguousarray(a, np.float32).tobytes())
    return h.hexdigest()
