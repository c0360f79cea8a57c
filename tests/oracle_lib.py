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
        _oracle = L
    return _oracle


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
    if name.startswith("libref_devmath"):
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
