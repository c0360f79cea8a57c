"""ctypes binding of libmpcf_b200 (include/mpcf_b200.h).

The shared library is built in-tree (``make -C cubism-jr-gpu-mpcf_b200``) and
loaded from ``cubism-jr-gpu-mpcf_b200/lib/libmpcf_b200.so``.  There is no
fallback: if the library is missing, loading raises, and every compute call
goes through the CUDA kernels.
"""
import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("MPCF_B200_LIB", os.path.join(PKG_DIR, "lib", "libmpcf_b200.so"))

PREC_FP32_REF = 0
PREC_FP32 = 1
PREC_MIXED = 2
PREC_FP64 = 3
PREC_FP64_FAST = 4
PRECISIONS = {"fp32_ref": PREC_FP32_REF, "fp32": PREC_FP32, "mixed": PREC_MIXED, "fp64": PREC_FP64,
              "fp64_fast": PREC_FP64_FAST}

BC_ABSORBING = 0
BC_REFLECTING = 1
BC_HALO = 2          # z faces of slabs: ghost planes filled from the neighbouring slab

ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_NUMERIC = -1, -2, -3, -4, -5
DUMP_TENSOR = 0
DUMP_SAVE = 1
ERRBIT_NONPHYSICAL = 1
ERRBIT_SOS = 2
ERRBIT_TMA_TIMEOUT = 4
ERRBIT_TMA_INFLIGHT = 16
TEST_DROP_LAST_COPY = 1
TEST_DROP_MID_COPY = 2
TILE_PERSISTENT = 1
TILE_TMA = 2

# every symbol the header declares, with (restype, argtypes)
_c = ctypes
_P = _c.c_void_p
_PP = _c.POINTER(_c.c_void_p)
_I = _c.c_int
_D = _c.c_double
_PD = _c.POINTER(_c.c_double)
_PI = _c.POINTER(_c.c_int)


class IcParams(ctypes.Structure):
    """mirror of mpcf_ic_params"""
    _fields_ = [("rho_l", _D), ("p_l", _D), ("gamma_l", _D), ("pc_l", _D),
                ("rho_g", _D), ("p_g", _D), ("gamma_g", _D), ("pc_g", _D),
                ("noise", _D), ("width", _D), ("seed", _c.c_ulonglong)]


class SicParams(ctypes.Structure):
    """mirror of mpcf_sic_params (the reference's SICCloud case options)"""
    _fields_ = [("rho0", _D), ("u0", _D), ("p0", _D), ("rhoB", _D), ("uB", _D), ("pB", _D),
                ("pressure_ratio", _D), ("shock_n", _D * 3), ("shock_s", _D * 3),
                ("g1", _D), ("g2", _D), ("pc1", _D), ("pc2", _D), ("eps", _D)]



class SteadyParams(ctypes.Structure):
    """mirror of mpcf_steady_params (Sim_SteadyStateMPI options)"""
    _fields_ = [(k, _D) for k in ("rho", "u", "v", "w", "p", "g", "pc")]


class SodParams(ctypes.Structure):
    """mirror of mpcf_sod_params (Sim_SodMPI options)"""
    _fields_ = [(k, _D) for k in ("x0", "rho1", "rho2", "u1", "u2", "p1", "p2", "g1", "g2", "pc1", "pc2")] + \
               [("reverse", _I), ("axis", _I)]


class SbiParams(ctypes.Structure):
    """mirror of mpcf_sbi_params (Sim_2DSBIMPI options)"""
    _fields_ = [(k, _D) for k in ("x0", "mach", "rho", "rhobubble", "u", "p", "pbubble", "g1", "g2", "pc1", "pc2")] + \
               [("reverse", _I), ("mollfactor", _I), ("axis0", _I), ("axis1", _I)]


SIGNATURES = {
    "mpcf_version": (_I, []),
    "mpcf_last_error": (_c.c_char_p, []),
    "mpcf_elem_size": (_I, [_I]),
    "mpcf_create": (_I, [_PP, _I, _PI, _PI, _I, _I]),
    "mpcf_destroy": (_I, [_P]),
    "mpcf_num_domains": (_I, [_P]),
    "mpcf_precision": (_I, [_P]),
    "mpcf_set_state": (_I, [_P, _I, _PP, _PP, _I]),
    "mpcf_get_state": (_I, [_P, _I, _PP, _PP, _I]),
    "mpcf_device_pointers": (_I, [_P, _I, _PP, _PP]),
    "mpcf_max_sos": (_I, [_P, _PD]),
    "mpcf_stage": (_I, [_P, _D, _D, _PD]),
    "mpcf_compute_dt": (_I, [_P, _D, _D, _PD]),
    "mpcf_step": (_I, [_P, _D, _D, _PD]),
    "mpcf_run": (_I, [_P, _I, _D, _D, _I, _PD]),
    "mpcf_run_host": (_I, [_P, _I, _D, _D, _PP, _I, _PD]),
    "mpcf_create_window": (_I, [_PP, _I, _I, _I, _I, _I, _I, _PI, _I]),
    "mpcf_run_window": (_I, [_P, _I, _D, _D, _PP, _PD]),
    "mpcf_window_info": (_I, [_P, _PI]),
    "mpcf_window_plan": (_I, [_I, _I, _I, _PI, _I]),
    "mpcf_window_stage_plan": (_I, [_I, _I, _PI, _I]),
    "mpcf_window_stage": (_I, [_P, _D, _D, _D, _PP, _PP]),
    "mpcf_window_max_sos": (_I, [_P, _PP, _PD]),
    "mpcf_synchronize": (_I, [_P]),
    "mpcf_stream": (_I, [_P, _PP]),
    "mpcf_sos_accumulator": (_I, [_P, _PP]),
    "mpcf_enqueue_sos": (_I, [_P]),
    "mpcf_enqueue_dt": (_I, [_P, _D, _D]),
    "mpcf_enqueue_stage": (_I, [_P, _D, _D]),
    "mpcf_update": (_I, [_P, _D]),
    "mpcf_conserved_sums": (_I, [_P, _PD]),
    "mpcf_conserved_sums_noalloc": (_I, [_PP, _c.c_longlong, _I, _PD, _I, _I, _P]),
    "mpcf_set_track_conservation": (_I, [_P, _I]),
    "mpcf_error_word": (_I, [_P, _c.POINTER(_c.c_uint), _I]),
    "mpcf_set_bc": (_I, [_P, _I, _PI]),
    "mpcf_fill_ghosts": (_I, [_P, _I, _P, _P, _P, _I]),
    "mpcf_link_z": (_I, [_P, _I, _I]),
    "mpcf_set_spacing": (_I, [_P, _I, _D]),
    "mpcf_exchange_halos": (_I, [_P]),
    "mpcf_set_origin": (_I, [_P, _I, _PI, _PI]),
    "mpcf_ic_cloud": (_I, [_P, _I, _c.POINTER(IcParams), _I, _PD]),
    "mpcf_ic_cloud_host": (_I, [_I, _I, _I, _c.POINTER(IcParams), _I, _PD, _I, _PP]),
    "mpcf_bubbles": (_I, [_c.c_ulonglong, _I, _D, _D, _PD, _PD, _D, _I, _PD]),
    "mpcf_sic_default_params": (None, [_c.POINTER(SicParams)]),
    "mpcf_sic_post_shock": (_I, [_c.POINTER(SicParams), _I, _PD]),
    "mpcf_ic_sic_cloud": (_I, [_P, _I, _c.POINTER(SicParams), _I, _PD]),
    "mpcf_case_default_params": (None, [_c.POINTER(SteadyParams), _c.POINTER(SodParams), _c.POINTER(SbiParams)]),
    "mpcf_ic_steady": (_I, [_P, _I, _c.POINTER(SteadyParams)]),
    "mpcf_ic_sod": (_I, [_P, _I, _c.POINTER(SodParams)]),
    "mpcf_ic_sbi": (_I, [_P, _I, _c.POINTER(SbiParams), _I, _PD]),
    "mpcf_pack": (_I, [_P, _I, _I, _P]),
    "mpcf_unpack_save": (_I, [_P, _I, _P]),
    "mpcf_dump": (_I, [_P, _I, _I, _c.c_char_p, _c.c_char_p, _I]),
    "mpcf_save": (_I, [_P, _I, _c.c_char_p, _D, _I, _I]),
    "mpcf_restart": (_I, [_P, _I, _c.c_char_p, _PD, _PI, _PI]),
    "mpcf_set_time": (_I, [_P, _I, _D]),
    "mpcf_get_time": (_I, [_P, _I, _PD]),
    "mpcf_set_tiling": (_I, [_P, _I, _I, _I]),
    "mpcf_set_weno_order": (_I, [_P, _I]),
    "mpcf_get_weno_order": (_I, [_P]),
    "mpcf_set_test_flags": (_I, [_P, _c.c_uint]),
    "mpcf_test_copy_count": (_I, [_P, _c.POINTER(_c.c_uint), _I]),
    "mpcf_get_tiling": (_I, [_P, _PI, _PI, _PI]),
    "mpcf_autotune": (_I, [_P, _I, _PI, _PD]),
    "mpcf_launch_shape": (_I, [_P, _c.POINTER(_c.c_longlong), _c.POINTER(_c.c_longlong), _PI]),
    "mpcf_time_stages": (_I, [_P, _I, _D, _PD]),
    "mpcf_probe_fp32_peak": (_I, [_I, _PD]),
    "mpcf_time_run": (_I, [_P, _I, _D, _D, _PD]),
    "mpcf_device_info": (_I, [_I, _c.c_char_p, _I, _c.POINTER(_c.c_longlong), _c.POINTER(_c.c_longlong), _PI]),
    "mpcf_device_synchronize": (_I, [_I]),
}

_lib = None


class MpcfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mpcf error {code}: {msg}")
        self.code = code


def lib():
    """Load (once) and return the shared library with typed entry points."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libmpcf_b200 not built: {LIB_PATH} is missing "
                          "(run `make -C cubism-jr-gpu-mpcf_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    """Raise MpcfError for a negative status; return non-negative values."""
    if rc < 0:
        raise MpcfError(rc, lib().mpcf_last_error().decode(errors="replace"))
    return rc
