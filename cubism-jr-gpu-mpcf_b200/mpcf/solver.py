"""Python host layer over the C ABI.

``Solver`` owns one or more independent domains on one GPU.  ``GPUlab``
mirrors the reference's lab interface (source/GPUlab.h:250-258) so a
Python driver reads like the reference's LSRK3_IntegratorMPI
(source/LSRK3_IntegratorMPI.cpp:27-62):

    lab.max_sos() -> (seconds, sos); lab.load_ghosts(); lab.process_all(a, b, dtinvh)
"""
import ctypes
import time

import numpy as np

from . import _lib
from ._lib import check, lib

FIELDS = ("rho", "rhou", "rhov", "rhow", "E", "G", "P")


def _ptr_array(arrays):
    return (ctypes.c_void_p * 7)(*[a.ctypes.data for a in arrays])


def dtype_of(precision):
    return np.float64 if precision in (_lib.PREC_FP64, _lib.PREC_FP64_FAST) else np.float32


class Solver:
    """Domains advanced by the fused sm_100a stage kernel.

    dims: list of (nx, ny, nz); bc: list of 6-tuples (x-, x+, y-, y+, z-, z+)
    or None (absorbing); precision: one of _lib.PREC_* or a name in
    _lib.PRECISIONS.
    """

    def __init__(self, dims, bc=None, precision="fp32_ref", device=0):
        if isinstance(precision, str):
            precision = _lib.PRECISIONS[precision]
        if isinstance(dims[0], int):
            dims = [tuple(dims)]
        self.dims = [tuple(int(v) for v in d) for d in dims]
        self.ndom = len(self.dims)
        self.precision = precision
        self.dtype = dtype_of(precision)
        flat = (ctypes.c_int * (3 * self.ndom))(*[v for d in self.dims for v in d])
        bcarr = None
        if bc is not None:
            if isinstance(bc[0], int):
                bc = [bc] * self.ndom
            bcarr = (ctypes.c_int * (6 * self.ndom))(*[int(v) for b in bc for v in b])
        h = ctypes.c_void_p()
        check(lib().mpcf_create(ctypes.byref(h), self.ndom, flat, bcarr, precision, device))
        self._h = h
        self.device = int(device)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().mpcf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state ------------------------------------------------------------
    def ncells(self, dom=0):
        nx, ny, nz = self.dims[dom]
        return nx * ny * nz

    def set_state(self, state, reg=None, dom=0):
        """state/reg: sequences of 7 host arrays (flattened x-fastest)."""
        st = [np.ascontiguousarray(a, dtype=self.dtype).ravel() for a in state]
        rg = None if reg is None else [np.ascontiguousarray(a, dtype=self.dtype).ravel() for a in reg]
        for a in st + (rg or []):
            if a.size != self.ncells(dom):
                raise ValueError("field size does not match the domain")
        check(lib().mpcf_set_state(self._h, dom, _ptr_array(st), None if rg is None else _ptr_array(rg), 0))

    def get_state(self, dom=0, with_reg=True):
        n = self.ncells(dom)
        st = [np.empty(n, self.dtype) for _ in range(7)]
        rg = [np.empty(n, self.dtype) for _ in range(7)] if with_reg else None
        check(lib().mpcf_get_state(self._h, dom, _ptr_array(st), None if rg is None else _ptr_array(rg), 0))
        return (st, rg) if with_reg else st

    def device_pointers(self, dom=0):
        st = (ctypes.c_void_p * 7)()
        rg = (ctypes.c_void_p * 7)()
        check(lib().mpcf_device_pointers(self._h, dom, st, rg))
        return list(st), list(rg)

    # -- hot path ---------------------------------------------------------
    def max_sos(self):
        out = (ctypes.c_double * self.ndom)()
        check(lib().mpcf_max_sos(self._h, out))
        return list(out)

    def stage(self, a, b, dtinvh=None):
        arr = None
        if dtinvh is not None:
            if np.isscalar(dtinvh):
                dtinvh = [dtinvh] * self.ndom
            arr = (ctypes.c_double * self.ndom)(*dtinvh)
        check(lib().mpcf_stage(self._h, float(a), float(b), arr))

    def update(self, b):
        """U <- U + b*R alone (the reference's _update)."""
        check(lib().mpcf_update(self._h, float(b)))

    def compute_dt(self, cfl, dt_max=1e30):
        out = (ctypes.c_double * self.ndom)()
        check(lib().mpcf_compute_dt(self._h, float(cfl), float(dt_max), out))
        return list(out)

    def step(self, cfl=0.3, dt_max=1e30, want_dt=True):
        out = (ctypes.c_double * self.ndom)() if want_dt else None
        check(lib().mpcf_step(self._h, float(cfl), float(dt_max), out))
        return list(out) if want_dt else None

    def run(self, nsteps, cfl=0.3, dt_max=1e30, graph=True):
        out = (ctypes.c_double * self.ndom)()
        check(lib().mpcf_run(self._h, int(nsteps), float(cfl), float(dt_max), 1 if graph else 0, out))
        return list(out)

    def run_host(self, host_state, nsteps, cfl=0.3, dt_max=1e30, nchunks=8):
        """nsteps steps of a state held in host memory (mpcf_run_host):
        `host_state` (7 contiguous arrays of the solver's dtype, pinned
        memory for overlap) is every step's input and is overwritten with
        every step's result.  Returns the time."""
        for a in host_state:
            if a.dtype != self.dtype or not a.flags["C_CONTIGUOUS"] or a.size != self.ncells(0):
                raise ValueError("host fields must be contiguous arrays of the solver's dtype and size")
        t = ctypes.c_double()
        check(lib().mpcf_run_host(self._h, int(nsteps), float(cfl), float(dt_max), _ptr_array(host_state),
                                  int(nchunks), ctypes.byref(t)))
        return t.value

    # -- stream-ordered building blocks (nothing synchronises) -------------
    def stream_handle(self):
        """The solver's cudaStream_t as an integer (mpcf_stream)."""
        p = ctypes.c_void_p()
        check(lib().mpcf_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def sos_accumulator(self):
        """Device address of the per-domain sound-speed accumulator."""
        p = ctypes.c_void_p()
        check(lib().mpcf_sos_accumulator(self._h, ctypes.byref(p)))
        return p.value

    def enqueue_sos(self):
        check(lib().mpcf_enqueue_sos(self._h))

    def enqueue_dt(self, cfl=0.3, dt_max=1e30):
        check(lib().mpcf_enqueue_dt(self._h, float(cfl), float(dt_max)))

    def enqueue_stage(self, a, b):
        check(lib().mpcf_enqueue_stage(self._h, float(a), float(b)))

    def synchronize(self):
        check(lib().mpcf_synchronize(self._h))

    def conserved_sums(self):
        out = (ctypes.c_double * (5 * self.ndom))()
        check(lib().mpcf_conserved_sums(self._h, out))
        return np.array(out).reshape(self.ndom, 5)

    def track_conservation(self, on=True):
        check(lib().mpcf_set_track_conservation(self._h, 1 if on else 0))

    def error_word(self, clear=False):
        w = ctypes.c_uint()
        check(lib().mpcf_error_word(self._h, ctypes.byref(w), 1 if clear else 0))
        return w.value

    # -- boundaries -------------------------------------------------------
    def set_bc(self, bc6, dom=0):
        check(lib().mpcf_set_bc(self._h, dom, (ctypes.c_int * 6)(*bc6)))

    # -- z-slab decomposition ----------------------------------------------
    def link_z(self, lower, upper):
        """Domain `upper` sits on top of domain `lower` (mpcf_link_z): every
        stage refreshes their facing ghost planes on the device, and the
        linked slabs share one dt."""
        check(lib().mpcf_link_z(self._h, lower, upper))

    def set_spacing(self, h, dom=0):
        check(lib().mpcf_set_spacing(self._h, dom, float(h)))

    def exchange_halos(self):
        check(lib().mpcf_exchange_halos(self._h))

    def set_origin(self, org, global_dims, dom=0):
        """The domain is the block at cell `org` of a global grid of
        `global_dims` cells (mpcf_set_origin): initial conditions are then
        generated in the global domain's coordinates."""
        check(lib().mpcf_set_origin(self._h, dom, (ctypes.c_int * 3)(*[int(v) for v in org]),
                                    (ctypes.c_int * 3)(*[int(v) for v in global_dims])))

    def fill_ghosts(self, dom=0):
        nx, ny, nz = self.dims[dom]
        gx = np.empty(2 * 7 * 3 * ny * nz, self.dtype)
        gy = np.empty(2 * 7 * nx * 3 * nz, self.dtype)
        gz = np.empty(2 * 7 * nx * ny * 3, self.dtype)
        check(lib().mpcf_fill_ghosts(self._h, dom, gx.ctypes.data, gy.ctypes.data, gz.ctypes.data, 0))
        return gx, gy, gz

    # -- initial conditions -----------------------------------------------
    def ic_cloud(self, params, bubbles, dom=0):
        b = np.ascontiguousarray(bubbles, dtype=np.float64).ravel()
        nb = b.size // 4
        check(lib().mpcf_ic_cloud(self._h, dom, ctypes.byref(params), nb,
                                  b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if nb else None))

    def ic_sic_cloud(self, params, shapes, dom=0):
        """The reference's shock-induced cloud-collapse IC (Sim_SICCloudMPI::_ic,
        Sim_SICCloudMPI.cpp:43-357) on domain `dom`: params is a SicParams
        (see sic_params), shapes an (n, 4) array of (x, y, z, radius)."""
        b = np.ascontiguousarray(shapes, dtype=np.float64).reshape(-1)
        n = b.size // 4
        check(lib().mpcf_ic_sic_cloud(self._h, dom, ctypes.byref(params), n,
                                      b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if n else None))

    def ic_steady(self, dom=0, **kw):
        """Sim_SteadyStateMPI's uniform state (options as keywords, see case_params)."""
        check(lib().mpcf_ic_steady(self._h, dom, ctypes.byref(case_params("steady", **kw))))

    def ic_sod(self, dom=0, **kw):
        """Sim_SodMPI's shock tube along axis (0 x, 1 y, 2 z)."""
        check(lib().mpcf_ic_sod(self._h, dom, ctypes.byref(case_params("sod", **kw))))

    def ic_sbi(self, bubbles, dom=0, **kw):
        """Sim_2DSBIMPI's shock-bubble interaction; bubbles (n, 4) = x, y, z, r."""
        b = np.ascontiguousarray(bubbles, dtype=np.float64).reshape(-1)
        n = b.size // 4
        check(lib().mpcf_ic_sbi(self._h, dom, ctypes.byref(case_params("sbi", **kw)), n,
                                b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if n else None))

    # -- output and restart (Sim_SteadyStateMPI.cpp:138-180) ---------------
    def pack(self, kind="tensor", dom=0):
        """The reference's dump ("tensor": rho, u, v, w, p, G, P, 0, 0) or save
        ("save": the conserved fields) array of a domain, shape (nz, ny, nx, ch)."""
        k = _lib.DUMP_TENSOR if kind == "tensor" else _lib.DUMP_SAVE
        nx, ny, nz = self.dims[dom]
        out = np.empty((nz, ny, nx, 9 if k == _lib.DUMP_TENSOR else 7), dtype=self.dtype)
        check(lib().mpcf_pack(self._h, dom, k, out.ctypes.data))
        return out

    def unpack_save(self, arr, dom=0):
        a = np.ascontiguousarray(arr, dtype=self.dtype)
        nx, ny, nz = self.dims[dom]
        if a.size != nx * ny * nz * 7:
            raise ValueError("save array has the wrong size")
        check(lib().mpcf_unpack_save(self._h, dom, a.ctypes.data))

    def dump(self, directory, name, step=0, kind="tensor", dom=0):
        k = _lib.DUMP_TENSOR if kind == "tensor" else _lib.DUMP_SAVE
        check(lib().mpcf_dump(self._h, dom, k, str(directory).encode(), name.encode(), int(step)))

    def save(self, directory, t, step, fcount=0, dom=0):
        check(lib().mpcf_save(self._h, dom, str(directory).encode(), float(t), int(step), int(fcount)))

    def restart(self, directory, dom=0):
        """(t, step, fcount) after loading <directory>/save.*, or None when
        there is no save record (the reference's _restart returning false)."""
        t, st, fc = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        rc = lib().mpcf_restart(self._h, dom, str(directory).encode(), ctypes.byref(t), ctypes.byref(st), ctypes.byref(fc))
        if rc == 0:
            return None
        check(rc if rc < 0 else 0)
        return t.value, st.value, fc.value

    def set_time(self, t, dom=0):
        check(lib().mpcf_set_time(self._h, dom, float(t)))

    def get_time(self, dom=0):
        t = ctypes.c_double()
        check(lib().mpcf_get_time(self._h, dom, ctypes.byref(t)))
        return t.value

    # -- launch configuration ----------------------------------------------
    def set_weno_order(self, order):
        """5 (WENO5) or 3 (the reference's compile-time WENO3 build; the
        reference-rounding forms only)."""
        check(lib().mpcf_set_weno_order(self._h, int(order)))

    def weno_order(self):
        return check(lib().mpcf_get_weno_order(self._h))

    def set_tiling(self, ty, dz, persistent=False, tma=True):
        flags = (_lib.TILE_PERSISTENT if persistent else 0) | (_lib.TILE_TMA if tma else 0)
        check(lib().mpcf_set_tiling(self._h, int(ty), int(dz), flags))

    def set_test_flags(self, flags):
        """Failure-detection tests only (mpcf_set_test_flags)."""
        check(lib().mpcf_set_test_flags(self._h, int(flags)))

    def test_copy_count(self, clear=False):
        """Failure-detection tests only: bulk copies issued while a test
        flag was set (mpcf_test_copy_count)."""
        c = ctypes.c_uint()
        check(lib().mpcf_test_copy_count(self._h, ctypes.byref(c), 1 if clear else 0))
        return c.value

    def tiling(self):
        """(ty, dz, persistent, tma) of the current launch configuration."""
        ty, dz, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().mpcf_get_tiling(self._h, ctypes.byref(ty), ctypes.byref(dz), ctypes.byref(f)))
        return ty.value, dz.value, bool(f.value & _lib.TILE_PERSISTENT), bool(f.value & _lib.TILE_TMA)

    def autotune(self, reps=3):
        best = (ctypes.c_int * 3)()
        ms = ctypes.c_double()
        check(lib().mpcf_autotune(self._h, int(reps), best, ctypes.byref(ms)))
        return (best[0], best[1], bool(best[2] & _lib.TILE_PERSISTENT), bool(best[2] & _lib.TILE_TMA)), ms.value

    def launch_shape(self):
        nt, g, th = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
        check(lib().mpcf_launch_shape(self._h, ctypes.byref(nt), ctypes.byref(g), ctypes.byref(th)))
        return nt.value, g.value, th.value

    def time_stages(self, reps, dtinvh=0.0):
        ms = ctypes.c_double()
        check(lib().mpcf_time_stages(self._h, int(reps), float(dtinvh), ctypes.byref(ms)))
        return ms.value


CONFIG_AXES = {"xy": (0, 1), "xz": (0, 2), "yx": (1, 0), "yz": (1, 2), "zx": (2, 0), "zy": (2, 1)}


def case_params(case, **kw):
    """Option structure of case "steady", "sod" or "sbi" with the reference's
    defaults, overridden by keyword (names of the reference's options; for
    "sod" `config` = "x"|"y"|"z", for "sbi" `config` = "xy", "xz", ...)."""
    st, so, sb = _lib.SteadyParams(), _lib.SodParams(), _lib.SbiParams()
    lib().mpcf_case_default_params(ctypes.byref(st), ctypes.byref(so), ctypes.byref(sb))
    p = {"steady": st, "sod": so, "sbi": sb}[case]
    for k, v in kw.items():
        if k == "config" and case == "sod":
            p.axis = "xyz".index(v)
        elif k == "config" and case == "sbi":
            p.axis0, p.axis1 = CONFIG_AXES[v]
        elif any(k == f[0] for f in p._fields_):
            setattr(p, k, int(v) if k in ("reverse", "axis", "axis0", "axis1", "mollfactor") else float(v))
        else:
            raise KeyError(k)
    return p


def case_bc(case, config="xy"):
    """Boundary conditions of the reference's lab of a case (the GPUlab*
    _apply_bc overrides): SteadyState reflecting everywhere, Sod and the
    cloud collapse absorbing, 2DSBI reflecting on the faces normal to the
    second axis of its config."""
    R, A = _lib.BC_REFLECTING, _lib.BC_ABSORBING
    if case == "steady":
        return (R,) * 6
    if case in ("sod", "sic"):
        return (A,) * 6
    a1 = CONFIG_AXES[config][1]
    return tuple(R if d // 2 == a1 else A for d in range(6))


def sic_params(**kw):
    """SicParams with the reference's option defaults (Sim_SICCloudMPI.cpp:52-76),
    overridden by keyword: rho0, u0, p0, rhoB, uB, pB, pressure_ratio,
    shock_n (3), shock_s (3), g1, g2, pc1, pc2, eps."""
    p = _lib.SicParams()
    lib().mpcf_sic_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if k in ("shock_n", "shock_s"):
            for i in range(3):
                getattr(p, k)[i] = float(v[i])
        elif hasattr(p, k):
            setattr(p, k, float(v))
        else:
            raise KeyError(k)
    return p


def sic_post_shock(params, precision="fp32_ref"):
    """(rho1, u1, p1, mach) behind the shock, as the given precision computes them."""
    out = (ctypes.c_double * 4)()
    check(lib().mpcf_sic_post_shock(ctypes.byref(params), _lib.PRECISIONS[precision], out))
    return tuple(out)


def ic_cloud_host(dims, params, bubbles, dtype=np.float32):
    """Host generator of the bubble-cloud IC (same formula as the device one)."""
    nx, ny, nz = dims
    n = nx * ny * nz
    out = [np.empty(n, dtype) for _ in range(7)]
    b = np.ascontiguousarray(bubbles, dtype=np.float64).ravel()
    nb = b.size // 4
    check(lib().mpcf_ic_cloud_host(nx, ny, nz, ctypes.byref(params), nb,
                                   b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if nb else None,
                                   np.dtype(dtype).itemsize, _ptr_array(out)))
    return out


def bubbles(seed, n, rmin, rmax, lo=(0.2, 0.2, 0.2), hi=(0.8, 0.8, 0.8), gap=0.0, max_tries=200000):
    """Seeded non-overlapping spheres (x, y, z, r), shape (placed, 4)."""
    out = np.zeros((max(n, 1), 4), np.float64)
    lo3 = (ctypes.c_double * 3)(*lo)
    hi3 = (ctypes.c_double * 3)(*hi)
    k = check(lib().mpcf_bubbles(ctypes.c_ulonglong(seed), int(n), float(rmin), float(rmax), lo3, hi3,
                                 float(gap), int(max_tries), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out[:k]


# LSRK3 coefficients (LSRK3_IntegratorMPI.cpp:46,51,56)
LSRK3 = ((0.0, 1.0 / 4), (-17.0 / 32, 8.0 / 9), (-32.0 / 27, 3.0 / 4))


class WindowSolver(Solver):
    """A domain of nx*ny*nz cells held in host memory, possibly larger than
    the device's, advanced by streaming z-chunks of `nslices` planes through
    `nslots` device slots (mpcf_create_window / mpcf_run_window; the
    reference's GPUlab with nslices < sizeZ, GPUlab.cpp:37-41,202-372).
    nslices >= 3 divides nz; nslots >= min(5, nz / nslices).  Only `run`
    advances it."""

    def __init__(self, dims, nslices, nslots=8, bc=None, precision="fp32_ref", device=0):
        if isinstance(precision, str):
            precision = _lib.PRECISIONS[precision]
        nx, ny, nz = (int(v) for v in dims)
        bcarr = None if bc is None else (ctypes.c_int * 6)(*[int(v) for v in bc])
        h = ctypes.c_void_p()
        check(lib().mpcf_create_window(ctypes.byref(h), nx, ny, nz, int(nslices), int(nslots), precision, bcarr, device))
        self._h = h
        self.device = int(device)
        self.precision = precision
        self.dtype = dtype_of(precision)
        info = (ctypes.c_int * 4)()
        check(lib().mpcf_window_info(self._h, info))
        self.global_dims = (nx, ny, nz)
        self.nslices, self.nchunks, self.nslots = info[1], info[2], info[3]
        self.dims = [(nx, ny, self.nslices)] * self.nslots
        self.ndom = self.nslots

    def run(self, host_state, nsteps, cfl=0.3, dt_max=1e30):
        """nsteps steps of `host_state` (7 contiguous arrays of nx*ny*nz of
        the solver's dtype, page-locked for overlap), overwritten with each
        step's result.  Returns the time."""
        n = self.global_dims[0] * self.global_dims[1] * self.global_dims[2]
        for a in host_state:
            if a.dtype != self.dtype or not a.flags["C_CONTIGUOUS"] or a.size != n:
                raise ValueError("host fields must be contiguous arrays of the solver's dtype and the domain's size")
        t = ctypes.c_double()
        check(lib().mpcf_run_window(self._h, int(nsteps), float(cfl), float(dt_max), _ptr_array(host_state),
                                    ctypes.byref(t)))
        return t.value


    def stage_host(self, host_state, host_reg, a, b, dtinvh):
        """One stage of a block whose state and register both live in host
        memory (mpcf_window_stage), both overwritten."""
        n = self.global_dims[0] * self.global_dims[1] * self.global_dims[2]
        for arr in list(host_state) + list(host_reg):
            if arr.dtype != self.dtype or not arr.flags["C_CONTIGUOUS"] or arr.size != n:
                raise ValueError("host fields must be contiguous arrays of the solver's dtype and the domain's size")
        check(lib().mpcf_window_stage(self._h, float(a), float(b), float(dtinvh), _ptr_array(host_state),
                                      _ptr_array(host_reg)))

    def max_sos_host(self, host_state):
        """The largest sound speed of a host-resident state (mpcf_window_max_sos)."""
        out = ctypes.c_double()
        check(lib().mpcf_window_max_sos(self._h, _ptr_array(host_state), ctypes.byref(out)))
        return out.value

    def set_bc(self, bc6, dom=0):
        """The block's six faces (absorbing or reflecting)."""
        check(lib().mpcf_set_bc(self._h, 0, (ctypes.c_int * 6)(*[int(v) for v in bc6])))


def window_stage_plan(nchunks, nslots):
    """The operations of one host-resident stage (mpcf_window_stage_plan),
    rows (kind, step, stage, chunk): kind 0 upload, 3 stage, 4 download."""
    n = check(lib().mpcf_window_stage_plan(int(nchunks), int(nslots), None, 0))
    buf = (ctypes.c_int * (4 * max(n, 1)))()
    check(lib().mpcf_window_stage_plan(int(nchunks), int(nslots), buf, n))
    return np.frombuffer(buf, dtype=np.int32)[:4 * n].reshape(n, 4).copy()


def window_plan(nchunks, nslots, nsteps):
    """The operations of a windowed run in enqueue order (mpcf_window_plan,
    no device work): an int array of rows (kind, step, stage, chunk), kind 0
    upload, 1 sound speed of the first step's input, 2 dt, 3 stage, 4
    download; step -1 is the sound-speed pass."""
    n = check(lib().mpcf_window_plan(int(nchunks), int(nslots), int(nsteps), None, 0))
    buf = (ctypes.c_int * (4 * max(n, 1)))()
    check(lib().mpcf_window_plan(int(nchunks), int(nslots), int(nsteps), buf, n))
    return np.frombuffer(buf, dtype=np.int32)[:4 * n].reshape(n, 4).copy()


class GPUlab:
    """Reference-shaped lab over a single-domain Solver (GPUlab.h:250-258).

    ``nslices`` is accepted for signature compatibility; the state is device
    resident, so there is no chunking.  ``process_all`` keeps the reference
    postcondition when ``sync_host`` is set: the host arrays hold the new
    state and register after each call (GPUlab.cpp:772-788).
    """

    def __init__(self, solver, nslices=None, host_state=None, host_reg=None, sync_host=False):
        self.solver = solver
        self.nslices = nslices
        self.host_state = host_state
        self.host_reg = host_reg
        self.sync_host = sync_host

    def load_ghosts(self, t=0.0):
        # ghosts are synthesised inside the stage kernel from the boundary
        # conditions; nothing to stage
        return None

    def max_sos(self):
        t0 = time.perf_counter()
        sos = self.solver.max_sos()[0]
        return time.perf_counter() - t0, sos

    def process_all(self, a, b, dtinvh):
        t0 = time.perf_counter()
        self.solver.stage(a, b, dtinvh)
        if self.sync_host and self.host_state is not None:
            st, rg = self.solver.get_state()
            for q in range(7):
                self.host_state[q][...] = st[q].reshape(self.host_state[q].shape)
                if self.host_reg is not None:
                    self.host_reg[q][...] = rg[q].reshape(self.host_reg[q].shape)
        return time.perf_counter() - t0


def lsrk3_step(lab, h, cfl, dt_max=1e30, real=np.float32):
    """LSRK3_IntegratorMPI::operator() on one rank, driving a GPUlab."""
    _, sos = lab.max_sos()
    dt = cfl * h / sos
    dt = dt_max if dt_max < dt else dt
    for a, b in LSRK3:
        lab.load_ghosts()
        # process_all takes Real arguments: the coefficients and dt/h are
        # rounded to the stage precision
        lab.process_all(float(real(a)), float(real(b)), float(real(dt / h)))
    return dt
