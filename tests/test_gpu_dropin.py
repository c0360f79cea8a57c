"""Drop-in: the reference's own LSRK3_IntegratorMPI (source/LSRK3_IntegratorMPI.cpp,
compiled unchanged) drives the B200 path through the C++ shim (GPUlab,
GridMPI, BoundaryConditions), on one rank.  The result must equal the CPU
oracle bit for bit (FP32 reference rounding).

The driver library (oracle/_ref/libref_lsrk3_driver.so) is built where the
reference tree is present (`make -C oracle ref`) and travels with the
repository; these tests need it and a GPU.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle_lib as O
from conftest import cloud_state

pytestmark = pytest.mark.gpu

DRV = os.path.join(O.REF_DIR, "libref_lsrk3_driver.so")


@pytest.fixture(scope="module")
def drv(mpcf):
    if not os.path.exists(DRV):
        pytest.fail("oracle/_ref/libref_lsrk3_driver.so missing: build it with `make -C oracle ref` "
                    "where the reference tree is present")
    L = ctypes.CDLL(DRV)
    L.drv_dims.argtypes = [ctypes.POINTER(ctypes.c_int)]
    L.drv_run.restype = ctypes.c_double
    L.drv_run.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                          ctypes.POINTER(ctypes.POINTER(ctypes.c_float)),
                          ctypes.POINTER(ctypes.POINTER(ctypes.c_float)), ctypes.c_int]
    d = (ctypes.c_int * 3)()
    L.drv_dims(d)
    L.dims = (d[0], d[1], d[2])
    return L


def bitwise(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("host_sync", [1, 0])
def test_reference_integrator_cuda_sos(drv, host_sync):
    dims = drv.dims
    bc = (0,) * 6
    U = cloud_state(dims, nb=2, seed=31)
    R = [np.zeros_like(a) for a in U]
    Ud = [a.copy() for a in U]
    Rd = [a.copy() for a in R]
    dt = drv.drv_run(2, 0.3, 0, O.bc_arr(bc), O.fptrs(Ud), O.fptrs(Rd), host_sync)
    for _ in range(2):
        dt_o, _ = O.step(dims, bc, U, R, cfl=0.3)
    assert dt == dt_o
    assert bitwise(Ud, U) and bitwise(Rd, R)


def test_reference_integrator_cpu_sos_reflecting(drv):
    """-SOSkernel cpp: the reference's MaxSpeedOfSound_CPP on the host state
    (the lab keeps the host copy current), reflecting walls."""
    dims = drv.dims
    bc = (1,) * 6
    U = cloud_state(dims, nb=2, seed=32)
    R = [np.zeros_like(a) for a in U]
    Ud = [a.copy() for a in U]
    Rd = [a.copy() for a in R]
    dt = drv.drv_run(1, 0.3, 1, O.bc_arr(bc), O.fptrs(Ud), O.fptrs(Rd), 1)
    # oracle with the CPU sound-speed formula (MaxSpeedOfSound.cpp:18-55)
    h = 1.0 / max(dims)
    sos = O.oracle().oracle_max_sos_cpp_f32(U[0].size, O.fptrs(U))
    dt_o = 0.3 * h / sos
    for a, b in ((0.0, 0.25), (-17.0 / 32, 8.0 / 9), (-32.0 / 27, 0.75)):
        O.stage(dims, bc, U, R, a, b, dt_o / h)
    assert dt == dt_o
    assert bitwise(Ud, U) and bitwise(Rd, R)


@pytest.mark.parametrize("nslices,sos_cpp,bc", [(4, 0, (0,) * 6), (8, 1, (1, 0, 0, 1, 1, 0))])
def test_reference_integrator_windowed_lab(drv, monkeypatch, nslices, sos_cpp, bc):
    """The lab streamed in chunks of nslices planes (MPCF_GPULAB_WINDOW=1: the
    path a block larger than device memory takes): the reference's
    process_all and max_sos over its host state and register chunk by chunk,
    through device slots.  Two steps equal the oracle bit for bit."""
    monkeypatch.setenv("MPCF_GPULAB_WINDOW", "1")
    monkeypatch.setenv("MPCF_GPULAB_SLOTS", "5")
    drv.drv_run_sliced.restype = ctypes.c_double
    drv.drv_run_sliced.argtypes = drv.drv_run.argtypes + [ctypes.c_int]
    dims = drv.dims
    U = cloud_state(dims, nb=2, seed=33)
    R = [np.zeros_like(a) for a in U]
    Ud = [a.copy() for a in U]
    Rd = [a.copy() for a in R]
    dt = drv.drv_run_sliced(2, 0.3, sos_cpp, O.bc_arr(bc), O.fptrs(Ud), O.fptrs(Rd), 1, nslices)
    h = 1.0 / max(dims)
    for _ in range(2):
        if sos_cpp:
            sos = O.oracle().oracle_max_sos_cpp_f32(U[0].size, O.fptrs(U))
            dt_o = 0.3 * h / sos
            for a, b in ((0.0, 0.25), (-17.0 / 32, 8.0 / 9), (-32.0 / 27, 0.75)):
                O.stage(dims, bc, U, R, a, b, dt_o / h)
        else:
            dt_o, _ = O.step(dims, bc, U, R, cfl=0.3)
    assert dt == dt_o
    assert bitwise(Ud, U) and bitwise(Rd, R)
