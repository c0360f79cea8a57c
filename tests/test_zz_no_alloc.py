"""The allocation-free conservation sums (mpcf_conserved_sums_noalloc).

Some callers may not allocate device memory: a host that gives a plug-in a
fixed device-memory budget at start-up and forbids cudaMalloc afterwards, or
a tight loop that cannot afford cudaMalloc/cudaFree, which may synchronise
the whole device.  For them the library offers the FP64 sums of a state
they own, with its scratch in a fixed device array of the library.  This
file runs last (pytest collects it last by name), so a failure here comes
after every other test has run; it also passes alone in a fresh process,
where its first call performs the one-time set-up on the device.
"""
import ctypes

import numpy as np
import pytest

from conftest import cloud_state

pytestmark = pytest.mark.gpu

LIMIT = 8192 * 32768


def noalloc_sums(mpcf, ptrs, ncells, esz, device=0, stream=None):
    """Host output on `device`, work on `stream` (a cudaStream_t or None)."""
    L = mpcf.lib()
    out = (ctypes.c_double * 5)()
    arr = (ctypes.c_void_p * 7)(*ptrs)
    rc = L.mpcf_conserved_sums_noalloc(arr, ncells, esz, out, 0, device, stream)
    return rc, np.array(out)


@pytest.mark.parametrize("precision", ["fp32_ref", "fp64"])
def test_noalloc_sums_match_existing_entry_on_two_calls(mpcf, precision):
    dims = (64, 48, 40)                      # 122880 cells: 4 chunks, the last one partial
    n = dims[0] * dims[1] * dims[2]
    dtype = mpcf.dtype_of(mpcf.PRECISIONS[precision])
    esz = np.dtype(dtype).itemsize
    with mpcf.Solver([dims], precision=precision) as s:
        for seed in (3, 4):                  # two calls in a row, on two different states
            s.set_state(cloud_state(dims, nb=2, seed=seed, dtype=dtype))
            want = s.conserved_sums()[0]
            st, _ = s.device_pointers()
            rc, got = noalloc_sums(mpcf, st, n, esz, device=s.device)
            assert rc == 0, mpcf.lib().mpcf_last_error()
            # same chunking and reduction order as mpcf_conserved_sums
            assert np.allclose(got, want, rtol=1e-12, atol=0), (got, want)
            assert np.array_equal(got, want)


def test_noalloc_sums_reject_oversize_and_bad_arguments(mpcf):
    L = mpcf.lib()
    dims = (16, 8, 8)
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(cloud_state(dims, nb=1))
        st, _ = s.device_pointers()
        rc, _ = noalloc_sums(mpcf, st, LIMIT + 1, 4, device=s.device)
        assert rc == mpcf._lib.ERR_ARG
        assert b"exceeds the no-allocation limit" in L.mpcf_last_error()
        rc, _ = noalloc_sums(mpcf, st, 16 * 8 * 8, 3, device=s.device)
        assert rc == mpcf._lib.ERR_ARG
        # still usable after the rejections
        rc, got = noalloc_sums(mpcf, st, 16 * 8 * 8, 4, device=s.device)
        assert rc == 0 and np.array_equal(got, s.conserved_sums()[0])


def test_noalloc_sums_into_device_memory_on_a_caller_stream(mpcf):
    """out_is_device = 1 writes the five sums into the caller's device
    buffer, with the work on the caller's (non-default) stream; bit-identical
    to mpcf_conserved_sums, on two calls in a row."""
    import torch
    dims = (48, 40, 36)
    n = dims[0] * dims[1] * dims[2]
    with mpcf.Solver([dims], precision="mixed") as s:
        torch.cuda.set_device(s.device)
        out = torch.zeros(5, dtype=torch.float64, device=f"cuda:{s.device}")
        stream = torch.cuda.Stream(device=s.device)
        for seed in (5, 6):
            s.set_state(cloud_state(dims, nb=3, seed=seed))
            want = s.conserved_sums()[0]
            st, _ = s.device_pointers()
            arr = (ctypes.c_void_p * 7)(*st)
            rc = mpcf.lib().mpcf_conserved_sums_noalloc(arr, n, 4, ctypes.cast(out.data_ptr(), ctypes.POINTER(ctypes.c_double)), 1,
                                                        s.device,
                                                        ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0, mpcf.lib().mpcf_last_error()
            stream.synchronize()
            assert np.array_equal(out.cpu().numpy(), want), (out.cpu().numpy(), want)
