"""Failure detection on the GPU without a fault: a bounded wait that runs out.

With MPCF_TEST_DROP_LAST_COPY a non-persistent stage launch arms the
mbarrier of each z-chunk's last bulk copy without issuing the copy (a flag
that nothing sets).  The CTA's final bounded wait gives up, the kernel
records MPCF_ERRBIT_TMA_TIMEOUT and returns with no copy in flight, the
host reads the status, and the same context then runs a clean stage whose
results equal a fresh solver's."""
import numpy as np
import pytest

from conftest import cloud_state
from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu


def test_bulk_copy_wait_runs_out_and_the_context_stays_usable(mpcf):
    dims = (32, 8, 12)             # one 32x8 tile, rows of 128 bytes: bulk copies
    U0 = cloud_state(dims, nb=1)
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_tiling(8, 6, persistent=False, tma=True)
        s.set_state(U0)
        s.set_test_flags(mpcf._lib.TEST_DROP_LAST_COPY)
        s.stage(0.0, 0.25, 0.05)
        w = s.error_word(clear=True)
        assert w & mpcf._lib.ERRBIT_TMA_TIMEOUT, hex(w)
        # the context is usable: a clean stage from the same state
        s.set_test_flags(0)
        s.set_state(U0)
        s.stage(0.0, 0.25, 0.05)
        assert s.error_word() == 0
        U, R = s.get_state()
    with mpcf.Solver([dims], precision="fp32_ref") as f:
        f.set_tiling(8, 6, persistent=False, tma=True)
        f.set_state(U0)
        f.stage(0.0, 0.25, 0.05)
        Uf, Rf = f.get_state()
    assert_bitwise(U, Uf, "state after the timed-out stage")
    assert_bitwise(R, Rf, "register after the timed-out stage")


def test_persistent_launches_ignore_the_test_flag(mpcf):
    dims = (32, 8, 12)
    with mpcf.Solver([dims], precision="mixed") as s:
        s.set_tiling(8, 6, persistent=True, tma=True)
        s.set_state(cloud_state(dims, nb=1))
        s.set_test_flags(mpcf._lib.TEST_DROP_LAST_COPY)
        s.stage(0.0, 0.25, 0.05)
        assert s.error_word() == 0
    with pytest.raises(mpcf.MpcfError):
        with mpcf.Solver([dims], precision="mixed") as s:
            s.set_test_flags(2)    # unknown flag
