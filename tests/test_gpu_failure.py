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


def test_no_copy_is_issued_after_a_give_up_and_none_is_left_in_flight(mpcf):
    """The chunk's first copy after the prologue is dropped: the wait one slab
    in runs out, the CTA issues no further copy (the count stops at the 3
    copies issued before: the prologue's two and the halo box issued with
    the dropped one), waits for that halo box before it exits (no
    MPCF_ERRBIT_TMA_INFLIGHT), and the context stays usable."""
    dims = (32, 8, 12)             # one 32x8 tile, two 6-slab chunks
    U0 = cloud_state(dims, nb=1)
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_tiling(8, 6, persistent=False, tma=True)
        s.set_state(U0)
        # a clean launch with the counter on (the last copy dropped: one
        # copy fewer than the 13 per chunk of a full chunk)
        s.set_test_flags(mpcf._lib.TEST_DROP_LAST_COPY)
        s.test_copy_count(clear=True)
        s.stage(0.0, 0.25, 0.05)
        assert s.test_copy_count(clear=True) == 2 * 12
        s.error_word(clear=True)
        s.set_state(U0)
        s.set_test_flags(mpcf._lib.TEST_DROP_MID_COPY)
        s.stage(0.0, 0.25, 0.05)
        w = s.error_word(clear=True)
        assert w & mpcf._lib.ERRBIT_TMA_TIMEOUT, hex(w)
        assert not (w & mpcf._lib.ERRBIT_TMA_INFLIGHT), hex(w)
        assert s.test_copy_count(clear=True) == 2 * 3
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
    assert_bitwise(U, Uf, "state after the given-up stage")
    assert_bitwise(R, Rf, "register after the given-up stage")


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
            s.set_test_flags(4)    # unknown flag
