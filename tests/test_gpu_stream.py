"""Runs over a host-resident state (mpcf_run_host): the reference's
host-resident block streamed through the GPU (GPUlab.cpp:202-372,703-793).

Every step uploads the state from host memory in z-chunks and runs the three
stages as a wavefront over the chunks: a stage of a chunk follows the stage
before it (stage 1: the upload) on every chunk within 3 planes above, and each
chunk of the new state is downloaded as soon as stage 3 has written it; the
next step's upload of a chunk follows its download.  The first step reduces
the sound speed chunk by chunk as the chunks land, later steps take the one
stage 3 accumulated.  The result must be bit-identical to the same steps of a
device-resident run (mpcf_run), for any chunking, chunks thinner than the
3-plane stencil reach included."""
import numpy as np
import pytest

from conftest import cloud_state
from test_gpu_parity import assert_bitwise

pytestmark = pytest.mark.gpu


def resident(mpcf, dims, prec, U0, tiling, steps):
    with mpcf.Solver([dims], precision=prec) as s:
        s.set_tiling(*tiling)
        s.set_state(U0)
        t = s.run(steps, cfl=0.3, graph=False)[0]
        return t, s.get_state(with_reg=False)


@pytest.mark.parametrize("prec,tiling,nchunks", [
    ("fp32_ref", (7, 16, True, True), 4),      # 6 tile layers in 4 chunks
    ("mixed", (8, 16, True, True), 6),         # one layer per chunk
    ("mixed", (8, 32, False, True), 2),
    ("fp64", (3, 16, False, False), 3),
    ("fp32", (8, 96, True, True), 4),          # one layer: a single chunk
    ("mixed", (8, 2, True, True), 48),         # 2-plane chunks: a stage waits for 2 above
    ("fp32_ref", (3, 1, True, True), 32),      # 3-plane chunks of 1-plane layers
])
def test_streamed_run_equals_resident_run(mpcf, prec, tiling, nchunks):
    dims = (64, 48, 96)
    dtype = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    U0 = cloud_state(dims, nb=3, seed=21, dtype=dtype)
    t_res, U_res = resident(mpcf, dims, prec, U0, tiling, 3)
    host = [np.ascontiguousarray(a, dtype=dtype).copy() for a in U0]
    with mpcf.Solver([dims], precision=prec) as s:
        s.set_tiling(*tiling)
        s.set_state(U0)
        t = s.run_host(host, 3, cfl=0.3, nchunks=nchunks)
        assert s.error_word() == 0
        dev = s.get_state(with_reg=False)
        # a device-resident step after the streamed ones continues the same run
        s.run(1, cfl=0.3, graph=True)
        after = s.get_state(with_reg=False)
    assert t == t_res, (t, t_res)
    assert_bitwise(host, U_res, f"host state, {prec} {tiling} in {nchunks} chunks")
    assert_bitwise(dev, U_res, "device state after the streamed run")
    _, U4 = resident(mpcf, dims, prec, U0, tiling, 4)
    assert_bitwise(after, U4, "a resident step after the streamed run")


def test_streamed_run_from_pinned_memory(mpcf):
    """Page-locked host buffers (the overlapping case), graph steps before
    and a second streamed call after: the same as one resident run."""
    import torch
    dims = (96, 64, 128)
    U0 = cloud_state(dims, nb=4, seed=5)
    _, U_res = resident(mpcf, dims, "mixed", U0, (8, 16, True, True), 5)
    host = [torch.empty(U0[0].size, dtype=torch.float32, pin_memory=True) for _ in range(7)]
    with mpcf.Solver([dims], precision="mixed") as s:
        s.set_tiling(8, 16, True, True)
        s.set_state(U0)
        s.run(1, cfl=0.3, graph=True)
        st = s.get_state(with_reg=False)
        for q in range(7):
            host[q].numpy()[:] = st[q]
        arrs = [h.numpy() for h in host]
        s.run_host(arrs, 2, nchunks=8)
        s.run_host(arrs, 2, nchunks=3)
        assert s.error_word() == 0
    assert_bitwise(arrs, U_res, "pinned host state")


def test_streamed_run_rejects_what_it_cannot_stream(mpcf):
    with mpcf.Solver([(32, 16, 16), (32, 16, 16)], precision="mixed") as s:
        host = [np.zeros(32 * 16 * 16, np.float32) for _ in range(7)]
        with pytest.raises(mpcf.MpcfError, match="one domain"):
            s.run_host(host, 1)
    with mpcf.Solver([(32, 16, 16)], precision="mixed") as s:
        with pytest.raises(ValueError):
            s.run_host([np.zeros(10, np.float32)] * 7, 1)
        with pytest.raises(mpcf.MpcfError):
            s.run_host([np.zeros(32 * 16 * 16, np.float32)] * 7, 1, nchunks=0)
