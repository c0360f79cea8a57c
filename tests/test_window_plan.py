"""The operation plan of windowed runs (mpcf_window_plan; CPU only, no device
work): the order in which mpcf_run_window enqueues uploads, sound-speed
reductions, dt, stages and downloads of z-chunks streamed through a few
device slots (the reference's GPUlab chunks, GPUlab.cpp:202-372).  The
sound-speed pass runs from the last chunk down and leaves the first chunks
in their slots for the first step.

An independent replay checks every plan: which chunk each slot holds after
every operation, and that each operation finds what it reads.  A stage of
chunk c reads chunks c-1 .. c+1 of the previous stage (stage 1: of the
upload), so those chunks must still sit in their slots; a slot takes its next
chunk only after its chunk was downloaded and the stage 3 above it (which
reads its top planes) is queued; dt comes after the sound speed of every
chunk of the step's input; every chunk of every step is uploaded, staged
three times and downloaded once.  The plan of one host-resident stage
(mpcf_window_stage, the shim's chunked process_all) is replayed the same way.
"""
import pytest

UPLOAD, SOS, DT, STAGE, DOWNLOAD = range(5)


def replay(plan, nch, ns, nsteps):
    """Raise AssertionError on the first operation whose inputs are not in
    place; return the count of each kind."""
    last = nch - 1
    hi = lambda c: min(c + 1, last)
    # chunk c of step n: the steps take the slots in turn (the sound-speed
    # pass, step -1, from slot 0)
    slot_of = lambda n, c: c % ns if n < 0 else (n * nch + c) % ns
    holds = [None] * ns            # (step, chunk) now in the slot
    done = set()                   # (kind, step, stage, chunk) already enqueued
    sos_done = set()
    count = [0] * 5
    for kind, n, k, c in plan:
        count[kind] += 1
        key = (kind, n, k, c)
        assert key not in done, ("repeated", key)
        if kind == UPLOAD:
            s = slot_of(n, c)
            prev = holds[s]
            if prev is not None:
                pn, pc = prev
                if pn < 0:
                    assert pc in sos_done, ("slot reused before its sound speed", key, prev)
                else:
                    assert (DOWNLOAD, pn, 0, pc) in done, ("slot reused before its download", key, prev)
                    above = pc if pc == last else pc + 1
                    assert (STAGE, pn, 2, above) in done, ("slot reused before the stage 3 above it", key, prev)
            holds[s] = (n, c)
        elif kind == SOS:
            assert holds[slot_of(-1, c)] == (-1, c), ("sound speed of a chunk not in its slot", key)
            sos_done.add(c)
        elif kind == DT:
            if n == 0:
                assert len(sos_done) == nch, ("dt before the sound speed of every chunk", key)
                # the pass ran from the last chunk down and left chunks
                # 0 .. ns-1 in place: they are the first step's input
                for s_ in range(min(ns, nch)):
                    assert holds[s_] == (-1, s_), ("the pass left the wrong chunk", s_, holds[s_])
                    holds[s_] = (0, s_)
                    done.add((UPLOAD, 0, 0, s_))
            else:
                for j in range(nch):
                    assert (STAGE, n - 1, 2, j) in done, ("dt before the previous step's stage 3", key, j)
        elif kind == STAGE:
            assert (DT, n, 0, 0) in done, ("stage before its dt", key)
            for j in range(max(0, c - 1), hi(c) + 1):
                assert holds[slot_of(n, j)] == (n, j), ("stage reads a chunk not in its slot", key, j, holds[slot_of(n, j)])
                if k == 0:
                    assert (UPLOAD, n, 0, j) in done, ("stage 1 before the upload", key, j)
                else:
                    assert (STAGE, n, k - 1, j) in done, ("stage before the previous stage", key, j)
        elif kind == DOWNLOAD:
            assert (STAGE, n, 2, c) in done, ("download before stage 3", key)
            assert holds[slot_of(n, c)] == (n, c), ("download of a chunk not in its slot", key)
        done.add(key)
    return count


CASES = [(16, 8), (16, 5), (16, 16), (7, 5), (48, 6), (3, 3), (2, 2), (1, 1), (5, 5), (9, 7), (32, 5), (6, 6)]


@pytest.mark.parametrize("nch,ns", CASES)
@pytest.mark.parametrize("nsteps", [1, 3])
def test_window_plan_is_complete_and_ordered(mpcf, nch, ns, nsteps):
    plan = mpcf.window_plan(nch, ns, nsteps).tolist()
    count = replay(plan, nch, ns, nsteps)
    # the sound-speed pass and every step, less the chunks the pass left in place
    assert count[UPLOAD] == nch * (nsteps + 1) - min(ns, nch)
    assert count[SOS] == nch
    assert count[DT] == nsteps
    assert count[STAGE] == 3 * nch * nsteps
    assert count[DOWNLOAD] == nch * nsteps


def test_window_plan_overlaps_chunks(mpcf):
    """The wavefront: with 16 chunks in 8 slots, the first chunk's stage 3
    and download are queued before the upload of chunk 8, and stage 3 of a
    chunk trails its stage 1 by two chunks."""
    plan = [tuple(r) for r in mpcf.window_plan(16, 8, 2).tolist()]
    pos = {r: i for i, r in enumerate(plan)}
    assert pos[(DOWNLOAD, 0, 0, 0)] < pos[(UPLOAD, 0, 0, 8)]
    for c in range(2, 15):
        assert pos[(STAGE, 0, 0, c)] < pos[(STAGE, 0, 2, c - 2)] < pos[(STAGE, 0, 0, c + 1)], c


@pytest.mark.parametrize("nch,ns", [(16, 4), (6, 3), (10, 2)])
def test_window_plan_rejects_too_few_slots(mpcf, nch, ns):
    with pytest.raises(mpcf.MpcfError, match="too few"):
        mpcf.window_plan(nch, ns, 1)


def replay_stage(plan, nch, ns):
    """The plan of one host-resident stage (mpcf_window_stage): a stage of
    chunk c reads the uploaded chunks c-1 .. c+1; a slot is reused only after
    its chunk was downloaded and the stage of the chunk above is queued."""
    last = nch - 1
    holds = [None] * ns
    done = set()
    for kind, n, k, c in plan:
        key = (kind, c)
        assert key not in done, ("repeated", key)
        s = c % ns
        if kind == UPLOAD:
            prev = holds[s]
            if prev is not None:
                assert (DOWNLOAD, prev) in done, ("slot reused before its download", c, prev)
                assert (STAGE, prev if prev == last else prev + 1) in done, ("slot reused before the stage above", c, prev)
            holds[s] = c
        elif kind == STAGE:
            for j in range(max(0, c - 1), min(c + 1, last) + 1):
                assert holds[j % ns] == j and (UPLOAD, j) in done, ("stage reads a chunk not in its slot", c, j)
        elif kind == DOWNLOAD:
            assert (STAGE, c) in done and holds[s] == c, ("download before its stage", c)
        else:
            raise AssertionError(("unexpected kind", kind))
        done.add(key)
    assert len(done) == 3 * nch


@pytest.mark.parametrize("nch,ns", [(1, 1), (2, 2), (3, 3), (5, 3), (12, 3), (12, 6), (42, 6), (4, 8)])
def test_window_stage_plan_is_complete_and_ordered(mpcf, nch, ns):
    replay_stage(mpcf.window_stage_plan(nch, ns).tolist(), nch, ns)


def test_window_stage_plan_rejects_too_few_slots(mpcf):
    with pytest.raises(mpcf.MpcfError, match="too few"):
        mpcf.window_stage_plan(6, 2)
