"""bench.py under torchrun: every rank builds its solvers on its own GPU
(LOCAL_RANK), not on GPU 0.  Checked on the CPU with a stand-in Solver that
records the device it is given."""
import importlib.util
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(os.path.dirname(HERE), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


class FakeSolver:
    made = []

    def __init__(self, dims, precision="fp32_ref", device=0, **kw):
        FakeSolver.made.append(device)

    def ic_cloud(self, params, bubbles, dom=0):
        pass


class FakeMpcf:
    Solver = FakeSolver


def test_each_rank_uses_its_local_gpu(monkeypatch):
    bench = load_bench()
    cfg = {"dims": [(8, 8, 8)], "bubbles": [None], "params": None}
    FakeSolver.made.clear()
    for local in (0, 3, 7):
        monkeypatch.setenv("RANK", str(local))
        monkeypatch.setenv("LOCAL_RANK", str(local))
        monkeypatch.setenv("WORLD_SIZE", "8")
        bench.make_solver(FakeMpcf, cfg, "mixed")
    monkeypatch.delenv("RANK")
    monkeypatch.delenv("LOCAL_RANK")
    monkeypatch.delenv("WORLD_SIZE")
    bench.make_solver(FakeMpcf, cfg, "mixed")          # no torchrun: GPU 0
    assert FakeSolver.made == [0, 3, 7, 0]
