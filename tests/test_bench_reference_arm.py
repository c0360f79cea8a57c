"""bench.py's reference arm runs on the host cores (the CPU restatement of
the reference kernels), so its JSON line is checked here without a GPU:
the keys of the bench contract, the reference-arm keys and a throughput
that matches its own sample."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CONTRACT = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
            "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e")


def test_reference_arm_prints_one_contract_line(monkeypatch):
    env = dict(os.environ, OMP_NUM_THREADS="2", MPCF_CPU_SAMPLE_PLANES="16")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "c1_64", "--steps", "2", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    for k in CONTRACT:
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is True
    assert d["unit"] == "cell-stage updates/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1 and "cpu_model" in d["cpu_baseline"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the sample: the middle 16 planes of the 64^3 domain; ms_per_step is its
    # measured step time, and the value is the sample's throughput
    assert "64x64x16 z-slab at planes 24-39" in d["config"]["cpu_sample"]
    assert abs(d["ms_per_step"] - 3 * 64 * 64 * 16 / d["value"] * 1e3) < 1e-6 * d["ms_per_step"]
    # the reference arm maps no library of the product, only the oracle's
    assert d["native_libs"], d
    assert all(l.startswith("oracle/") for l in d["native_libs"]), d["native_libs"]
    # the same config object as the GPU arm's line
    sys.path.insert(0, ROOT)
    import bench
    import oracle_lib as O
    from mpcf import configs
    monkeypatch.setattr(bench, "CPU_SAMPLE_PLANES", 16)
    assert d["config"] == bench.bench_config(configs.config("c1_64", placer=O.bubbles), 1)


def test_cpu_sample_is_a_slab_of_the_workload():
    """The oracle's cloud set-up of the sample equals the same planes of the
    whole domain's (library host generator), and the oracle's placement
    equals the library's."""
    import numpy as np
    import mpcf
    import oracle_lib as O
    sys.path.insert(0, ROOT)
    import bench
    cfg = mpcf.configs.config("c1_64")
    cfg_o = mpcf.configs.config("c1_64", placer=O.bubbles)
    assert all(np.array_equal(a, b) for a, b in zip(cfg["bubbles"], cfg_o["bubbles"]))
    dims, org, glob = bench.cpu_sample_block(cfg)
    sub = bench.cpu_sample_state(cfg)
    full = mpcf.ic_cloud_host(glob, cfg["params"], cfg["bubbles"][0], np.float32)
    n = dims[0] * dims[1]
    for q in range(7):
        assert np.array_equal(sub[q], full[q][org[2] * n:(org[2] + dims[2]) * n])


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "c1_64", "--steps", "1", "--warmup", "0", "--gpus", "2"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]
