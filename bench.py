#!/usr/bin/env python
"""Benchmark: cell-stage updates/s of the CUBISM-MPCF hot path on B200.

Workload (one GPU): 512^3 cells, a cloud of 200 non-overlapping gas bubbles
(radii U[0.02,0.06], centres uniform in [0.2,0.8]^3, seeded rejection
sampling) in a stiffened-gas liquid at p=1000 (gamma=6.59, pc=4096,
rho=1000; gas gamma=1.4, pc=0, rho=1, p=0.0234), tanh interface over 1.5
cells, U(-1e-3,1e-3) velocity noise, absorbing boundaries, CFL 0.3.
Synthetic inputs of that shape (no dataset is involved).

One step = max speed of sound + on-device dt + three LSRK3 stages, replayed
as a CUDA graph over device-resident state (inputs 11 GB > L2, so no flush
is needed between steps).  The headline `value` is the MIXED form
(FP32 bulk, compensated FP32 pressure recovery, FP64 conservation sums); the line also
carries the all-FP64 throughput on the same workload and the L1 / L-inf
error of rho, p and G of the mixed run against the FP64 run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference algorithm's CPU implementation (the
C restatement in oracle/, OpenMP over all host cores; the reference's own
GPU convection does not build with CUDA 12) on a bounded sample of the
same workload.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "cubism-jr-gpu-mpcf_b200"))

WORKLOAD = "c3_512"
METRIC = "cell-stage updates/s on 1 B200: mixed vs plain FP64 at stated L1 error"
UNIT = "cell-stage updates/s"
BYTES_PER_CELL_STAGE = {"fp32_ref": 112, "fp32": 112, "mixed": 112, "fp64": 224, "fp64_fast": 224}
# DRAM bytes per cell-stage of the mixed stage kernel measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum = 2.135 + 1.831 GB for one
# launch over the 512 x 512 x 128 lower quarter of the 512^3 cloud, 33.55 M
# cells, 32 x 8 tiles over whole columns, persistent, bulk-copy staging: a
# few-GB case of the bench's kernel and tiling).  The per-launch figure of the
# bench line is this times the workload's cells.
# the arithmetic each precision form computes in, and its name in the workload
DTYPE_OF = {"mixed": "f32+f64 (mixed)", "fp32": "f32", "fp32_ref": "f32 (reference rounding)", "fp64": "f64",
            "fp64_fast": "f64 (fast form)"}
FORM_OF = {"mixed": "mixed form", "fp32": "fast FP32 form", "fp32_ref": "FP32 reference-rounding form",
           "fp64": "FP64 form", "fp64_fast": "fast FP64 form (factored algebra, refined reciprocals)"}
MEASURED_DRAM_BYTES_PER_CELL_STAGE = {"mixed": (2.135219968e9 + 1.831107072e9) / (512 * 512 * 128)}


# Algorithmic floating-point operations of one cell-stage, counted by
# oracle/count_ops (the oracle's face pipeline run with an operation-counting
# number type; add/sub/mul/div/sqrt/compare/min/max = 1, FMA = 2):
# 3 faces x 1546 (WENO5 x 14, wave speeds, HLLC, u*) + 13 (primitive
# conversion, once per cell) + 91 (extra terms, divergence, updates).
# tests/test_oracle.py checks this constant against the counter.
FLOPS_PER_CELL_STAGE = 4742


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def make_solver(mpcf, cfg, precision):
    # one GPU per rank: the rank's local GPU under torchrun (LOCAL_RANK), else 0
    s = mpcf.Solver(cfg["dims"], precision=precision, device=env_rank()[2])
    for d, bub in enumerate(cfg["bubbles"]):
        s.ic_cloud(cfg["params"], bub, dom=d)
    return s


def all_state(s):
    """First 7 fields of every domain, concatenated (precision comparisons)."""
    parts = [s.get_state(dom=d, with_reg=False) for d in range(s.ndom)]
    if len(parts) == 1:
        return parts[0]
    return [np.concatenate([p[q] for p in parts]) for q in range(7)]


CHUNK = 1 << 24


def derived_chunk(st, sl):
    """(rho, p, G) in FP64 of cells `sl` of a stored state."""
    rho = st[0][sl].astype(np.float64)
    ke = st[1][sl].astype(np.float64) ** 2 + st[2][sl].astype(np.float64) ** 2 + st[3][sl].astype(np.float64) ** 2
    G = st[5][sl].astype(np.float64)
    p = (st[4][sl].astype(np.float64) - 0.5 * ke / rho - st[6][sl]) / G
    return rho, p, G


def derived_fields(st):
    """(rho, p, G) in FP64 of a stored state, computed in chunks of cells."""
    n = st[0].size
    out = [np.empty(n, np.float64) for _ in range(3)]
    for i in range(0, n, CHUNK):
        sl = slice(i, min(n, i + CHUNK))
        for o, v in zip(out, derived_chunk(st, sl)):
            o[sl] = v
    return out


def errors_against(st, ref):
    """Relative L1 (mean |x - x64| / mean |x64|) and L-inf (max |x - x64| /
    max |x64|) of rho, p and G of state `st` against the FP64 run's `ref`,
    accumulated in chunks of cells."""
    n = st[0].size
    acc = np.zeros((3, 4))          # sum |d|, sum |ref|, max |d|, max |ref|
    for i in range(0, n, CHUNK):
        sl = slice(i, min(n, i + CHUNK))
        for k, v in enumerate(derived_chunk(st, sl)):
            r = ref[k][sl]
            d = np.abs(v - r)
            a = np.abs(r)
            acc[k] += (d.sum(), a.sum(), 0, 0)
            acc[k, 2] = max(acc[k, 2], d.max())
            acc[k, 3] = max(acc[k, 3], a.max())
    out = {}
    for k, name in enumerate(("rho", "p", "G")):
        out["L1_" + name] = float(acc[k, 0] / acc[k, 1])
        out["Linf_" + name] = float(acc[k, 2] / acc[k, 3])
    return out


def time_steps(mpcf, s, steps, warmup, cfl, dist=None):
    """Device-timed graph replay of `steps` LSRK3 steps; returns ms (max over ranks)."""
    import torch
    s.run(warmup, cfl=cfl, graph=True)
    s.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    # events on the solver's own stream are not reachable from torch; the
    # library replays the graph on its stream and synchronises it, and the
    # elapsed device time is taken with CUDA events around the same replay
    # inside mpcf_time_run (below)
    ms = run_timed(mpcf, s, steps, cfl)
    torch.cuda.synchronize()
    if dist is not None:
        import mpcf.replicas as rp
        ms = rp.max_over_ranks(dist, ms, device="cuda")
        dist.barrier()
    return ms


def run_timed(mpcf, s, steps, cfl):
    L = mpcf.lib()
    ms = ctypes.c_double()
    mpcf._lib.check(L.mpcf_time_run(s._h, int(steps), float(cfl), 1e30, ctypes.byref(ms)))
    return ms.value


def stage_kernel_ms(mpcf, s, reps=6):
    """Average duration of one stage-kernel launch (CUDA events on the
    solver's stream), for the roofline."""
    return s.time_stages(reps, dtinvh=0.0)


# The CPU sample of a workload: the middle CPU_SAMPLE_PLANES-plane z-slab of
# its first domain (its whole first domain when that is thinner), with the
# domain's cell spacing, bubbles and material data; one LSRK3 step of it per
# timed step.
CPU_SAMPLE_PLANES = int(os.environ.get("MPCF_CPU_SAMPLE_PLANES", "32"))


def cpu_sample_block(cfg):
    """(dims, origin, global dims) of the CPU sample of workload `cfg`."""
    nx, ny, nz = cfg["dims"][0]
    p = min(nz, CPU_SAMPLE_PLANES)
    z0 = (nz - p) // 2
    return (nx, ny, p), (0, 0, z0), (nx, ny, nz)


def cpu_sample_name(cfg):
    (nx, ny, p), (_, _, z0), _ = cpu_sample_block(cfg)
    return f"one LSRK3 step of the {nx}x{ny}x{p} z-slab at planes {z0}-{z0 + p - 1} of the first domain"


def cpu_sample_state(cfg):
    """The sample's FP32 state from the oracle's restatement of the cloud
    set-up (the product library is not loaded)."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_lib as O
    dims, org, glob = cpu_sample_block(cfg)
    return O.ic_cloud(dims, cfg["params"], cfg["bubbles"][0], np.float32, origin=org, glob=glob)


def cpu_step(dims, U0, threads):
    """One oracle LSRK3 step of the sample (C restatement, OpenMP); returns
    seconds."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_lib as O
    os.environ["OMP_NUM_THREADS"] = str(threads)
    U = [a.copy() for a in U0]
    R = [np.zeros_like(a) for a in U]
    t0 = time.perf_counter()
    O.step(dims, (0,) * 6, U, R, cfl=0.3)
    return time.perf_counter() - t0


def cpu_model():
    """The host CPU's model name (first entry of /proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def loaded_libs():
    """Shared objects of this repository mapped into this process."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if line.strip() else ""
                if path.endswith(".so") or ".so." in path:
                    if os.path.realpath(path).startswith(os.path.realpath(REPO) + os.sep):
                        out.add(os.path.relpath(os.path.realpath(path), os.path.realpath(REPO)))
    except OSError:
        pass
    return sorted(out)


def bench_config(cfg, world):
    """The `config` object of both arms' lines (the workload, not the
    implementation)."""
    return {"workload": cfg["name"] + ": " + cfg["desc"] + ", absorbing, CFL 0.3",
            "cells_per_gpu": sum(d[0] * d[1] * d[2] for d in cfg["dims"]),
            "l2": "inputs larger than the 126 MB L2 (no flush needed)" if cfg["name"] != "c1_64"
                  else "state 7.3 MB: L2-resident, no flush (latency-bound size)",
            "parallelism": "replicas" if world > 1 else "single GPU",
            "cpu_sample": cpu_sample_name(cfg)}


def reference_arm(args):
    """The reference algorithm's CPU implementation (the oracle: the C
    restatement of the reference kernels, OpenMP over all host cores) on a
    bounded sample of the workload; the product library is never loaded."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_lib as O
    from mpcf import configs   # plain data and numpy: loads no library
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    cfg = configs.config(args.workload, placer=O.bubbles)
    sub, _, _ = cpu_sample_block(cfg)
    U0 = cpu_sample_state(cfg)
    secs = []
    for i in range(args.warmup + args.steps):
        dt = cpu_step(sub, U0, cores)
        if i >= args.warmup:
            secs.append(dt)
    n_sub = sub[0] * sub[1] * sub[2]
    value = 3.0 * n_sub * len(secs) / sum(secs)
    sample = ("C restatement of the reference kernels (oracle/), FP32 reference rounding, OpenMP over "
              f"{cores} threads, {cpu_sample_name(cfg)}")
    # the reference's own CPU sound speed (source/MaxSpeedOfSound.cpp, compiled
    # from its sources into oracle/_ref, serial as written) on the same sample
    sos = None
    L = O.ref_lib("libref_sos")
    if L is not None:
        t0 = time.perf_counter()
        reps = 3
        for _ in range(reps):
            L.ref_max_sos_cpp(n_sub, O.fptrs(U0))
        sec = (time.perf_counter() - t0) / reps
        sos = {"value": n_sub / sec, "unit": "cells/s", "cores": 1, "kind": "reference",
               "sample": f"MaxSpeedOfSound_CPP::compute over the {sub[0]}x{sub[1]}x{sub[2]} sample"}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": bench_config(cfg, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                             "cpu_model": cpu_model()},
            "reference_sos_cpu": sos,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "native_libs": loaded_libs()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--only-mixed-fp64", action="store_true", help="skip the fp32_ref / fp32 throughput runs")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp32_ref", "fp64", "fp64_fast"],
                    help="precision of the headline run (profiling of the other forms)")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--e2e-chunks", type=int, default=8, help="z-chunks of the streamed e2e run")
    ap.add_argument("--window-slots", type=int, default=8,
                    help="device slots of the windowed e2e run (0: skip it)")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = tdist
    else:
        torch.cuda.set_device(0)
    import mpcf
    cfg = mpcf.configs.config(args.workload)
    ncell = sum(d[0] * d[1] * d[2] for d in cfg["dims"])
    K, W = args.steps, max(3, args.warmup)
    cfl = mpcf.configs.CFL

    # ---------------- mixed (headline): W warm-up + K timed graph replays
    s = make_solver(mpcf, cfg, args.precision)
    s.set_tiling(*pick_tiling(mpcf, s))
    s.track_conservation(True)
    sums0 = s.conserved_sums()
    clocks = ClockSampler(local)
    clocks.start()
    ms = time_steps(mpcf, s, K, W, cfl, dist)
    clk = clocks.stop()
    value = world * ncell * 3.0 * K / (ms * 1e-3)
    ms_step = ms / K
    sums1 = s.conserved_sums()
    # the device error word after the warm-up and timed steps (0: every
    # update stayed physical, every sound speed real and finite)
    err_word = s.error_word()
    # states of the forms compared with the FP64 run, kept until it exists;
    # the FP64 run's (rho, p, G)
    states, ref64 = {}, None
    if rank == 0:
        states[args.precision] = all_state(s)
    # roofline of the dominant kernel (the stage) on this same solver
    st_ms = stage_kernel_ms(mpcf, s)
    nt, grid, threads = s.launch_shape()
    tiling = s.tiling()
    s.close()
    hbm, peak_kind = measured_peaks()
    bytes_launch = BYTES_PER_CELL_STAGE["mixed"] * ncell
    achieved = bytes_launch / (st_ms * 1e-3) / 1e9

    # ---------------- the other precisions on the same workload and steps
    others = {}
    err_by = {}
    precs = [] if args.no_fp64 else ["fp64", "fp64_fast"]
    if not args.no_fp64 and not args.only_mixed_fp64:
        precs += ["fp32_ref", "fp32", "mixed"]
    precs = [p for p in precs if p != args.precision]
    for prec in precs:
        so = make_solver(mpcf, cfg, prec)
        so.set_tiling(*pick_tiling(mpcf, so))
        mso = time_steps(mpcf, so, K, W, cfl, dist)
        others[prec] = {"value": world * ncell * 3.0 * K / (mso * 1e-3), "ms_per_step": mso / K,
                        "tiling": so.tiling()}
        if rank == 0:
            if prec == "fp64":
                ref64 = derived_fields(all_state(so))
            else:
                states[prec] = all_state(so)
        so.close()
        if rank == 0 and ref64 is not None:
            # errors against the FP64 run as soon as both exist; the states
            # are then dropped (1024^3 states are tens of GB)
            for pr in list(states):
                err_by[pr] = errors_against(states.pop(pr), ref64)
    err = None
    if err_by:
        err = dict(err_by)
        err["note"] = ("relative L1 (mean |x-x64| / mean |x64|) and L-inf (max |x-x64| / max |x64|) "
                       "against the all-FP64 GPU run after the same %d steps (W+K) from the same IC" % (W + K))
    states.clear()
    ref64 = None

    # ---------------- e2e through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = e2e_measure(mpcf, cfg, K=K, W=W, cfl=cfl, dist=dist, precision=args.precision, tiling=tiling,
                          nchunks=args.e2e_chunks, window_slots=args.window_slots)
    # the same for the drop-in form (FP32 reference rounding, bit-identical
    # to the reference's arithmetic), on its own tiling
    e2e_drop_in = None
    if not args.no_e2e and args.precision != "fp32_ref" and "fp32_ref" in others:
        e2e_drop_in = e2e_measure(mpcf, cfg, K=K, W=W, cfl=cfl, dist=dist, precision="fp32_ref",
                                  tiling=others["fp32_ref"]["tiling"], nchunks=args.e2e_chunks, serial_form=False)

    # ---------------- CPU baseline (rank 0, N=1 only): the oracle on the
    # workload's CPU sample, its state from the oracle's cloud set-up
    cpu = None
    if not args.no_cpu and world == 1 and rank == 0:
        cores = os.cpu_count() or 1
        sub, _, _ = cpu_sample_block(cfg)
        dtc = cpu_step(sub, cpu_sample_state(cfg), cores)
        cpu = {"value": 3.0 * sub[0] * sub[1] * sub[2] / dtc, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "C restatement of the reference kernels (oracle/), FP32 reference rounding, OpenMP over "
                         "%d threads, %s (%.1f s)" % (cores, cpu_sample_name(cfg), dtc), "cpu_model": cpu_model()}

    if rank == 0:
        fp32_peak = ctypes.c_double()
        mpcf._lib.check(mpcf.lib().mpcf_probe_fp32_peak(local, ctypes.byref(fp32_peak)))
        fp64 = others.get("fp64", {}).get("value")
        fp64f = others.get("fp64_fast", {}).get("value")
        ach_tf = FLOPS_PER_CELL_STAGE * ncell / (st_ms * 1e-3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE_OF[args.precision], "data": "synthetic",
            "config": bench_config(cfg, world),
            "form": FORM_OF[args.precision],
            "tiling": {"ty": tiling[0], "dz": tiling[1], "persistent": tiling[2], "tma": tiling[3], "graph": True},
            "fp64_value": fp64, "mixed_over_fp64": (value / fp64) if fp64 else None,
            "fp64_fast_value": fp64f, "mixed_over_fp64_fast": (value / fp64f) if fp64f else None,
            "other_precisions": others,
            "precision_error": err,
            "conservation_drift": {"mass": float((sums1[:, 0].sum() - sums0[:, 0].sum()) / sums0[:, 0].sum()),
                                   "energy": float((sums1[:, 4].sum() - sums0[:, 4].sum()) / sums0[:, 4].sum()),
                                   "note": "FP64 sums over W+K steps, absorbing boundaries (boundary fluxes included)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm,
                         "traffic": (MEASURED_DRAM_BYTES_PER_CELL_STAGE[args.precision] * ncell
                                     if args.precision in MEASURED_DRAM_BYTES_PER_CELL_STAGE else None),
                         "traffic_note": "ncu DRAM bytes of one launch over the 512x512x128 lower quarter of the cloud "
                                         "(32x8 tiles, whole columns, persistent, TMA), scaled by the cells of a launch",
                         "kernel": "stage_kernel<Pol%s>" % {"mixed": "Mixed", "fp32": "Fast32", "fp32_ref": "Ref32", "fp64": "FP64",
                                                             "fp64_fast": "Fast64"}[args.precision],
                         "ms_per_launch": st_ms,
                         "algorithmic_bytes_per_launch": bytes_launch, "peak_kind": peak_kind,
                         "note": "the stage kernel is bound by the FP32 pipe, not HBM: see roofline_fp32"},
            "roofline_fp32": {"bound": "fp32", "achieved": ach_tf, "peak": fp32_peak.value, "unit": "TFLOP/s",
                              "frac": ach_tf / fp32_peak.value, "flops_per_cell_stage": FLOPS_PER_CELL_STAGE,
                              "peak_kind": "measured (mpcf_probe_fp32_peak, FMA chains)"},
            # per timed step: dt, three stages, the tile sums of stage 3;
            # the sound speed comes fused from the previous step's last
            # stage (the stand-alone reduction ran in the first warm-up step)
            "gpu_launches": 5 * K,
            "device_error_word": err_word,
            "clocks": clk,
            "e2e": e2e,
            "e2e_drop_in": e2e_drop_in,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def pick_tiling(mpcf, s):
    """Tiling for the bench: MPCF_TILING="ty,dz,persistent" if set, else the
    library's autotuner on the solver's own state (state left unchanged)."""
    env = os.environ.get("MPCF_TILING")
    if env:
        v = [int(x) for x in env.split(",")]
        return v[0], v[1], bool(v[2]), bool(v[3]) if len(v) > 3 else True
    try:
        best, _ = s.autotune(reps=2)
    except mpcf.MpcfError:
        # no room for the autotuner's scratch register (FP64 at 1024^3):
        # the solver's own tiling
        return s.tiling()
    return best


def pcie_peak(nbytes=1 << 30, chunks=16, reps=5):
    """Measured host-device copy rates (GB/s, 1e9 B): page-locked host
    buffer to device, device to host, and both directions at once on two
    streams (the rate each direction keeps while the other runs), in
    `chunks` copies of nbytes/chunks each way per repetition."""
    import torch
    n = nbytes // 4
    cs = n // chunks
    host_a = torch.empty(n, dtype=torch.float32, pin_memory=True)
    host_b = torch.empty(n, dtype=torch.float32, pin_memory=True)
    dev_a = torch.empty(n, dtype=torch.float32, device="cuda")
    dev_b = torch.empty(n, dtype=torch.float32, device="cuda")
    host_a.fill_(1.0)
    dev_b.fill_(1.0)
    up, down = torch.cuda.Stream(), torch.cuda.Stream()

    def h2d():
        with torch.cuda.stream(up):
            for c in range(chunks):
                dev_a[c * cs:(c + 1) * cs].copy_(host_a[c * cs:(c + 1) * cs], non_blocking=True)

    def d2h():
        with torch.cuda.stream(down):
            for c in range(chunks):
                host_b[c * cs:(c + 1) * cs].copy_(dev_b[c * cs:(c + 1) * cs], non_blocking=True)

    def rate(*fns):
        for f in fns:
            f()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            for f in fns:
                f()
        torch.cuda.synchronize()
        return reps * cs * chunks * 4 / (time.perf_counter() - t0) / 1e9

    out = {"h2d_gbs": rate(h2d), "d2h_gbs": rate(d2h), "both_gbs_per_direction": rate(h2d, d2h),
           "sample": f"{chunks} copies of {cs * 4 >> 20} MiB each way, {reps} repetitions"}
    del host_a, host_b, dev_a, dev_b
    torch.cuda.empty_cache()
    return out


def window_measure(mpcf, cfg, K, W, cfl, dist, precision, tiling, host, nslots, nslices=32):
    """The same steps through a windowed solver (mpcf_run_window): the
    domain streamed through `nslots` device slots of `nslices` planes, as a
    domain larger than device memory runs; each call's first step adds a
    pass that streams the state once more for its sound speed."""
    import mpcf.replicas as rp
    dims = cfg["dims"][0]
    ncell = dims[0] * dims[1] * dims[2]
    with mpcf.WindowSolver(dims, nslices, nslots, precision=precision) as w:
        if tiling is not None:
            w.set_tiling(tiling[0], nslices, tiling[2], tiling[3])
        w.run(host, W, cfl=cfl)
        import torch
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        w.run(host, K, cfl=cfl)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        esz = 8 if precision in ("fp64", "fp64_fast") else 4
        slot_bytes = 3 * 7 * esz * dims[0] * dims[1] * (nslices + 6)
        v, _ = rp.throughput(dist, ncell, 3.0 * K, sec * 1e3, device="cuda" if dist is not None else None)
        out = {"value": v, "unit": UNIT, "ms_per_step": sec * 1e3 / K, "nslices": nslices, "slots": w.nslots,
               "device_bytes": w.nslots * slot_bytes, "resident_bytes": 3 * 7 * esz * ncell,
               "path": f"mpcf_run_window: {w.nchunks} chunks of {nslices} planes through {w.nslots} device slots, "
                       f"host wall clock over one call of {K} steps"}
        # the reference's per-stage form (the shim's GPUlab for a block that
        # does not fit): every stage streams the state and the register
        # through the slots and back, every step streams the state once more
        # for its sound speed (mpcf_window_max_sos, mpcf_window_stage)
        reg = [torch.zeros(ncell, dtype=torch.float64 if esz == 8 else torch.float32, pin_memory=True)
               for _ in range(7)]
        regs = [r.numpy() for r in reg]
        h = 1.0 / max(dims)

        def per_stage(k):
            for _ in range(k):
                dt = cfl * h / w.max_sos_host(host)
                for a, b in mpcf.LSRK3:
                    w.stage_host(host, regs, a, b, dt / h)

        ks = 2
        per_stage(1)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        per_stage(ks)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        v, _ = rp.throughput(dist, ncell, 3.0 * ks, sec * 1e3, device="cuda" if dist is not None else None)
        out["per_stage"] = {"value": v, "unit": UNIT, "ms_per_step": sec * 1e3 / ks,
                            "h2d_bytes_per_step": (1 + 3 * 2) * 7 * esz * ncell,
                            "d2h_bytes_per_step": 3 * 2 * 7 * esz * ncell,
                            "path": f"mpcf_window_max_sos + 3 x mpcf_window_stage per step (state and register in "
                                    f"host memory, the reference's per-stage streaming), {ks} steps"}
        del reg, regs
        return out


def e2e_measure(mpcf, cfg, K, W, cfl, dist, precision="mixed", tiling=None, nchunks=8, serial_form=True,
                window_slots=0):
    """Same metric through the C ABI with the state in page-locked host
    memory, as the reference keeps it: every step reads its input state from
    the host buffers and writes its result back to them (mpcf_run_host: z-chunk
    uploads, the three stages as a wavefront over the chunks, each chunk
    downloaded as soon as stage 3 has written it, the next step's upload of
    a chunk after its download, copies in both directions overlapping the
    kernels).  The register stays on the
    device (stage 1 multiplies it by a = 0), so the state is the step's whole
    input and result.  Host wall clock over the K timed steps.  Also the
    serial form: mpcf_set_state + mpcf_step + mpcf_get_state per step."""
    import torch
    s = make_solver(mpcf, cfg, precision)
    L = mpcf.lib()
    if tiling is not None:
        ty, _, persist, tma = tiling
        nz = cfg["dims"][0][2]
        s.set_tiling(ty, max(1, nz // nchunks), persist, tma)
    dtype = torch.float64 if precision in ("fp64", "fp64_fast") else torch.float32
    esz = 8 if precision in ("fp64", "fp64_fast") else 4
    ncell = sum(d[0] * d[1] * d[2] for d in cfg["dims"])
    streamed = len(cfg["dims"]) == 1
    bufs = []
    for d, dims in enumerate(cfg["dims"]):
        n = dims[0] * dims[1] * dims[2]
        h = [torch.empty(n, dtype=dtype, pin_memory=True) for _ in range(7)]
        st = s.get_state(dom=d, with_reg=False)
        for q in range(7):
            h[q].numpy()[:] = st[q]
        del st
        bufs.append((h, (ctypes.c_void_p * 7)(*[h[q].data_ptr() for q in range(7)])))
    import mpcf.replicas as rp

    def timed(fn, k):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn(k)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    out = {"unit": UNIT, "h2d_bytes_per_step": 7 * esz * ncell, "d2h_bytes_per_step": 7 * esz * ncell}
    if streamed:
        host = [b.numpy() for b in bufs[0][0]]
        s.run_host(host, W, cfl=cfl, nchunks=nchunks)
        sec = timed(lambda k: s.run_host(host, k, cfl=cfl, nchunks=nchunks), K)
        out["value"], _ = rp.throughput(dist, ncell, 3.0 * K, sec * 1e3, device="cuda" if dist is not None else None)
        out["path"] = (f"mpcf_run_host: state in pinned host memory read and written every step, {nchunks} z-chunks, "
                       f"tiling {list(s.tiling())}, host wall clock over {K} steps")
        # the bound of a streamed step: its bytes each way at the measured
        # rate of concurrent host-to-device and device-to-host copies
        pk = pcie_peak()
        bound_ms = out["h2d_bytes_per_step"] / (pk["both_gbs_per_direction"] * 1e9) * 1e3
        step_ms = sec * 1e3 / K
        out["roofline"] = {"bound": "pcie", "achieved": out["h2d_bytes_per_step"] / step_ms / 1e6,
                           "peak": pk["both_gbs_per_direction"], "unit": "GB/s per direction",
                           "frac": bound_ms / step_ms, "bound_ms_per_step": bound_ms, "ms_per_step": step_ms,
                           "copies": pk}
        if window_slots:
            try:
                out["window"] = window_measure(mpcf, cfg, K, W, cfl, dist, precision, tiling, host, window_slots)
            except Exception as e:          # a side leg: the line stands without it
                out["window"] = {"error": f"{type(e).__name__}: {e}"}

    def serial(k):
        for _ in range(k):
            for d, (_, up) in enumerate(bufs):
                mpcf._lib.check(L.mpcf_set_state(s._h, d, up, None, 0))
            mpcf._lib.check(L.mpcf_step(s._h, cfl, 1e30, None))
            for d, (_, up) in enumerate(bufs):
                mpcf._lib.check(L.mpcf_get_state(s._h, d, up, None, 0))

    if streamed and not serial_form:
        s.close()
        return out
    ks = max(2, min(K, 4))
    serial(1)
    sec = timed(serial, ks)
    v, _ = rp.throughput(dist, ncell, 3.0 * ks, sec * 1e3, device="cuda" if dist is not None else None)
    ser = {"value": v, "unit": UNIT, "path": f"mpcf_set_state + mpcf_step + mpcf_get_state per step, {ks} steps"}
    if streamed:
        out["serial"] = ser
    else:
        out.update(ser)
    s.close()
    return out


if __name__ == "__main__":
    sys.exit(main())
