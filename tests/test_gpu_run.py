"""The simulation runner (mpcf.run) on the GPU: the reference's loop with
dumps at the dump times, saves and a restart that continues the run bit for
bit, and every case's initial condition as the API sets it."""
import io

import numpy as np
import pytest

from mpcf import run as R

pytestmark = pytest.mark.gpu

SOD = ["-sim", "SodMPI", "-nx", "64", "-ny", "8", "-nz", "8", "-cfl", "0.3", "-nslices", "8", "-autotune", "0"]


def run(argv):
    out = io.StringIO()
    sim = R.Simulation(argv, out=out)
    try:
        sim.run()
        return sim.t, sim.step, out.getvalue()
    finally:
        sim.close()


def test_dumps_land_on_the_dump_times(tmp_path):
    t, step, log = run(SOD + ["-tend", "0.03", "-dumpinterval", "0.01", "-saveinterval", "1000",
                              "-fpath", str(tmp_path), "-verb", "1"])
    assert log.count("step time") == step
    assert t == pytest.approx(0.03, rel=1e-12)
    # the IC, the three dump times (the last is tend) and the final dump
    names = sorted(p.name for p in tmp_path.glob("data_*.bin"))
    assert names == ["data_%04d.bin" % i for i in range(5)], names
    times = [float(l.split("time ")[1]) for l in log.splitlines() if l.startswith("Dumping")]
    assert times[:4] == pytest.approx([0.0, 0.01, 0.02, 0.03], abs=1e-6)


def test_restart_continues_the_run(tmp_path):
    # dumps far apart, so the time step is the CFL step throughout (the
    # reference's restart moves the next dump time one interval on)
    common = SOD + ["-tend", "10", "-dumpinterval", "100", "-saveinterval", "6"]
    a, b = tmp_path / "a", tmp_path / "b"
    run(common + ["-fpath", str(a), "-nsteps", "12"])
    ta, sa, log = run(common + ["-fpath", str(a), "-restart", "1", "-nsteps", "18"])
    assert "Restarting at step 12" in log and sa == 18
    tb, sb, _ = run(common + ["-fpath", str(b), "-nsteps", "18"])
    assert sb == 18 and ta == pytest.approx(tb, rel=1e-13)
    assert (a / "save.data.bin").read_bytes() == (b / "save.data.bin").read_bytes()
    assert (a / "restart_ic_0001.bin").exists()


def test_restart_without_a_save_fails(tmp_path):
    with pytest.raises(R.ArgumentError):
        run(SOD + ["-tend", "1", "-dumpinterval", "1", "-saveinterval", "1", "-restart", "1",
                   "-fpath", str(tmp_path)])


CASES = {
    "SteadyStateMPI": (["-rho", "2", "-u", "0.5", "-p", "3", "-g", "1.67", "-pc", "1"],
                       lambda s: s.ic_steady(rho=2, u=0.5, p=3, g=1.67, pc=1)),
    "SodMPI": (["-config", "y", "-reverse", "1", "-rho1", "2"],
               lambda s: s.ic_sod(config="y", reverse=1, rho1=2)),
    "2DSBIMPI": (["-config", "xz", "-mollfactor", "2", "-mach", "1.5"],
                 lambda s: s.ic_sbi(np.array([[0.5, 0.25, 0.125, 0.1]]), config="xz", mollfactor=2, mach=1.5)),
    "SICCloudMPI": (["-pressureratio", "20", "-shockSx", "0.1"],
                    lambda s: s.ic_sic_cloud(R.S.sic_params(pressure_ratio=20, shock_s=(0.1, 0.0, 0.0)),
                                             np.array([[0.4, 0.25, 0.125, 0.06], [0.6, 0.2, 0.1, 0.05]]))),
}


@pytest.mark.parametrize("case", list(CASES))
def test_cases_start_from_the_api_initial_condition(tmp_path, monkeypatch, case):
    import mpcf
    flags, api = CASES[case]
    monkeypatch.chdir(tmp_path)
    (tmp_path / "xzbubbles.dat").write_text("1\n0.5 0.25 0.125 0.1\n")
    (tmp_path / "cloud.dat").write_text("0 0.4 0.25 0.125 0.06\n1 0.6 0.2 0.1 0.05\n")
    dims = (32, 16, 8)
    run(["-sim", case, "-nx", "32", "-ny", "16", "-nz", "8", "-tend", "1", "-cfl", "0.3", "-nslices", "8",
         "-dumpinterval", "1", "-saveinterval", "100", "-nsteps", "2", "-autotune", "0",
         "-fpath", str(tmp_path / "run")] + flags)
    sim = R.Simulation(["-sim", case, "-nx", "32", "-ny", "16", "-nz", "8", "-dryrun", "1"] + flags)
    (tmp_path / "api").mkdir()
    with mpcf.Solver([dims], bc=[sim._bc()], precision="fp32_ref") as s:
        api(s)
        s.dump(tmp_path / "api", "ic", 0)
    assert (tmp_path / "run" / "data_0000.bin").read_bytes() == (tmp_path / "api" / "ic.bin").read_bytes()


@pytest.mark.parametrize("config", ["xy", "zx", "yz"])
def test_static_ic_counts_cells_in_the_config_order(tmp_path, config):
    nx, ny, nz = 8, 6, 4
    run(["-sim", "StaticIC", "-config", config, "-nx", str(nx), "-ny", str(ny), "-nz", str(nz),
         "-fpath", str(tmp_path)])
    dump = np.fromfile(tmp_path / "staticIC_0000.bin", dtype="<f4").reshape(nz, ny, nx, 9)
    n = {"x": nx, "y": ny, "z": nz}
    fast, mid = config
    slow = ({"x", "y", "z"} - set(config)).pop()
    cnt = 0
    expect = np.empty((nz, ny, nx), np.float32)
    ranges = {a: range(n[a]) for a in "xyz"}
    for k in ranges[slow]:
        for j in ranges[mid]:
            for i in ranges[fast]:
                idx = {fast: i, mid: j, slow: k}
                expect[idx["z"], idx["y"], idx["x"]] = cnt
                cnt += 1
    assert np.array_equal(dump[..., 0], expect)      # rho holds the count
    assert np.array_equal(dump[..., 5], expect)      # and so does G
