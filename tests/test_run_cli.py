"""The simulation runner's command line (mpcf.run), without a GPU: the
reference's "-key value" parsing, its mandatory arguments, its case names
and its input files (2DSBI bubbles, cloud-collapse shapes)."""
import io

import numpy as np
import pytest

from mpcf import run as R

BASE = ["-nx", "16", "-ny", "8", "-nz", "8"]
MANDATORY = ["-tend", "0.1", "-cfl", "0.3", "-nslices", "8", "-dumpinterval", "0.05", "-saveinterval", "10"]


def test_arguments_parse_like_the_reference():
    a = R.Arguments(["stray", "-sim", "SodMPI", "-cfl", "0.3", "-cfl", "0.25", "-reverse", "-fname", "a", "b",
                     "-shockNx", "-1", "-x0", "-0.25"])
    assert a.str("sim") == "SodMPI"
    assert a.float("cfl") == 0.25                 # the last value wins
    assert a.bool("reverse") and a.str("reverse") == "1"   # a bare option is "1"
    assert not a.bool("restart")
    assert a.str("fname") == "a b"                # values joined by spaces
    assert a.float("shockNx") == -1.0 and a.float("x0") == -0.25   # negative numbers are values
    assert not a.has("stray")
    assert a.int("nsteps", 0) == 0
    with pytest.raises(R.ArgumentError):
        a.float("tend")                           # mandatory, missing


@pytest.mark.parametrize("missing", ["-tend", "-cfl", "-nslices", "-dumpinterval", "-saveinterval"])
def test_mandatory_arguments(missing):
    argv = list(MANDATORY)
    i = argv.index(missing)
    del argv[i:i + 2]
    with pytest.raises(R.ArgumentError):
        R.Simulation(["-sim", "SodMPI"] + BASE + argv)
    # a dry run needs none of them
    R.Simulation(["-sim", "SodMPI", "-dryrun", "1"] + BASE)


@pytest.mark.parametrize("flag,value", [("-saveinterval", "0"), ("-dumpinterval", "0"), ("-cfl", "-0.3")])
def test_run_options_are_validated(flag, value):
    argv = list(MANDATORY)
    argv[argv.index(flag) + 1] = value
    with pytest.raises(R.ArgumentError):
        R.Simulation(["-sim", "SodMPI"] + BASE + argv)


def test_cases_and_limits():
    with pytest.raises(R.ArgumentError):
        R.Simulation(["-sim", "NoSuchCase"] + BASE + MANDATORY)
    with pytest.raises(R.ArgumentError):
        R.Simulation(["-sim", "SodMPI", "-npez", "2"] + BASE + MANDATORY)
    with pytest.raises(R.ArgumentError):
        R.Simulation(["-sim", "SodMPI", "-precision", "fp16"] + BASE + MANDATORY)
    s = R.Simulation(["-sim", "SodMPI", "-precision", "mixed"] + BASE + MANDATORY)
    assert (s.dims, s.precision, s.case, s.nsteps, s.fpath) == ((16, 8, 8), "mixed", "SodMPI", 0, ".")
    assert R.Simulation(BASE + MANDATORY).case == "SteadyStateMPI"      # the reference's default


def test_dry_run_touches_no_gpu():
    out = io.StringIO()
    s = R.Simulation(["-sim", "SICCloudMPI", "-dryrun", "1"] + BASE, out=out)
    s.run()
    assert "Dry Run..." in out.getvalue() and s.solver is None


def test_case_options_keep_the_reference_names():
    a = R.Arguments(["-config", "y", "-reverse", "1", "-rho1", "2.0", "-p2", "0.2"])
    assert R._case_kwargs(a, "SodMPI") == {"config": "y", "reverse": 1, "rho1": 2.0, "p2": 0.2}
    a = R.Arguments(["-config", "xz", "-mach", "1.5", "-mollfactor", "2"])
    assert R._case_kwargs(a, "2DSBIMPI") == {"config": "xz", "reverse": 0, "mollfactor": 2, "mach": 1.5}


def test_input_files(tmp_path):
    (tmp_path / "xybubbles.dat").write_text("2\n0.5 0.3 0.4 0.1\n0.2 0.4 0.25 0.08\n")
    b = R.read_bubbles(tmp_path / "xybubbles.dat")
    assert b.shape == (2, 4) and b[1, 3] == 0.08
    (tmp_path / "short.dat").write_text("3\n0.5 0.3 0.4 0.1\n")
    with pytest.raises(R.ArgumentError):
        R.read_bubbles(tmp_path / "short.dat")
    (tmp_path / "cloud.dat").write_text("0 0.1 0.2 0.3 0.05\n1 0.4 0.5 0.6 0.07\n\n")
    c = R.read_cloud(tmp_path / "cloud.dat")
    assert np.array_equal(c, [[0.1, 0.2, 0.3, 0.05], [0.4, 0.5, 0.6, 0.07]])


def test_static_ic_takes_no_run_options():
    s = R.Simulation(["-sim", "StaticIC", "-config", "zx", "-fname", "pattern"] + BASE)
    assert (s.config, s.fname) == ("zx", "pattern")
    for bad in ("xx", "xyz", "ab"):
        with pytest.raises(R.ArgumentError):
            R.Simulation(["-sim", "StaticIC", "-config", bad] + BASE)
    with pytest.raises(R.ArgumentError):
        R.Simulation(["-sim", "StaticIC"] + BASE)          # -config is mandatory
