"""The drop-in shim fails loudly on a hand-written halo fill.

The B200 lab synthesises its ghost cells on the device from the boundary
conditions that a GPUlab subclass states through
BoundaryConditions::applyBC_absorbing / applyBC_reflecting (every lab of the
reference does).  A subclass whose _apply_bc writes halox/haloy/haloz by
hand (an inflow condition, say) cannot be honoured: the first load_ghosts
call finds the halo buffers changed, prints the lab's error and exits with
status 1, like the reference's configuration errors (GPUlab.cpp:37-47).
The harness (tests/shim/halo_check.cpp) is compiled here against the shim
sources and libmpcf_b200.so."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SHIM = os.path.join(ROOT, "cubism-jr-gpu-mpcf_b200", "shim")
LIBDIR = os.path.join(ROOT, "cubism-jr-gpu-mpcf_b200", "lib")


@pytest.fixture(scope="module")
def harness(tmp_path_factory, mpcf):
    mpcf.lib()   # the library is built
    exe = str(tmp_path_factory.mktemp("shim") / "halo_check")
    cmd = ["g++", "-O1", "-std=c++11", "-w", "-D_FLOAT_PRECISION_", "-D_BLOCKSIZEX_=32", "-D_BLOCKSIZEY_=24",
           "-D_BLOCKSIZEZ_=16", "-DNDEBUG", "-DWENOEPS=1e-6", "-I" + SHIM, "-I" + os.path.join(SHIM, "compat"),
           "-I/usr/local/cuda/include", os.path.join(HERE, "shim", "halo_check.cpp"),
           os.path.join(SHIM, "GPUlab.cpp"), os.path.join(SHIM, "GPU.cpp"), os.path.join(SHIM, "Types.cpp"),
           "-L" + LIBDIR, "-lmpcf_b200", "-Wl,-rpath," + LIBDIR, "-o", exe]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    return exe


def test_boundary_conditions_through_the_interface_run(harness):
    p = subprocess.run([harness, "bc"], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "halo_check bc: ok" in p.stdout


def test_hand_written_halo_fill_stops_the_lab(harness):
    p = subprocess.run([harness, "raw"], capture_output=True, text=True, timeout=120)
    assert p.returncode == 1, (p.returncode, p.stdout, p.stderr)
    assert "[GPUlab ERROR: _apply_bc wrote the halo buffers directly" in p.stderr
    assert "not detected" not in p.stdout
