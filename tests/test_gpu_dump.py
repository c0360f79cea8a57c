"""Dump, save and restart through the C ABI (mpcf_pack / mpcf_dump /
mpcf_save / mpcf_restart): the arrays equal the reference's streamers'
(golden record and the restatement), the files hold them, the XDMF wrapper
describes them, and a restart restores the state bit for bit."""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import oracle_lib as O
from conftest import cloud_state

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_dump.npz")


def test_pack_equals_reference_streamers(mpcf):
    g = np.load(GOLD)
    U = list(g["U"])
    with mpcf.Solver([(12, 10, 8)], precision="fp32_ref") as s:
        s.set_state(U)
        for kind in ("tensor", "save"):
            assert np.array_equal(s.pack(kind), g[kind]), kind


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_pack_in_chunks(mpcf, prec):
    """A domain larger than one 64 MiB staging chunk (several chunks)."""
    dims = (256, 192, 64)
    dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
    U = [a.astype(dt) for a in cloud_state(dims, nb=3)]
    with mpcf.Solver([dims], precision=prec) as s:
        s.set_state(U)
        for kind in ("tensor", "save"):
            assert np.array_equal(s.pack(kind), O.pack(U, dims, kind)), kind


def test_dump_files_and_xdmf(mpcf, tmp_path):
    dims = (40, 33, 20)
    U = cloud_state(dims, nb=2)
    with mpcf.Solver([dims], precision="fp32_ref") as s:
        s.set_state(U)
        s.dump(tmp_path, "data_0007", step=123)
    nx, ny, nz = dims
    raw = np.fromfile(tmp_path / "data_0007.bin", dtype="<f4").reshape(nz, ny, nx, 9)
    assert np.array_equal(raw, O.pack(U, dims, "tensor"))
    root = ET.parse(tmp_path / "data_0007.xmf").getroot()
    grid = root.find("Domain/Grid")
    assert grid.find("Time").get("Value") == "00123"
    assert grid.find("Topology").get("Dimensions") == f"{nz} {ny} {nx}"
    spacing = [float(v) for v in grid.find("Geometry/DataItem[@Name='Spacing']").text.split()]
    assert np.allclose(spacing, 1.0 / max(dims), rtol=1e-6)
    item = grid.find("Attribute/DataItem")
    assert item.get("Dimensions") == f"{nz} {ny} {nx} 9"
    assert item.get("Precision") == "4" and item.get("Format") == "Binary"
    assert item.text.strip() == "data_0007.bin"
    assert grid.find("Attribute").get("AttributeType") == "Tensor"


@pytest.mark.parametrize("prec", ["fp32_ref", "fp64"])
def test_save_restart_roundtrip(mpcf, tmp_path, prec):
    dims = (37, 21, 18)
    with mpcf.Solver([dims], precision=prec) as s:
        s.ic_sic_cloud(mpcf.sic_params(p0=100.0, shock_s=(0.2, 0, 0)), [(0.5, 0.4, 0.3, 0.15)])
        t = s.run(2, cfl=0.3, graph=False)[0]
        assert s.get_time() == t
        s.save(tmp_path, t, step=2, fcount=1)
        U0 = s.get_state(with_reg=False)
        s.run(3, cfl=0.3, graph=False)
        U5 = s.get_state(with_reg=False)
        t5 = s.get_time()
    # save.info keeps t to 15 significant digits, as the reference's
    # setprecision(15) does, so a restart resumes at t rounded to 15 digits
    t15 = float(f"{t:.15g}")
    info = (tmp_path / "save.info").read_text().split()
    assert float(info[0]) == t15 and info[1:] == ["2", "1"]
    with mpcf.Solver([dims], precision=prec) as s2:
        assert s2.restart(tmp_path / "nowhere") is None
        assert s2.restart(tmp_path) == (t15, 2, 1)
        assert s2.get_time() == t15
        U = s2.get_state(with_reg=False)
        for q in range(7):
            assert np.array_equal(U[q], U0[q]), q
        # the first stage multiplies the (cleared) register by a = 0, so the
        # continued run is the original one
        s2.run(3, cfl=0.3, graph=False)
        U = s2.get_state(with_reg=False)
        assert s2.get_time() == pytest.approx(t5, rel=1e-14)
        for q in range(7):
            assert np.array_equal(U[q], U5[q]), q


def test_restart_rejects_wrong_size(mpcf, tmp_path):
    with mpcf.Solver([(16, 16, 16)], precision="fp32_ref") as s:
        s.set_state(cloud_state((16, 16, 16), nb=1))
        s.save(tmp_path, 0.5, 3)
    with mpcf.Solver([(16, 16, 8)], precision="fp32_ref") as s:
        with pytest.raises(mpcf.MpcfError):
            s.restart(tmp_path)
