"""Format2024 reload particle files (gdem_read_reload_particles,
gdem_write_reload_particles), against a file written by the Grains3D
reference itself (tests/golden/reload_settling.npz, made by
tests/golden/make_golden.py with the reference's Particle::write2014).

* Reading the reference's file and stepping reproduces the reference's next
  states: one step to the golden tolerances of the FP64 mode (positions
  1e-15, forces 1e-10 of each particle's contact-force sum), and the cells
  and contact memory exactly; 50 steps to 1e-12 m.
* Writing right after reading gives the reference's file back, token for
  token, except the spheres' orientation matrices (the reference composes a
  rotation per step; the file written here has R(q)), which agree to 1e-12.
* A file written after N steps and read into a fresh system continues the
  run: byte for byte in FP32-split mode; in FP64 mode to round-off, because
  the file (like the reference's) holds no body-frame angular velocity,
  which is then rebuilt as q* w q a few ulps away from the integrated one.
"""
from pathlib import Path

import numpy as np
import pytest

from pacific_b200 import FP32_SPLIT, FP64, Grains, scenarios

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "reload_settling.npz"
# token layout of a particle line: class ID tag active | x(3) basis(9) type |
# v(3) q(4) w(3) F(3) T(3) | n ...
BASIS = slice(7, 16)


@pytest.fixture(scope="module")
def golden(tmp_path_factory, lib):
    g = np.load(GOLDEN)
    d = tmp_path_factory.mktemp("reload")
    xml = d / "reload.xml"
    xml.write_text(str(g["xml"]))
    pf = d / "reload_Particles"
    pf.write_text(str(g["particles"]))
    return g, str(xml), pf


def test_reference_file_then_steps(golden):
    g, xml, pf = golden
    sim = Grains(xml, FP64)
    sim.read_reload_particles(pf)
    sim.set_diagnostics(True)
    sim.step(1)
    s = sim.download_state()
    assert sim.status() == 0
    assert np.array_equal(sim.download_cells(), g["s1_cells"])
    id0, id1, _ = sim.download_contacts()
    ref = {(min(a, b), max(a, b)) if b >= 0 else (a, b)
           for a, b in zip(g["s1_hist_owner"].tolist(), g["s1_hist_partner"].tolist())}
    got = {(min(a, b), max(a, b)) if b >= 0 else (a, b) for a, b in zip(id0.tolist(), id1.tolist())}
    assert got == ref and len(ref) > 0
    assert np.max(np.abs(s["x"] - g["s1_x"])) <= 1e-15
    scale = g["s1_scale"]
    c = scale > 0
    assert c.any()
    fe = np.linalg.norm(s["F"] - g["s1_F"], axis=1)[c] / scale[c]
    te = np.linalg.norm(s["T"] - g["s1_T"], axis=1)[c] / (1e-3 * scale[c])
    assert fe.max() <= 1e-10 and te.max() <= 1e-10
    sim.set_diagnostics(False)
    sim.step(49)
    s = sim.download_state()
    assert np.max(np.abs(s["x"] - g["s50_x"])) <= 1e-12
    sim.close()


def test_write_after_read_gives_the_reference_file(golden, tmp_path):
    g, xml, pf = golden
    sim = Grains(xml, FP64)
    sim.read_reload_particles(pf)
    out = tmp_path / "again_Particles"
    sim.write_reload_particles(out)
    sim.close()
    ref_lines = pf.read_text().splitlines()
    got_lines = out.read_text().splitlines()
    assert len(got_lines) == len(ref_lines)
    for r, o in zip(ref_lines, got_lines):
        rt, ot = r.split(), o.split()
        assert len(rt) == len(ot)
        assert rt[:BASIS.start] == ot[:BASIS.start]
        assert rt[BASIS.stop:] == ot[BASIS.stop:]
        rb = np.array(rt[BASIS], dtype=float)
        ob = np.array(ot[BASIS], dtype=float)
        assert np.max(np.abs(rb - ob)) <= 1e-12


@pytest.mark.parametrize("precision", [FP64, FP32_SPLIT], ids=["fp64", "fp32split"])
def test_round_trip_continues_the_run(tmp_path, lib, precision):
    sc = scenarios.settling_box(n=300, seed=29)
    xml = str(sc.write_xml(tmp_path / "rt.xml"))
    a = Grains(xml, precision)
    a.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    a.do_before_time_stepping()
    a.step(400)
    pf = tmp_path / "rt_Particles"
    a.write_reload_particles(pf)
    b = Grains(xml, precision)
    b.read_reload_particles(pf)
    a.step(150)
    b.step(150)
    sa, sb = a.download_state(), b.download_state()
    assert a.status() == 0 and b.status() == 0
    if precision == FP32_SPLIT:
        for k in ("x", "v", "w", "q", "F", "T"):
            assert np.array_equal(sa[k], sb[k]), k
    else:
        assert np.max(np.abs(sa["x"] - sb["x"])) <= 1e-12
        for k in ("v", "w", "F", "T"):
            assert np.max(np.abs(sa[k] - sb[k])) <= 1e-7 * np.abs(sa[k]).max(), k
    a.close()
    b.close()


def test_reload_velocity_reset(golden, tmp_path):
    """<Reload ... Velocity="Reset"/> (Grains::Construction then
    AllComponents::resetKinematics, ParticleKinematics::reset): the particles
    of the file with zero translational and angular velocities and identity
    quaternions; positions, orientation matrices, forces and contact memory
    as read."""
    g, xml, pf = golden
    text = Path(xml).read_text()
    assert "<Construction>" in text
    rxml = tmp_path / "reset.xml"
    rxml.write_text(text.replace(
        "<Construction>",
        f'<Construction>\n    <Reload Type="new" Filename="{tmp_path}/none" Velocity="Reset"/>', 1))
    keep = Grains(xml, FP64)
    keep.read_reload_particles(pf)
    sk = keep.download_state()
    keep.close()
    sim = Grains(str(rxml), FP64)
    sim.read_reload_particles(pf)
    s = sim.download_state()
    sim.close()
    assert np.abs(sk["v"]).max() > 0
    assert not s["v"].any() and not s["w"].any()
    assert np.array_equal(s["q"], np.tile([0.0, 0.0, 0.0, 1.0], (len(s["q"]), 1)))
    for k in ("x", "F", "T"):
        assert np.array_equal(s[k], sk[k]), k
