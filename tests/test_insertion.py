"""Particle insertion during a run (gdem_reserve / gdem_insert_particle,
Grains::insertParticle with LinkedCell::insertParticleSerial).

* The overlap test decides as RigidBodyWithCrust::isContact does: a
  candidate on top of a particle, across a periodic boundary from one, or
  into a wall is refused; one at a free spot goes in; ForceInsertion puts it
  in regardless.  Boxes: refused when the bodies overlap, accepted when only
  their circumscribed spheres do -- unless the test is the bounding-volume
  one (GeometricOverlap Value="BV").
* An inserted particle is the same as one that was there from the start:
  stepping on after the insertion equals, to the bit, a system uploaded with
  the state, forces and contact memory that the insertion left.
"""
import numpy as np
import pytest

from pacific_b200 import FP32_SPLIT, FP64, Grains, GrainsError, scenarios
from pacific_b200.scenarios import Scenario

pytestmark = pytest.mark.gpu


def _free_spot(state, radii, r, box, rng):
    """A point at least r + radius + 1e-4 from every particle and 2r from the walls."""
    lo = np.array([2 * r] * 3)
    hi = np.array(box) - 2 * r
    for _ in range(10000):
        p = lo + rng.random(3) * (hi - lo)
        d = np.linalg.norm(state["x"] - p, axis=1) - radii - r
        if d.min() > 1e-4:
            return p
    raise AssertionError("no free spot")


@pytest.mark.parametrize("precision", [FP64, FP32_SPLIT], ids=["fp64", "fp32split"])
def test_insertion_decisions_and_equivalence(tmp_path, lib, precision):
    sc = scenarios.settling_box(n=300, seed=12, box=(0.02, 0.02, 0.05))
    xml = str(sc.write_xml(tmp_path / "box.xml"))
    r = sc.types[0]["radius"]
    g = Grains(xml, precision)
    g.reserve(8)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    g.step(200)
    s = g.download_state()
    radii = np.full(sc.n, r)
    # on top of a particle, half-way into a wall, far outside: refused
    assert g.insert_particle(0, s["x"][7]) is None
    assert g.insert_particle(0, s["x"][7] + np.array([1.9 * r, 0., 0.])) is None
    assert g.insert_particle(0, (0.5 * r, 0.01, 0.04)) is None
    rng = np.random.default_rng(5)
    p = _free_spot(s, radii, r, (0.02, 0.02, 0.05), rng)
    pid = g.insert_particle(0, p, v=(0.01, -0.02, 0.0), w=(3.0, 0.0, 1.0))
    assert pid == sc.n and g.n == sc.n + 1
    # just out of touch with particle 7 (the sum of radii plus 1e-9 m)
    x7 = s["x"][7]
    d = np.array([0., 0., 1.])
    near = x7 + d * (2 * r + 1e-9)
    others = np.delete(s["x"], 7, axis=0)
    if (np.linalg.norm(others - near, axis=1) > 2 * r).all() and near[2] < 0.05 - r:
        assert g.insert_particle(0, near) == sc.n + 1
        n_in = sc.n + 2
    else:
        n_in = sc.n + 1
    # the new particle's force is its weight, its torque zero
    after = g.download_state()
    m = 2500.0 * 4.0 / 3.0 * np.pi * r ** 3
    assert np.allclose(after["F"][sc.n], [0.0, 0.0, -9.81 * m], rtol=1e-12, atol=0.0)
    assert np.array_equal(after["T"][sc.n], [0.0, 0.0, 0.0])
    h = g.download_history()
    # the same state uploaded into a fresh system steps to the same bits
    b = Grains(xml, precision)
    b.upload_state(np.concatenate([sc.type, np.zeros(n_in - sc.n, np.int32)]), after["x"],
                   after["v"], after["w"], after["q"], wbf=after["wbf"])
    b.upload_forces(after["F"], after["T"])
    b.upload_history(h["owner"], h["partner"], h["kdelta"], h["prevn"], h["spring"])
    g.step(150)
    b.step(150)
    sa, sb = g.download_state(), b.download_state()
    assert g.status() == 0 and b.status() == 0
    for k in ("x", "v", "w", "q", "F", "T"):
        assert np.array_equal(sa[k], sb[k]), k
    # the inserted particle moved (it falls under gravity)
    assert sa["x"][sc.n][2] < p[2]
    g.close()
    b.close()
    # room: a system without reserve refuses an insertion with an error
    c = Grains(xml, precision)
    c.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    with pytest.raises(GrainsError):
        c.insert_particle(0, p)
    c.close()


def test_forced_insertion(tmp_path, lib):
    sc = scenarios.settling_box(n=50, seed=3, box=(0.02, 0.02, 0.05))
    xml = str(sc.write_xml(tmp_path / "box.xml"))
    g = Grains(xml, FP64)
    g.reserve(1)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    assert g.insert_particle(0, sc.x[3]) is None
    assert g.insert_particle(0, sc.x[3] + 1e-4, force=True) == sc.n
    g.close()


def test_insertion_across_periodic_boundary(tmp_path, lib):
    """A candidate near the x = L face that overlaps, through the boundary, a
    particle near the x = 0 face (and nothing directly) is refused; moved
    2e-5 m away from that image it goes in."""
    sc = scenarios.periodic_gas(n_fcc=4, seed=9, spacing=3.0e-3)
    xml = str(sc.write_xml(tmp_path / "gas.xml"))
    L = np.array(sc.maxc) - np.array(sc.origin)
    g = Grains(xml, FP64)
    g.reserve(2)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    s = g.download_state()
    radii = np.array([t["radius"] for t in sc.types])[sc.type]
    r0 = sc.types[0]["radius"]
    shift = np.array([L[0], 0.0, 0.0])
    found = False
    for i in np.argsort(s["x"][:, 0]):
        cand = s["x"][i] + shift - np.array([radii[i] + r0 - 1e-6, 0.0, 0.0])
        if not (sc.origin[0] <= cand[0] < sc.maxc[0]):
            continue
        direct = np.linalg.norm(s["x"] - cand, axis=1) - radii - r0
        images = np.linalg.norm(s["x"] + shift - cand, axis=1) - radii - r0
        others = np.delete(np.minimum(direct, images), i)
        if direct.min() > 1e-4 and others.min() > 1e-4:
            found = True
            break
    assert found
    assert g.insert_particle(0, cand) is None
    assert g.insert_particle(0, cand - np.array([2e-5, 0.0, 0.0])) == sc.n
    g.close()


def _two_cubes(tmp_path, gap, bv):
    edge = 2.0e-3
    r = edge * np.sqrt(3.0) / 2.0
    crust = 0.1 * r
    types = [dict(shape="box", size=(edge,) * 3, radius=float(r), crust=float(crust),
                  density=2500.0, material="matP")]
    models = [dict(matA="matP", matB="matP", kn=1e4, en=0.7, etat=None, muc=0.5, kt=2e4 / 7),
              dict(matA="matP", matB="matW", kn=1e4, en=0.7, etat=None, muc=0.5, kt=2e4 / 7)]
    box = (0.02, 0.02, 0.02)
    sc = Scenario("cubes", (0.0, 0.0, 0.0), box, (0, 0, 0), (0.0, 0.0, 0.0), 1e-5, types,
                  scenarios._box_walls(box, 2e-3, float(crust), "matW"), models,
                  np.zeros(1, np.int32), np.array([[0.01, 0.01, 0.01]]), np.zeros((1, 3)),
                  np.zeros((1, 3)), np.array([[0.0, 0.0, 0.0, 1.0]]))
    xml = str(sc.write_xml(tmp_path / f"cubes_{gap}_{bv}.xml"))
    g = Grains(xml, FP64)
    g.reserve(1)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    # face to face along x, the faces `gap` apart (negative: overlapping)
    out = g.insert_particle(0, (0.01 + edge + gap, 0.01, 0.01), bv_only=bv)
    g.close()
    return out


def test_box_insertion_gjk_and_bounding_volume(tmp_path, lib):
    assert _two_cubes(tmp_path, 1e-5, False) == 1        # apart: GJK says no contact
    assert _two_cubes(tmp_path, -1e-5, False) is None    # overlapping
    assert _two_cubes(tmp_path, 1e-5, True) is None      # circumscribed spheres overlap
