"""Known-answer and property tests of the CPU oracle (no GPU needed).

The reference's own regression fixtures (tests/test-grains/*) use a contact
tag the current Grains3D factory no longer parses, so they cannot pin the
HookeMemory law; these analytic checks and the golden vectors produced by the
reference itself (tests/golden/) do.
"""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle
from pacific_b200 import scenarios


def _two_spheres(tmp_path, kn=1e4, en=0.7, muc=0.5, etat=None, gravity=(0.0, 0.0, 0.0), dt=1e-6):
    sc = scenarios.settling_box(n=2, kn=kn, en=en, etat=etat, muc=muc, dt=dt)
    sc.gravity = gravity
    sc.walls = []
    sc.models = sc.models[:1]
    return sc, sc.write_xml(tmp_path / "two.xml")


def test_binary_collision_restitution_and_duration(tmp_path, oracle_lib):
    """Head-on collision: post-collision relative speed / pre = en, contact
    time = pi / sqrt(kn/m* - eta_n^2) (HookeMemoryContactForceModel::
    computeAndWriteEstimates, Component/src/HookeMemoryContactForceModel.cpp:319-388)."""
    kn, en, dt = 1e4, 0.7, 1e-7
    sc, xml = _two_spheres(tmp_path, kn=kn, en=en, dt=dt)
    r = sc.types[0]["radius"]
    x = np.array([[0.01, 0.015, 0.03], [0.01 + 2 * r + 1e-6, 0.015, 0.03]])
    v0 = 0.1
    v = np.array([[v0, 0, 0], [-v0, 0, 0]], float)
    o = Oracle(xml)
    o.set_particles(np.zeros(2, np.int32), x, v, np.zeros((2, 3)), np.tile([0, 0, 0, 1.0], (2, 1)))
    o.init()
    steps_in_contact = 0
    for _ in range(20000):
        o.step(1)
        if len(o.contacts()[0]):
            steps_in_contact += 1
        elif steps_in_contact:
            break
    s = o.state()
    vrel = s["v"][1, 0] - s["v"][0, 0]
    m = sc.types[0]["density"] * 4 / 3 * math.pi * r ** 3
    mstar = m / 2
    beta = math.log(en) / math.sqrt(math.pi ** 2 + math.log(en) ** 2)
    eta = -beta * math.sqrt(kn / mstar)
    tc = math.pi / math.sqrt(kn / mstar - eta ** 2)
    assert abs(vrel / (2 * v0) - en) < 2e-3
    assert abs(steps_in_contact * dt - tc) / tc < 2e-3


def test_sliding_contact_saturates_at_coulomb(tmp_path, oracle_lib):
    """A sphere sliding on a wall: the tangential force reaches mu_c |Fn|."""
    sc = scenarios.settling_box(n=1, muc=0.3, etat=None, dt=1e-6)
    r = sc.types[0]["radius"]
    xml = sc.write_xml(tmp_path / "slide.xml")
    o = Oracle(xml)
    m = sc.types[0]["density"] * 4 / 3 * math.pi * r ** 3
    x = np.array([[0.015, 0.015, r - m * 9.81 / 1e4]])     # resting overlap m g / kn
    o.set_particles(np.zeros(1, np.int32), x, np.array([[0.2, 0, 0]]), np.zeros((1, 3)),
                    np.array([[0, 0, 0, 1.0]]))
    o.init()
    o.step(200)
    id0, id1, dl, pt, f = o.contacts()
    assert len(id0) == 1 and id1[0] == -(4 + 2)     # bottom wall is the 5th obstacle
    fn = abs(f[0, 2])
    ft = math.hypot(f[0, 0], f[0, 1])
    assert fn > 0 and abs(ft - 0.3 * fn) / (0.3 * fn) < 1e-9


def test_periodic_gas_conserves_momentum(tmp_path, oracle_lib):
    sc = scenarios.periodic_gas(n_fcc=5, seed=3)
    xml = sc.write_xml(tmp_path / "gas.xml")
    o = Oracle(xml)
    o.set_particles(sc.type, sc.x, sc.v, sc.w, sc.q)
    o.init()
    m = np.array([t["density"] * 4 / 3 * math.pi * t["radius"] ** 3 for t in sc.types])[sc.type]
    p0 = (m[:, None] * sc.v).sum(0)
    ke0 = 0.5 * (m[:, None] * sc.v ** 2).sum()
    assert o.step(300) == 0
    s = o.state()
    p1 = (m[:, None] * s["v"]).sum(0)
    ke1 = 0.5 * (m[:, None] * s["v"] ** 2).sum()
    scale = (m[:, None] * np.abs(sc.v)).sum()
    assert np.all(np.abs(p1 - p0) < 1e-13 * scale)
    assert ke1 < ke0
    assert len(o.contacts()[0]) > 0


def test_cell_index_is_floor_of_offset(tmp_path, oracle_lib):
    """Cell::GetCell: floor((x - origin) / edge) (Base/src/Cell.cpp:172-184);
    periodic directions carry one extra cell layer on each side."""
    sc = scenarios.periodic_gas(n_fcc=5, seed=4)
    xml = sc.write_xml(tmp_path / "g.xml")
    o = Oracle(xml)
    o.set_particles(sc.type, sc.x, sc.v, sc.w, sc.q)
    nb, edge, org = o.grid()
    side = sc.maxc[0]
    n_in = int((side + 1e-10) / (2 * max(t["radius"] for t in sc.types)))
    assert np.all(nb == n_in + 2)
    assert np.allclose(edge, side / n_in, rtol=0, atol=0)
    expect = np.floor((sc.x - org) / edge).astype(int)
    assert np.array_equal(o.cells(), expect)


def test_motion_error_flag(tmp_path, oracle_lib):
    sc = scenarios.settling_box(n=8)
    xml = sc.write_xml(tmp_path / "m.xml")
    o = Oracle(xml)
    v = sc.v.copy()
    v[2] = [100.0, 0, 0]
    o.set_particles(sc.type, sc.x, v, sc.w, sc.q)
    o.init()
    assert o.step(1) & 2


@pytest.mark.parametrize("seed", [1, 2])
def test_scenarios_are_seeded(seed):
    a = scenarios.periodic_gas(n_fcc=4, seed=seed)
    b = scenarios.periodic_gas(n_fcc=4, seed=seed)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v) and np.array_equal(a.type, b.type)
    # no initial overlap on the lattice
    r = np.array([t["radius"] for t in a.types])[a.type]
    d = a.x[:, None, :] - a.x[None, :, :]
    L = a.maxc[0]
    d -= L * np.rint(d / L)
    dist = np.sqrt((d ** 2).sum(-1)) + np.eye(len(r)) * 1e9
    assert np.all(dist > r[:, None] + r[None, :])
