"""Analytic known answers, on the CPU restatement (oracle/) and on the CUDA
path in both precision modes.

* Head-on collision of two spheres under HookeMemory: the relative speed
  after / before is en and the contact lasts pi / sqrt(kn/m* - eta_n^2)
  (HookeMemoryContactForceModel::computeAndWriteEstimates,
  Component/src/HookeMemoryContactForceModel.cpp:319-388).
* A sphere sliding on a wall: the tangential force saturates at muc |Fn|
  (HookeMemoryContactForceModel::performForcesCalculus, Coulomb cap).
* Two cubes of half edge H and crust c (RigidBodyWithCrust::ClosestPoint,
  Geometry/src/RigidBodyWithCrust.cpp:277-351: GJK between the bodies
  shrunk by their crust, overlap = distance - 2c), at rest: face to face at
  centre distance 2H - d, edge to face (one cube turned 45 degrees about z)
  at (H - c)(1 + sqrt 2) + 2c - d, corner to face (its body diagonal along
  x) at (H - c)(1 + sqrt 3) + 2c - d all overlap by d, and the first force
  evaluation gives kn d along x.
"""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle
from pacific_b200 import FP32_SPLIT, FP64, Grains, scenarios

IMPLS = [pytest.param("oracle", id="oracle"),
         pytest.param(FP64, id="fp64", marks=pytest.mark.gpu),
         pytest.param(FP32_SPLIT, id="fp32split", marks=pytest.mark.gpu)]


class _Run:
    """One system on the oracle or on the GPU, behind one small interface."""

    def __init__(self, impl, sc, xml, basis=False):
        self.impl = impl
        b = scenarios.rotation_matrices(sc.q) if basis else None
        if impl == "oracle":
            self.o = Oracle(xml)
            assert self.o.set_particles(sc.type, sc.x, sc.v, sc.w, sc.q, b) == 0
            assert self.o.init() == 0
        else:
            self.g = Grains(xml, impl)
            self.g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
            self.g.set_diagnostics(True)
            self.g.do_before_time_stepping()

    def step(self, k=1):
        if self.impl == "oracle":
            assert self.o.step(k) == 0
        else:
            self.g.step(k)

    def contacts(self):
        """(id0, id1, overlap distance, force on id0) of the last force evaluation."""
        if self.impl == "oracle":
            id0, id1, dl, _, f = self.o.contacts()
            return id0, id1, dl, f
        return self.g.download_contacts(forces=True)

    def state(self):
        return self.o.state() if self.impl == "oracle" else self.g.download_state()

    def close(self):
        if self.impl != "oracle":
            assert self.g.status() == 0
            self.g.close()


def _backend(request, impl):
    """Builds and loads what the implementation needs: the oracle's library
    for the CPU runs, the CUDA library for the GPU runs."""
    request.getfixturevalue("oracle_lib" if impl == "oracle" else "lib")


@pytest.mark.parametrize("impl", IMPLS)
def test_binary_collision_restitution_and_duration(tmp_path, request, impl):
    _backend(request, impl)
    kn, en, dt = 1e4, 0.7, 1e-7
    sc = scenarios.settling_box(n=2, kn=kn, en=en, etat=None, muc=0.5, dt=dt)
    sc.gravity = (0.0, 0.0, 0.0)
    sc.walls = []
    sc.models = sc.models[:1]
    r = sc.types[0]["radius"]
    v0 = 0.1
    sc.type = np.zeros(2, np.int32)
    sc.x = np.array([[0.01, 0.015, 0.03], [0.01 + 2 * r + 1e-6, 0.015, 0.03]])
    sc.v = np.array([[v0, 0, 0], [-v0, 0, 0]], float)
    sc.w = np.zeros((2, 3))
    sc.q = np.tile([0, 0, 0, 1.0], (2, 1))
    run = _Run(impl, sc, str(sc.write_xml(tmp_path / "two.xml")))
    steps_in_contact = 0
    for _ in range(20000):
        run.step(1)
        if len(run.contacts()[0]):
            steps_in_contact += 1
        elif steps_in_contact:
            break
    s = run.state()
    run.close()
    vrel = s["v"][1, 0] - s["v"][0, 0]
    m = sc.types[0]["density"] * 4 / 3 * math.pi * r ** 3
    mstar = m / 2
    beta = math.log(en) / math.sqrt(math.pi ** 2 + math.log(en) ** 2)
    eta = -beta * math.sqrt(kn / mstar)
    tc = math.pi / math.sqrt(kn / mstar - eta ** 2)
    # the time discretisation (dt = tc / 700) bounds both to 2e-3
    assert abs(vrel / (2 * v0) - en) < 2e-3
    assert abs(steps_in_contact * dt - tc) / tc < 2e-3


@pytest.mark.parametrize("impl", IMPLS)
def test_sliding_contact_saturates_at_coulomb(tmp_path, request, impl):
    _backend(request, impl)
    sc = scenarios.settling_box(n=1, muc=0.3, etat=None, dt=1e-6)
    r = sc.types[0]["radius"]
    m = sc.types[0]["density"] * 4 / 3 * math.pi * r ** 3
    sc.type = np.zeros(1, np.int32)
    sc.x = np.array([[0.015, 0.015, r - m * 9.81 / 1e4]])     # resting overlap m g / kn
    sc.v = np.array([[0.2, 0, 0]])
    sc.w = np.zeros((1, 3))
    sc.q = np.array([[0, 0, 0, 1.0]])
    run = _Run(impl, sc, str(sc.write_xml(tmp_path / "slide.xml")))
    run.step(200)
    id0, id1, _, f = run.contacts()
    run.close()
    assert len(id0) == 1 and id1[0] == -(4 + 2)     # the bottom wall is the 5th obstacle
    fn = abs(f[0, 2])
    ft = math.hypot(f[0, 0], f[0, 1])
    tol = 1e-5 if impl == FP32_SPLIT else 1e-9
    assert fn > 0 and abs(ft - 0.3 * fn) / (0.3 * fn) < tol


def _quat(axis, angle):
    a = np.asarray(axis, float)
    a = a / np.linalg.norm(a)
    return np.array([*(a * math.sin(angle / 2)), math.cos(angle / 2)])


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("case", ["face", "edge", "corner"])
def test_cube_cube_overlap(tmp_path, request, impl, case):
    _backend(request, impl)
    poly = scenarios.write_tetrahedron(tmp_path / "tet.poly")
    sc = scenarios.convex_pour(n=2, seed=1, poly_path=poly, box=(0.03, 0.03, 0.02))
    sc.gravity = (0.0, 0.0, 0.0)
    sc.walls = []
    sc.models = sc.models[:1]
    sc.type = np.zeros(2, np.int32)
    H = sc.types[0]["size"][0] / 2
    c = sc.types[0]["crust"]
    d = 0.3 * c
    q0 = np.array([0, 0, 0, 1.0])
    if case == "face":
        q1, dx = q0, 2 * H - d
    elif case == "edge":
        q1 = _quat((0, 0, 1), math.pi / 4)
        dx = (H - c) * (1 + math.sqrt(2)) + 2 * c - d
    else:
        q1 = _quat((0, 1, -1), math.acos(1 / math.sqrt(3)))
        dx = (H - c) * (1 + math.sqrt(3)) + 2 * c - d
        R = scenarios.rotation_matrices(q1[None])[0].reshape(3, 3)
        assert np.allclose(R @ np.ones(3) / math.sqrt(3), [1, 0, 0], atol=1e-15)
    sc.x = np.array([[0.010, 0.015, 0.010], [0.010 + dx, 0.015, 0.010]])
    sc.v = np.zeros((2, 3))
    sc.w = np.zeros((2, 3))
    sc.q = np.stack([q0, q1])
    run = _Run(impl, sc, str(sc.write_xml(tmp_path / f"{case}.xml")), basis=True)
    id0, id1, dl, f = run.contacts()
    run.close()
    assert list(id0) == [0] and list(id1) == [1]
    kn = sc.models[0]["kn"]
    # FP32-split: the pair's relative position is resolved to the FP32 ulp
    # of a 1 cm coordinate (9.3e-10 m, 1.8e-5 of d)
    tol = 1e-4 if impl == FP32_SPLIT else 1e-10
    assert abs(-dl[0] - d) <= tol * d
    assert abs(-f[0, 0] - kn * d) <= tol * kn * d
    assert np.all(np.abs(f[0, 1:]) <= tol * kn * d)
