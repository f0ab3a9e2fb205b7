"""Parity of the CUDA DEM step against the CPU FP64 restatement (oracle/).

Tolerances (stated per the DEM step's accuracy targets):
  * FP64 mode: cell indices and contact-pair sets equal exactly; per-particle
    force and torque within 1e-10 of the particle's sum of contact-force
    magnitudes (|dF_i| / sum_c |f_ic|); positions after one step equal to
    1e-15 relative.
  * FP32-split mode: per-particle force error within 1e-5 of the same
    normaliser and per-contact force error within 1e-5 of the contact's
    force; cell indices and contact sets equal exactly (the narrow phase runs
    on the FP64 positions in both modes).
"""
import numpy as np
import pytest

from pacific_b200 import FP32_SPLIT, FP64, Grains, scenarios
from oracle.oracle import Oracle
from tests.helpers import (contact_forces, contact_scale, contact_set, force_errors, gpu_from_oracle,
                           oracle_for, per_contact_errors, radii_of)

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-5


def _cases():
    return {
        "settling_box": (scenarios.settling_box(), [0, 1500, 3000]),
        "periodic_gas": (scenarios.periodic_gas(n_fcc=6), [0, 100, 300]),
        "periodic_dense": (scenarios.periodic_gas(n_fcc=8, seed=77, spacing=2.35e-3), [0, 200]),
    }


@pytest.fixture(scope="module")
def cases(tmp_path_factory, lib, oracle_lib):
    d = tmp_path_factory.mktemp("xml")
    out = {}
    for name, (sc, marks) in _cases().items():
        p = sc.write_xml(d / f"{name}.xml")
        out[name] = (sc, str(p), marks)
    return out


def _check_step(sc, xml, o, precision, tol):
    """Both sides advance one step from the oracle's current state."""
    g = gpu_from_oracle(xml, sc, o, precision)
    g.set_diagnostics(True)
    assert o.step(1) == 0
    g.step(1)
    os_, gs = o.state(), g.download_state()
    id0, id1, dl, pt, f = o.contacts()
    scale = contact_scale(sc.n, id0, id1, f)
    fe, te = force_errors(os_, gs, scale, radii_of(sc))
    oc = contact_set(id0, id1)
    g0, g1, gdl, gf = g.download_contacts(forces=True)
    gc = contact_set(g0, g1)
    # both modes decide contacts on the FP64 positions: identical contact sets
    assert oc == gc
    assert np.array_equal(o.cells(), g.download_cells())
    if precision == FP64:
        assert np.max(np.abs(os_["x"] - gs["x"])) <= 1e-15 * np.max(np.abs(os_["x"]))
    # per contact: |df| / |f_ref|
    pe = per_contact_errors(contact_forces(id0, id1, f), contact_forces(g0, g1, gf))
    assert pe.max(initial=0) <= tol, f"per-contact force error {pe.max():.3e}"
    assert fe.max() <= tol, f"force error {fe.max():.3e}"
    assert te.max() <= tol * 10, f"torque error {te.max():.3e}"
    assert g.status() == 0
    g.close()
    return fe.max(), te.max(), len(oc)


@pytest.mark.parametrize("name", ["settling_box", "periodic_gas", "periodic_dense"])
def test_init_forces_fp64(cases, name):
    sc, xml, _ = cases[name]
    o = oracle_for(sc, xml)
    assert o.init() == 0
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.set_diagnostics(True)
    g.do_before_time_stepping()
    assert np.array_equal(o.cells(), g.download_cells())
    id0, id1, dl, pt, f = o.contacts()
    g0, g1, _ = g.download_contacts()
    assert contact_set(id0, id1) == contact_set(g0, g1)
    scale = contact_scale(sc.n, id0, id1, f)
    fe, te = force_errors(o.state(), g.download_state(), scale, radii_of(sc))
    assert fe.max() <= FP64_TOL and te.max() <= FP64_TOL


@pytest.mark.parametrize("precision,tol", [(FP64, FP64_TOL), (FP32_SPLIT, FP32_TOL)],
                         ids=["fp64", "fp32split"])
@pytest.mark.parametrize("name", ["settling_box", "periodic_gas", "periodic_dense"])
def test_one_step_from_oracle_state(cases, name, precision, tol):
    sc, xml, marks = cases[name]
    o = oracle_for(sc, xml)
    assert o.init() == 0
    done = 0
    ncontacts = 0
    for m in marks:
        assert o.step(m - done) == 0
        done = m
        fe, te, nc = _check_step(sc, xml, o, precision, tol)
        done += 1
        ncontacts += nc
    assert ncontacts > 0


@pytest.mark.parametrize("name", ["settling_box", "periodic_gas"])
def test_trajectory_fp64(cases, name):
    """100 steps from the same start: FP64 trajectories stay together."""
    sc, xml, _ = cases[name]
    o = oracle_for(sc, xml)
    o.init()
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    for _ in range(4):
        o.step(25)
        g.step(25)
    os_, gs = o.state(), g.download_state()
    assert np.max(np.abs(os_["x"] - gs["x"])) < 1e-12
    assert np.max(np.abs(os_["v"] - gs["v"])) < 1e-9
    assert np.array_equal(o.cells(), g.download_cells())


@pytest.mark.parametrize("precision", [FP64, FP32_SPLIT], ids=["fp64", "fp32split"])
def test_deterministic_and_graphs(cases, precision):
    """Two runs give identical bytes; graph replay equals plain launches."""
    sc, xml, _ = cases["periodic_dense"]
    res = []
    for graphs in (True, True, False):
        g = Grains(xml, precision)
        g.use_graphs(graphs)
        g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
        g.do_before_time_stepping()
        g.step(37)
        g.step(20)
        res.append(g.download_state())
        g.close()
    for k in ("x", "v", "w", "q", "F", "T"):
        assert np.array_equal(res[0][k], res[1][k])
        assert np.array_equal(res[0][k], res[2][k])


def test_error_status(cases):
    sc, xml, _ = cases["settling_box"]
    # MotionError: one particle moving faster than crust / dt
    v = sc.v.copy()
    v[5] = [50.0, 0.0, 0.0]
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, v, sc.w, sc.q)
    g.do_before_time_stepping()
    g.step(1)
    assert g.status() & 0x02
    # ContactError: two spheres overlapping by more than both crusts
    x = sc.x.copy()
    x[1] = x[0] + np.array([1.5e-3, 0.0, 0.0])
    g = Grains(xml, FP64)
    g.upload_state(sc.type, x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    assert g.status() & 0x01
    # SimulationError: a particle outside the linked-cell grid
    x = sc.x.copy()
    x[3] = [0.5, 0.5, 0.5]
    g = Grains(xml, FP32_SPLIT)
    g.upload_state(sc.type, x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    assert g.status() & 0x04


def test_batched_instances_equal_separate_runs(tmp_path, lib, oracle_lib):
    """Instances stepped together in one batch give the same bytes as each
    instance stepped alone, and each matches the oracle."""
    inst = scenarios.batched_boxes(n_inst=3, nmin=200, nmax=600, seed=99)
    xmls = [str(s.write_xml(tmp_path / f"i{k}.xml")) for k, s in enumerate(inst)]
    ins, typ, x, v, w, q = scenarios.concat_state(inst)
    for prec in (FP64, FP32_SPLIT):
        gb = Grains(xmls, prec)
        gb.upload_state(typ, x, v, w, q, inst=ins)
        gb.do_before_time_stepping()
        gb.step(60)
        sb = gb.download_state()
        assert gb.status() == 0
        base = 0
        for k, sc in enumerate(inst):
            g = Grains(xmls[k], prec)
            g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
            g.do_before_time_stepping()
            g.step(60)
            s = g.download_state()
            for key in ("x", "v", "w", "q", "F", "T"):
                assert np.array_equal(s[key], sb[key][base:base + sc.n]), (k, key)
            if prec == FP64:
                o = oracle_for(sc, xmls[k])
                o.init()
                o.step(60)
                assert np.max(np.abs(o.state()["x"] - s["x"])) < 1e-12
            base += sc.n


@pytest.mark.parametrize("precision", [FP64, FP32_SPLIT], ids=["fp64", "fp32split"])
def test_convex_trajectory(tmp_path, lib, oracle_lib, precision):
    """Cubes and tetrahedra (GJK narrow phase, 3D rotational dynamics) in a
    box, launched at up to 1 m/s: 1000 steps from the same start on the
    oracle and the GPU, with collisions throughout.  FP64 positions stay
    within 1e-11 m, FP32-split within 1e-8 m (its FP32 force law perturbs
    each contact force by about 1e-5 of its size)."""
    poly = scenarios.write_tetrahedron(tmp_path / "tet.poly")
    sc = scenarios.convex_pour(n=400, seed=21, poly_path=poly, box=(0.03, 0.03, 0.02), vmax=1.0)
    xml = str(sc.write_xml(tmp_path / "convex.xml"))
    basis = scenarios.rotation_matrices(sc.q)
    o = Oracle(xml)
    assert o.set_particles(sc.type, sc.x, sc.v, sc.w, sc.q, basis) == 0
    assert o.init() == 0
    g = Grains(xml, precision)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    assert np.array_equal(g.download_basis(), basis)
    g.do_before_time_stepping()
    ncontact = 0
    for _ in range(10):
        assert o.step(100) == 0
        g.step(100)
        ncontact += len(o.contacts()[0])
    os_, gs = o.state(), g.download_state()
    fp64 = precision == FP64
    assert np.max(np.abs(os_["x"] - gs["x"])) < (1e-11 if fp64 else 1e-8)
    assert np.max(np.abs(o.basis() - g.download_basis())) < (1e-8 if fp64 else 1e-5)
    assert g.status() == 0
    assert ncontact > 20
    g.close()


def _q_conj_w_q(q, w):
    """Body-frame image q* w q of space-frame vectors w (rows), q = (x, y, z, w)."""
    qv, qw = q[:, :3], q[:, 3:4]
    # rotate by the inverse quaternion: w' = w + 2 qw (w x -qv) + 2 (-qv) x ((-qv) x w) ... written
    # as the sandwich conj(q) (0, w) q
    t = 2.0 * np.cross(-qv, w)
    return w + qw * t + np.cross(-qv, t)


def test_fp32split_sphere_angular_state(tmp_path, lib):
    """FP32-split spheres integrate the space-frame angular velocity (the
    body-frame one is derived as q* w q on output): it tracks the FP64 mode,
    which integrates the body-frame one, and the derived w_bf is q* w q."""
    sc = scenarios.periodic_gas(n_fcc=6, seed=31, spacing=3.0e-3)
    rng = np.random.default_rng(4)
    w0 = rng.normal(0.0, 200.0, (sc.n, 3))
    xml = str(sc.write_xml(tmp_path / "spin.xml"))
    out = {}
    for prec in (FP64, FP32_SPLIT):
        g = Grains(xml, prec)
        g.upload_state(sc.type, sc.x, sc.v, w0, sc.q)
        g.do_before_time_stepping()
        g.step(200)
        out[prec] = g.download_state()
        assert g.status() == 0
        g.close()
    a, b = out[FP64], out[FP32_SPLIT]
    scale = np.abs(a["w"]).max()
    assert np.max(np.abs(a["w"] - b["w"])) <= 1e-6 * scale
    assert np.max(np.abs(a["q"] - b["q"])) <= 1e-9
    assert np.max(np.abs(b["wbf"] - _q_conj_w_q(b["q"], b["w"]))) <= 1e-12 * scale
    assert np.max(np.abs(a["wbf"] - b["wbf"])) <= 1e-6 * scale
