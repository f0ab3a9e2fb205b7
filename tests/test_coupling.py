"""Fluid coupling: gdem_set_fluid / set_time_step / set_velocities /
set_hydro_forces and the Basilisk C ABI of libgrains_b200_basilisk.so
(InterfaceGrains3DBasilisk.h: Init_Grains, Simu_Grains, GrainsToBasilisk,
UpdateVelocityGrains, NumberOfRigidBodiesInBasilisk, ...).

* Buoyancy and the coupling factor: a free sphere in a fluid of density
  rho_f falls at g (1 - rho_f / rho) without the corrected acceleration and
  at g with it (the reference divides the buoyant weight by m c,
  c = 1 - rho_f / rho).
* Simu_Grains(dt_fluid) sub-steps as GrainsCoupledWithFluid::Simulation:
  the same state as gdem_step with dt = dt_fluid / ndt, byte for byte, with
  the coupled step's contact memory (ended contacts kept) and the
  reference's coupling factor of 1 for reloaded particles.
* Against the reference's own Basilisk interface on the same reload: the
  GrainsToBasilisk streams after two fluid steps, around an
  UpdateVelocityGrains, to FP64 round-off.
* GrainsToBasilisk writes the GrainsToFluid stream of the state: count,
  then per sphere its ID - 1, velocities, density, mass, space-fixed inertia,
  orientation, centre, radius and envelope point.
* UpdateVelocityGrains and hydrodynamic forces act on the next step.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from pacific_b200 import FP64, Grains, scenarios

pytestmark = pytest.mark.gpu

BASILISK = Path(__file__).resolve().parent.parent / "pacific_b200" / "libgrains_b200_basilisk.so"


def _coupled_xml(sc, reload_name, mindt=1e-5, maxdt=2e-5, ndt=4):
    text = sc.xml()
    text = text.replace('<TimeStep dt="1e-05"/>',
                        f'<TimeStep mindt="{mindt}" maxdt="{maxdt}" ndt="{ndt}"/>')
    text = text.replace("  </Construction>",
                        f'    <Reload Type="new" Filename="{reload_name}"/>\n  </Construction>')
    return text


def _free_sphere(tmp_path):
    sc = scenarios.settling_box(n=1, seed=3, vmax=0.0)
    sc.x[:] = [0.015, 0.015, 0.03]
    return sc, str(sc.write_xml(tmp_path / "one.xml"))


@pytest.mark.parametrize("corrected", [0, 1])
def test_buoyant_free_fall(tmp_path, lib, corrected):
    sc, xml = _free_sphere(tmp_path)
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.set_fluid(1000.0, corrected)
    g.do_before_time_stepping()
    g.step(100)
    s = g.download_state()
    t = 100 * 1e-5
    a = 9.81 * (1.0 if corrected else 1.0 - 1000.0 / 2500.0)
    assert abs(s["v"][0, 2] + a * t) <= 1e-12
    g.close()


def _settled(tmp_path, n=200, steps=300):
    sc = scenarios.settling_box(n=n, seed=31)
    g = Grains(str(sc.write_xml(tmp_path / "plain.xml")), FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    g.step(steps)
    g.write_reload_particles(tmp_path / "res_Particles.result")
    g.close()
    (tmp_path / "coupled.xml").write_text(_coupled_xml(sc, str(tmp_path / "res.resA")))
    return sc


def _basilisk():
    b = ctypes.CDLL(str(BASILISK))
    b.Init_Grains.argtypes = [ctypes.c_char_p, ctypes.c_double, ctypes.c_bool, ctypes.c_bool]
    b.Simu_Grains.argtypes = [ctypes.c_double]
    b.GrainsToBasilisk.argtypes = [ctypes.POINTER(ctypes.c_int)]
    b.GrainsToBasilisk.restype = ctypes.c_void_p
    b.UpdateVelocityGrains.argtypes = [ctypes.POINTER(ctypes.POINTER(ctypes.c_double)), ctypes.c_int]
    b.NumberOfRigidBodiesInBasilisk.argtypes = [ctypes.POINTER(ctypes.c_size_t)] * 2
    return b


def test_basilisk_abi(tmp_path, lib):
    sc = _settled(tmp_path)
    b = _basilisk()
    b.Init_Grains(str(tmp_path / "coupled.xml").encode(), 1000.0, False, True)
    npart, nobs = ctypes.c_size_t(0), ctypes.c_size_t(0)
    b.NumberOfRigidBodiesInBasilisk(ctypes.byref(npart), ctypes.byref(nobs))
    assert npart.value == sc.n and nobs.value == 0
    # a reference run through the plain ABI: same file, same fluid, ndt = 4
    # sub-steps of dt_fluid / 4 (dt_fluid / ndt = 1e-5 lies in [mindt, maxdt])
    ref = Grains(str(tmp_path / "coupled.xml"), FP64)
    # as Init_Grains: the coupled step keeps ended contacts' memory, and the
    # reloaded particles get the buoyant weight with a coupling factor of 1
    # (the reference's), whatever the corrected-acceleration flag
    ref.set_contact_memory_pruning(False)
    ref.read_reload_particles(tmp_path / "res_Particles.result")
    ref.set_fluid(1000.0, False)
    ref.set_time_step(4e-5 / 4)
    b.Simu_Grains(4e-5)
    ref.step(4)
    size = ctypes.c_int(0)
    ptr = b.GrainsToBasilisk(ctypes.byref(size))
    text = ctypes.string_at(ptr).decode()
    tok = text.split()
    s = ref.download_state()
    assert int(tok[0]) == sc.n
    # per sphere: id ncorners, P v(3) w(3) density mass inertia(6) basis(9)
    # centre(3), radius npoints, point(3), nfaces
    k = 1
    for i in range(sc.n):
        assert int(tok[k]) == i and int(tok[k + 1]) == 1 and tok[k + 2] == "P"
        vals = np.array(tok[k + 3:k + 3 + 26], dtype=float)
        assert np.array_equal(vals[0:3], s["v"][i]) and np.array_equal(vals[3:6], s["w"][i])
        assert vals[6] == 2500.0
        assert np.array_equal(vals[23:26], s["x"][i])
        k += 3 + 26
        assert float(tok[k]) == 0.001 and int(tok[k + 1]) == 1
        assert np.array_equal(np.array(tok[k + 2:k + 5], dtype=float), s["x"][i])
        assert tok[k + 5] == "0"
        k += 6
    assert k == len(tok)
    # velocities from the fluid act on the next sub-steps
    rows = np.zeros((sc.n, 6))
    rows[:, 2] = -0.05
    arr = (ctypes.POINTER(ctypes.c_double) * sc.n)(
        *[rows[i].ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for i in range(sc.n)])
    b.UpdateVelocityGrains(arr, sc.n)
    ref.set_velocities(rows[:, :3], rows[:, 3:])
    b.Simu_Grains(4e-5)
    ref.step(4)
    ptr = b.GrainsToBasilisk(ctypes.byref(size))
    tok = ctypes.string_at(ptr).decode().split()
    s = ref.download_state()
    for i in range(sc.n):
        k = 1 + i * 35
        assert np.array_equal(np.array(tok[k + 3:k + 6], dtype=float), s["v"][i])
    ref.close()


def test_hydro_forces(tmp_path, lib):
    sc, xml = _free_sphere(tmp_path)
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    m = 2500.0 * 4.0 / 3.0 * np.pi * 1e-9
    F = np.array([[0.0, 0.0, m * 9.81]])   # cancels gravity
    T = np.zeros((1, 3))
    g.set_hydro_forces(F, T)
    g.step(50)
    s = g.download_state()
    assert abs(s["v"][0, 2]) <= 1e-12
    g.close()


def test_basilisk_rawdata_output(tmp_path, lib):
    """SaveResults_Grains with a RawData writer in the XML: the first call
    starts the writer (GrainsCoupledWithFluid::InitialPostProcessing), later
    ones add an output time (doPostProcessing); Simu_Grains records the last
    sub-step's contacts, so the coordination numbers written are those of
    the plain ABI stepped the same way with diagnostics on."""
    sc = _settled(tmp_path)
    raw = tmp_path / "out"
    text = (tmp_path / "coupled.xml").read_text().replace(
        "  </Simulation>",
        f'    <PostProcessing>\n      <Writers>\n        <RawData Name="{raw}" WritingMode="Text"/>\n'
        "      </Writers>\n    </PostProcessing>\n  </Simulation>")
    (tmp_path / "coupled_raw.xml").write_text(text)
    b = _basilisk()
    b.SetInitialTime.argtypes = [ctypes.c_double]
    b.Init_Grains(str(tmp_path / "coupled_raw.xml").encode(), 1000.0, False, True)
    b.SetInitialTime(0.0)
    b.SaveResults_Grains()
    b.Simu_Grains(4e-5)
    b.SaveResults_Grains()
    ref = Grains(str(tmp_path / "coupled.xml"), FP64)
    # as Init_Grains: the coupled step keeps ended contacts' memory, and the
    # reloaded particles get the buoyant weight with a coupling factor of 1
    # (the reference's), whatever the corrected-acceleration flag
    ref.set_contact_memory_pruning(False)
    ref.read_reload_particles(tmp_path / "res_Particles.result")
    ref.set_fluid(1000.0, False)
    ref.set_time_step(1e-5)
    ref.step(3)
    ref.set_diagnostics(True)
    ref.step(1)
    s = ref.download_state()
    coord = ref.download_coordination()
    ref.close()
    lines = (tmp_path / "out_position_x.dat").read_text().splitlines()
    assert len(lines) == 2
    tok = lines[1].split()
    assert float(tok[0]) == 4e-5
    assert np.array_equal(np.array(tok[1:], dtype=float), np.array([float(f"{x:.6e}") for x in s["x"][:, 0]]))
    c = (tmp_path / "out_coordinationNumber.dat").read_text().splitlines()
    assert c[0].split() == ["0"] * sc.n
    assert np.array_equal(np.array(c[1].split(), dtype=int), coord) and coord.sum() > 0


def test_basilisk_hybrid_reload(tmp_path, lib):
    """Init_Grains reads the reload's reading mode (the word after its
    "NbFiles" line, AllComponents::read) and, for "Hybrid", the binary
    particle file <stem>_Particles.result.bin: the state it starts from is the one
    of the same reload written as text, token for token in the stream, and
    the IDs and classes come from the loaded file."""
    sc = _settled(tmp_path)
    g = Grains(str(tmp_path / "coupled.xml"), FP64)
    g.read_reload_particles(tmp_path / "res_Particles.result")
    g.write_reload_particles_hybrid(tmp_path / "resH_Particles.result.bin")
    g.close()
    # the reload header: the reload name with ".result" appended
    (tmp_path / "resH.resA.result").write_text(f"NbFiles 1\nHybrid {sc.n}\n")
    (tmp_path / "coupledH.xml").write_text(
        (tmp_path / "coupled.xml").read_text().replace(str(tmp_path / "res.resA"),
                                                       str(tmp_path / "resH.resA")))
    b = _basilisk()
    size = ctypes.c_int(0)
    streams = []
    for xml in ("coupled.xml", "coupledH.xml"):
        b.Init_Grains(str(tmp_path / xml).encode(), 1000.0, False, True)
        npart, nobs = ctypes.c_size_t(0), ctypes.c_size_t(0)
        b.NumberOfRigidBodiesInBasilisk(ctypes.byref(npart), ctypes.byref(nobs))
        assert npart.value == sc.n
        b.Simu_Grains(4e-5)
        streams.append(ctypes.string_at(b.GrainsToBasilisk(ctypes.byref(size))).decode())
    assert streams[0] == streams[1]
    assert int(streams[0].split()[0]) == sc.n


REF_EXE = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "grains_b200"
REF_BASILISK = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libgrains_ref_basilisk.so"


def _reference_parity(tmp_path, sc, settle_steps, dt, rows, dt_fluid):
    """Settles sc with the reference's serial step (Type="Standard",
    insertion at the initial time from its positions, reload written at the
    end), then drives the reference's Basilisk interface and this library's
    through the same calls on that reload: Init_Grains (fluid density 1000,
    corrected acceleration), Simu_Grains(dt_fluid) (4 sub-steps),
    GrainsToBasilisk, UpdateVelocityGrains(rows), Simu_Grains, GrainsToBasilisk.
    Returns both runs' results."""
    import os
    import re
    import subprocess

    from oracle import ref_basilisk_run

    np.savetxt(tmp_path / "positions.txt", sc.x, fmt="%.17g")
    end = settle_steps * dt
    text = re.sub(r"<TimeInterval[^>]*/>", f'<TimeInterval Start="0." End="{end!r}"/>', sc.xml())
    sim = (f'    <RestartFile Name="{tmp_path}/res" WritingMode="Text"/>\n'
           f'    <TimeSave Start="0." End="{end!r}" Every="{end!r}"/>\n'
           "    <ParticleInsertion>\n      <Mode Type=\"InitialTime\"/>\n"
           "      <Order Type=\"Ordered\"/>\n"
           "      <RandomGeneratorSeed Type=\"UserDefined\" Value=\"7\"/>\n"
           f"      <ParticlePosition>\n        <File Name=\"{tmp_path}/positions.txt\"/>\n"
           "      </ParticlePosition>\n      <InitialVelocity Mode=\"Random\">\n"
           "        <Translational Amplitude=\"0.3\"/>\n        <Angular Amplitude=\"0.\"/>\n"
           "      </InitialVelocity>\n    </ParticleInsertion>\n")
    (tmp_path / "settle.xml").write_text(text.replace("  </Simulation>", sim + "  </Simulation>"))
    r = subprocess.run([str(REF_EXE), "settle.xml"], cwd=str(tmp_path), capture_output=True,
                       text=True, timeout=900, env=dict(os.environ, GRAINS_HOME=str(tmp_path)))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    reload = (tmp_path / "res_RFTable.txt").read_text().split()[-1]
    # the reference's coupled application is built for Type="CoupledFluid"
    # (GrainsBuilderFactory::createCoupledWithFluid)
    coupled = sc.xml().replace('<Grains3D Type="Standard">', '<Grains3D Type="CoupledFluid">')
    coupled = re.sub(r'<TimeStep dt="[^"]*"/>',
                     f'<TimeStep mindt="{dt!r}" maxdt="{2 * dt!r}" ndt="4"/>', coupled)
    coupled = coupled.replace(
        "  </Construction>",
        f'    <Reload Type="new" Filename="{reload}" Velocity="Keep"/>\n  </Construction>')
    coupled = coupled.replace(
        "  </Simulation>",
        f'    <RestartFile Name="{tmp_path}/cres" WritingMode="Text"/>\n  </Simulation>')
    xml = tmp_path / "coupled.xml"
    xml.write_text(coupled)
    ref = ref_basilisk_run.run(REF_BASILISK, xml, 1000.0, dt_fluid, rows)
    ours = ref_basilisk_run.run(BASILISK, xml, 1000.0, dt_fluid, rows)
    return ref, ours


def _compare_streams(ref, ours, n, record=None):
    assert (ours["particles"], ours["obstacles"]) == (ref["particles"], ref["obstacles"]) == (n, 0)
    for k, (sa, sb) in enumerate(zip(ref["streams"], ours["streams"])):
        ta, tb = sa.split(), sb.split()
        assert len(ta) == len(tb) and int(ta[0]) == n
        if record:
            assert len(ta) == 1 + record * n
        where, num_a, num_b = [], [], []
        for i, (a, b) in enumerate(zip(ta, tb)):
            try:
                num_a.append(float(a))
                num_b.append(float(b))
                where.append(i)
            except ValueError:
                assert a == b
        fa, fb = np.array(num_a), np.array(num_b)
        # integers (counts, IDs, corner codes, face indices) and exact
        # constants compare equal; the rest to FP64 round-off
        err = np.abs(fa - fb) / np.maximum(np.abs(fa), 1e-6)
        worst = np.argsort(err)[::-1][:8]
        print(f"stream {k}: max relative token difference {err.max():.3g}; "
              f"{int((err > 1e-9).sum())} tokens above 1e-9; worst (token, ref, ours):",
              [(where[j], ta[where[j]], tb[where[j]]) for j in worst])
        assert err.max() <= 1e-9


@pytest.mark.skipif(not (REF_EXE.exists() and REF_BASILISK.exists()),
                    reason="the reference's executable and Basilisk library were not built")
def test_basilisk_matches_reference_interface(tmp_path, lib):
    """The coupling library against the reference's own Basilisk interface
    (InterfaceGrains3DBasilisk.cpp over the reference's objects) on the same
    reload: 200 spheres settled for 300 steps by the reference's serial
    step, then two fluid steps of 4 sub-steps around an UpdateVelocityGrains.
    Both streams agree token for token in their words and counts and to FP64
    round-off in their numbers; the rigid-body counts are the same."""
    sc = scenarios.settling_box(n=200, seed=31)
    rows = np.zeros((sc.n, 6))
    rows[:, 2] = -0.05
    rows[:, 3] = np.linspace(-1.0, 1.0, sc.n)
    ref, ours = _reference_parity(tmp_path, sc, 300, 1e-5, rows, 4e-5)
    _compare_streams(ref, ours, sc.n, record=35)


@pytest.mark.skipif(not (REF_EXE.exists() and REF_BASILISK.exists()),
                    reason="the reference's executable and Basilisk library were not built")
def test_basilisk_convex_matches_reference_interface(tmp_path, lib):
    """The same comparison for cubes, tetrahedra and cylinders: each record
    carries the class's corner code (666 box, the vertex count of a
    polyhedron, 777 cylinder), the envelope points through the particle's
    transform and the faces (RigidBody::writePositionInFluid)."""
    poly = scenarios.write_tetrahedron(tmp_path / "tet.poly")
    sc = scenarios.convex_pour(n=120, seed=1239, poly_path=poly, box=(0.02, 0.02, 0.06),
                               vmax=0.5, cylinders=True)
    rows = np.zeros((sc.n, 6))
    rows[:, 1] = 0.02
    rows[:, 5] = np.linspace(-2.0, 2.0, sc.n)
    ref, ours = _reference_parity(tmp_path, sc, 1000, 2e-6, rows, 8e-6)
    _compare_streams(ref, ours, sc.n)
    # every class's record is there: box and cylinder corner codes
    assert {"666", "777"} <= set(ours["streams"][0].split())


def _glancing_pair(tmp_path):
    """Two spheres that meet off-centre (a tangential spring builds up) and
    part again, with no gravity and no walls."""
    sc = scenarios.settling_box(n=2, kn=1e4, en=0.7, muc=0.5, dt=1e-6)
    sc.gravity = (0.0, 0.0, 0.0)
    sc.walls = []
    r = sc.types[0]["radius"]
    sc.type = np.zeros(2, np.int32)
    sc.x = np.array([[0.010, 0.015, 0.03], [0.010 + 2 * r + 1e-6, 0.015 + 0.5 * r, 0.03]])
    sc.v = np.array([[0.1, 0.0, 0.0], [-0.1, 0.0, 0.0]])
    sc.w = np.zeros((2, 3))
    sc.q = np.tile([0.0, 0.0, 0.0, 1.0], (2, 1))
    return sc, str(sc.write_xml(tmp_path / "pair.xml"))


def test_contact_memory_kept_without_pruning(tmp_path, lib):
    """gdem_set_contact_memory_pruning: with pruning (the plain step) the
    memory of a contact that has ended is gone at the next evaluation;
    without it (the coupled step) both views stay, with the values of the
    contact's last evaluation, and the trajectories are the same."""
    sc, xml = _glancing_pair(tmp_path)
    runs = {}
    for prune in (True, False):
        g = Grains(xml, FP64)
        g.set_contact_memory_pruning(prune)
        g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
        g.do_before_time_stepping()
        # the spheres meet after ~320 steps and part ~70 steps later
        last = None
        for _ in range(800):
            g.step(1)
            h = g.download_history()
            if len(h["owner"]):
                last = h
        runs[prune] = (g.download_history(), last, g.download_state())
        assert g.status() == 0
        g.close()
    (h_pruned, last_p, s_p), (h_kept, _, s_k) = runs[True], runs[False]
    assert last_p is not None and np.abs(last_p["kdelta"]).max() > 0
    assert len(h_pruned["owner"]) == 0
    pairs = sorted(zip(h_kept["owner"].tolist(), h_kept["partner"].tolist()))
    assert len(pairs) == 2 and pairs[0] == pairs[1][::-1] and pairs[0][0] != pairs[0][1]
    # the memory kept is the one the contact's last evaluation wrote
    for k in ("kdelta", "prevn", "spring"):
        assert np.array_equal(h_kept[k], last_p[k]), k
    for k in ("x", "v", "w"):
        assert np.array_equal(s_p[k], s_k[k]), k


def test_pruning_is_set_before_the_particles(tmp_path, lib):
    sc, xml = _glancing_pair(tmp_path)
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    with pytest.raises(Exception):
        g.set_contact_memory_pruning(False)
    g.close()
