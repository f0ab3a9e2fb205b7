"""Generates the golden vectors in this directory by running the Grains3D
reference itself (oracle/_ref/libgrains_ref.so, built by oracle/build_ref.sh
from the unmodified reference sources).

    python tests/golden/make_golden.py

Each fixture holds the scenario parameters, the initial state, and the
reference's state, cells and contact memory at a few step counts.  The
"settling_box" fixture records consecutive snapshots (k, k+1) so that a
single step can be checked from the reference's own state.  The
"reload_settling" fixture holds a Format2024 reload particle file written by
the reference itself and the reference's state after it.
"""
from __future__ import annotations

import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import reference  # noqa: E402
from pacific_b200 import scenarios  # noqa: E402


def _quiet(f, *a):
    sys.stdout.flush()
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        return f(*a)
    finally:
        os.dup2(fd, 1)
        os.close(fd)
        os.close(nul)


POLY_TOKEN = "@POLYHEDRON_FILE@"


def _convex(cylinders=False, seed=5, vmax=0.2):
    d = Path(tempfile.mkdtemp())
    poly = scenarios.write_tetrahedron(d / "tet.poly")
    return scenarios.convex_pour(n=400, seed=seed, poly_path=poly, box=(0.03, 0.03, 0.02),
                                 vmax=vmax, cylinders=cylinders)


SCENARIOS = {
    "settling_box": (lambda: scenarios.settling_box(n=500, seed=11), [0, 1, 800, 801, 1600, 1601]),
    "periodic_gas": (lambda: scenarios.periodic_gas(n_fcc=5, seed=12), [0, 1, 20, 21]),
    "convex_pour": (_convex, [0, 1, 3000, 3001, 6000, 6001]),
    # cubes, tetrahedra and cylinders (GJK with the cylinder support function)
    "convex_cylinders": (lambda: _convex(cylinders=True, seed=6, vmax=1.0),
                         [0, 1, 3000, 3001, 6000, 6001]),
    # Hooke law (no tangential memory) with a rolling-resistance moment
    "settling_hooke": (lambda: scenarios.settling_box(n=500, seed=17, etat=None, law="Hooke",
                                                      kr=0.05, vmax=0.2),
                       [0, 1, 800, 801, 1600, 1601]),
}


def snapshot(r, prefix, out):
    s = r.state()
    for k, v in s.items():
        out[f"{prefix}_{k}"] = v
    out[f"{prefix}_cells"] = r.cells()
    out[f"{prefix}_basis"] = r.basis()
    own, par, kd, pn, sp = r.history()
    out[f"{prefix}_hist_owner"] = own
    out[f"{prefix}_hist_partner"] = par
    out[f"{prefix}_hist_kdelta"] = kd
    out[f"{prefix}_hist_prevn"] = pn


def run(name):
    """One scenario per process: the reference keeps its configuration in
    static members (ContactBuilderFactory, App, GrainsExec), so a process
    hosts a single Grains object, as the grains executable does."""
    make, marks = SCENARIOS[name]
    if True:
        sc = make()
        with tempfile.TemporaryDirectory() as d:
            xml = sc.write_xml(Path(d) / f"{name}.xml")
            r = _quiet(reference.Reference, xml)
            assert _quiet(r.set_particles, sc.type, sc.x, sc.v, sc.w, sc.q) == 0
            # initial state as the reference holds it after insertion (its
            # quaternion is rebuilt from the rotated basis)
            s0 = r.state()
            b0 = r.basis()
            assert _quiet(r.init) == 0
            text = sc.xml()
            polys = [t["file"] for t in sc.types if t.get("shape") == "polyhedron"]
            if polys:
                out_poly = Path(polys[0]).read_text()
                text = text.replace(polys[0], POLY_TOKEN)
            out = {"xml": np.array(text), "type": sc.type, "x0": s0["x"], "v0": s0["v"],
                   "w0": s0["w"], "q0": s0["q"], "basis0": b0, "marks": np.array(marks)}
            if polys:
                out["poly"] = np.array(out_poly)
            # the CPU restatement runs alongside only to record, per particle,
            # the sum of its contact-force magnitudes (the error normaliser)
            from oracle.oracle import Oracle
            from tests.helpers import contact_scale
            o = Oracle(xml)
            o.set_particles(sc.type, s0["x"], s0["v"], s0["w"], s0["q"], b0)
            o.init()
            done = 0
            for m in marks:
                assert _quiet(r.step, m - done) == 0
                o.step(m - done)
                done = m
                snapshot(r, f"s{m}", out)
                id0, id1, dl, pt, f = o.contacts()
                out[f"s{m}_scale"] = contact_scale(len(sc.type), id0, id1, f)
                # each particle's polyhedron support vertex (Polyhedron::
                # m_curr_vertex): hidden state of the reference, taken from the
                # restatement, which reproduces the reference bit for bit
                # (the periodic gas's restatement agrees to round-off only,
                # minimum image against clones: it records neither)
                st = o.state()
                if name != "periodic_gas":
                    assert np.array_equal(st["x"], out[f"s{m}_x"])
                    out[f"s{m}_curv"] = o.support_vertices()
                    # the body-frame angular velocity, which the reference
                    # integrates (ParticleKinematics::m_angularVelocity_bf, no
                    # accessor): taken from the restatement too, whose
                    # space-frame angular velocity and quaternion equal the
                    # reference's to the bit
                    assert np.array_equal(st["w"], out[f"s{m}_w"])
                    assert np.array_equal(st["q"], out[f"s{m}_q"])
                    out[f"s{m}_wbf"] = st["wbf"]
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"wrote {name}.npz ({len(sc.type)} particles, steps {marks})")


def run_reload():
    """The reload fixture: 200 spheres settling in the walled box, stepped
    600 times by the reference, which then writes the particle file of a
    Format2024 reload with its own Particle::write2014; then the reference's
    state after 1 and 50 more steps."""
    sc = scenarios.settling_box(n=200, seed=23)
    with tempfile.TemporaryDirectory() as d:
        xml = sc.write_xml(Path(d) / "reload.xml")
        r = _quiet(reference.Reference, xml)
        assert _quiet(r.set_particles, sc.type, sc.x, sc.v, sc.w, sc.q) == 0
        assert _quiet(r.init) == 0
        assert _quiet(r.step, 600) == 0
        pfile = Path(d) / "reload_Particles"
        assert r.write_particles(pfile) == 0
        bfile = Path(d) / "reload_Particles.bin"
        assert r.write_particles_hybrid(bfile) == 0
        out = {"xml": np.array(sc.xml()), "particles": np.array(pfile.read_text()),
               "particles_hybrid": np.frombuffer(bfile.read_bytes(), np.uint8),
               "marks": np.array([1, 50])}
        from oracle.oracle import Oracle
        from tests.helpers import contact_scale
        done = 0
        for m in (1, 50):
            assert _quiet(r.step, m - done) == 0
            done = m
            snapshot(r, f"s{m}", out)
            # the error normaliser (each particle's sum of contact-force
            # magnitudes) from the CPU restatement at the reference's state
            st = r.state()
            o = Oracle(xml)
            o.set_particles(sc.type, st["x"], st["v"], st["w"], st["q"], r.basis())
            o.init()
            id0, id1, dl, pt, f = o.contacts()
            out[f"s{m}_scale"] = contact_scale(len(sc.type), id0, id1, f)
    np.savez_compressed(HERE / "reload_settling.npz", **out)
    print("wrote reload_settling.npz (200 particles, particle file after 600 steps)")


RAW_SUFFIXES = ("position_x", "position_y", "position_z", "translational_velocity_x",
                "translational_velocity_y", "translational_velocity_z", "angular_velocity_x",
                "angular_velocity_y", "angular_velocity_z", "coordinationNumber", "particleType")
RAW_SETTLE = 6000
RAW_MARKS = (0, 10, 100)


def run_rawdata(mode):
    """The RawData fixtures: 200 spheres settling in the walled box, stepped
    6,000 times by the reference, which writes the particle file of a
    Format2024 reload there; then the reference's own
    RawDataPostProcessingWriter (text or binary) is started at that time and
    written after 10 and 100 more steps, with the reference's velocity
    max/mean (the _VelocityMaxMean.dat figures) at each output time.  A run
    reloaded from the file starts its writer before any force evaluation,
    so its first coordination numbers are zero; the ones stored here for
    that time are the reference's from step 6,000."""
    binary = mode == "binary"
    sc = scenarios.settling_box(n=200, seed=29)
    dt = 1e-5
    out = {"xml": np.array(sc.xml()), "marks": np.array(RAW_MARKS)}
    with tempfile.TemporaryDirectory() as d:
        xml = sc.write_xml(Path(d) / "raw.xml")
        root = Path(d) / "res"
        r = _quiet(reference.Reference, xml)
        assert _quiet(r.set_particles, sc.type, sc.x, sc.v, sc.w, sc.q) == 0
        assert _quiet(r.init) == 0
        assert _quiet(r.step, RAW_SETTLE) == 0
        pfile = Path(d) / "raw_Particles"
        assert r.write_particles(pfile) == 0
        if not binary:      # the same file for both modes: kept once
            out["particles"] = np.array(pfile.read_text())
        times, vstats, done = [], [], 0
        for m in RAW_MARKS:
            t = (RAW_SETTLE + m) * dt
            if m == 0:
                assert _quiet(r.rawdata_start, root, binary, t) == 0
            else:
                assert _quiet(r.step, m - done) == 0
                done = m
                assert _quiet(r.rawdata_write, t) == 0
            times.append(t)
            vstats.append(r.velocity_max_mean())
        _quiet(r.rawdata_end)
        for name in RAW_SUFFIXES:
            data = (Path(d) / f"res_{name}.dat").read_bytes()
            out[name] = np.frombuffer(data, np.uint8) if binary else np.array(data.decode())
        out["times"] = np.array(times)
        out["velocity_max_mean"] = np.array(vstats)
    np.savez_compressed(HERE / f"rawdata_settling_{mode}.npz", **out)
    print(f"wrote rawdata_settling_{mode}.npz (RawData files of the reference, {mode})")


FEATURE_MARKS = (0, 400, 1200)


def run_features():
    """The contact-features fixture: 300 spheres settling in the walled box
    from their inserted state, with the reference's own contact features
    (AppCollision: largest and mean overlap over all contacts of all
    evaluations so far, time of the largest, mean GJK iterations) after the
    leapfrog start and after 400 and 1,200 steps."""
    sc = scenarios.settling_box(n=300, seed=41)
    out = {"xml": np.array(sc.xml()), "type": sc.type, "marks": np.array(FEATURE_MARKS)}
    with tempfile.TemporaryDirectory() as d:
        xml = sc.write_xml(Path(d) / "features.xml")
        r = _quiet(reference.Reference, xml)
        assert _quiet(r.set_particles, sc.type, sc.x, sc.v, sc.w, sc.q) == 0
        s0 = r.state()
        for k in ("x", "v", "w", "q"):
            out[f"{k}0"] = s0[k]
        assert _quiet(r.init) == 0
        done = 0
        for m in FEATURE_MARKS:
            assert _quiet(r.step, m - done) == 0
            done = m
            out[f"s{m}_features"] = r.contact_features()
            out[f"s{m}_x"] = r.state()["x"]
    np.savez_compressed(HERE / "contact_features.npz", **out)
    print("wrote contact_features.npz (300 particles, features at steps", FEATURE_MARKS, ")")


def main():
    import subprocess
    if not reference.available():
        reference.build()
    for name in SCENARIOS:
        subprocess.run([sys.executable, __file__, name], check=True)
    subprocess.run([sys.executable, __file__, "reload"], check=True)
    for mode in ("text", "binary"):
        subprocess.run([sys.executable, __file__, "rawdata", mode], check=True)
    subprocess.run([sys.executable, __file__, "features"], check=True)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        if sys.argv[1] == "reload":
            run_reload()
        elif sys.argv[1] == "rawdata":
            run_rawdata(sys.argv[2])
        elif sys.argv[1] == "features":
            run_features()
        else:
            run(sys.argv[1])
    else:
        main()
