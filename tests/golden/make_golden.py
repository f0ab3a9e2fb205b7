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
        out = {"xml": np.array(sc.xml()), "particles": np.array(pfile.read_text()),
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


def main():
    import subprocess
    if not reference.available():
        reference.build()
    for name in SCENARIOS:
        subprocess.run([sys.executable, __file__, name], check=True)
    subprocess.run([sys.executable, __file__, "reload"], check=True)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        run_reload() if sys.argv[1] == "reload" else run(sys.argv[1])
    else:
        main()
