"""Generates the golden vectors in this directory by running the Grains3D
reference itself (oracle/_ref/libgrains_ref.so, built by oracle/build_ref.sh
from the unmodified reference sources).

    python tests/golden/make_golden.py

Each fixture holds the scenario parameters, the initial state, and the
reference's state, cells and contact memory at a few step counts.  The
"settling_box" fixture records consecutive snapshots (k, k+1) so that a
single step can be checked from the reference's own state.
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


SCENARIOS = {
    "settling_box": (lambda: scenarios.settling_box(n=500, seed=11), [0, 1, 800, 801, 1600, 1601]),
    "periodic_gas": (lambda: scenarios.periodic_gas(n_fcc=5, seed=12), [0, 1, 20, 21]),
}


def snapshot(r, prefix, out):
    s = r.state()
    for k, v in s.items():
        out[f"{prefix}_{k}"] = v
    out[f"{prefix}_cells"] = r.cells()
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
            assert _quiet(r.init) == 0
            out = {"xml": np.array(sc.xml()), "type": sc.type, "x0": sc.x, "v0": sc.v,
                   "w0": sc.w, "q0": sc.q, "marks": np.array(marks)}
            # the CPU restatement runs alongside only to record, per particle,
            # the sum of its contact-force magnitudes (the error normaliser)
            from oracle.oracle import Oracle
            from tests.helpers import contact_scale
            o = Oracle(xml)
            o.set_particles(sc.type, sc.x, sc.v, sc.w, sc.q)
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


def main():
    import subprocess
    if not reference.available():
        reference.build()
    for name in SCENARIOS:
        subprocess.run([sys.executable, __file__, name], check=True)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        run(sys.argv[1])
    else:
        main()
