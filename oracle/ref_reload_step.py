"""TEST INFRASTRUCTURE: the Grains3D reference (oracle/_ref, built by
oracle/build_ref.sh from the unmodified reference sources) stepped from a
Format2024 particle file, in a process of its own.

    python -m oracle.ref_reload_step <xml> <stem> <n> <steps> <out.npz>

reads <stem>_Particles.result through the reference's reload path
(AllComponents::read_particles, AllComponents::Link, checkClonesReload),
runs <steps> leapfrog steps of its serial Type="Standard" step and saves
the state (x, v, w, q, F, T by particle index, ID - 1), the cells
(Cell::GetCell), the contact memory (owner, partner, kdelta, previous normal)
and the wall-clock seconds of the load and of the steps.  The reference
keeps its configuration in static members, so each run gets its own
process; the checks in tests/ and bench.py call run() below.
"""
from __future__ import annotations

import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


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


def main(xml, stem, n, steps, out):
    sys.path.insert(0, str(ROOT))
    from oracle import reference
    r = _quiet(reference.Reference, xml)
    t0 = time.perf_counter()
    rc = _quiet(r.load_particles, stem, n)
    t_load = time.perf_counter() - t0
    if rc != 0:
        raise SystemExit(f"reference could not load {stem}_Particles.result (rc {rc})")
    t0 = time.perf_counter()
    rc = _quiet(r.step, steps)
    t_step = time.perf_counter() - t0
    s = r.state()
    own, par, kd, pn, sp = r.history()
    np.savez(out, rc=rc, load_s=t_load, step_s=t_step, cells=r.cells(), hist_owner=own,
             hist_partner=par, hist_kdelta=kd, hist_prevn=pn, **s)


def run(xml, particle_file, n, steps=1, timeout=1800):
    """Runs the reference from particle_file (any name: it is linked under
    the name the reference's reader builds) and returns its results."""
    import tempfile
    with tempfile.TemporaryDirectory(prefix="refstep") as d:
        d = Path(d)
        if "." in str(d):
            raise RuntimeError("temporary directory name holds a '.'")
        os.symlink(Path(particle_file).resolve(), d / "state_Particles.result")
        out = d / "out.npz"
        env = dict(os.environ)
        r = subprocess.run([sys.executable, "-m", "oracle.ref_reload_step", str(xml),
                            str(d / "state"), str(n), str(steps), str(out)], cwd=str(ROOT),
                           capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed: {r.stderr[-2000:]}")
        with np.load(out) as z:
            return {k: z[k] for k in z.files}


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), sys.argv[5])
