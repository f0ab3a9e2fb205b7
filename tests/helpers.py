"""Shared parity metrics between the CUDA path and the CPU oracle."""
from __future__ import annotations

import numpy as np

from oracle.oracle import Oracle
from pacific_b200 import Grains


def contact_set(id0, id1):
    a = np.minimum(id0, id1)
    b = np.maximum(id0, id1)
    # walls are negative and stay as the second element
    first = np.where(id1 < 0, id0, a)
    second = np.where(id1 < 0, id1, b)
    return set(zip(first.tolist(), second.tolist()))


def contact_forces(id0, id1, f):
    """{(lower ID, higher ID) or (particle, wall): force on the first body}."""
    out = {}
    for a, b, v in zip(id0.tolist(), id1.tolist(), np.asarray(f)):
        if b >= 0 and a > b:
            out[(b, a)] = -v
        else:
            out[(a, b)] = v
    return out


def per_contact_errors(ref, got):
    """|f_got - f_ref| / |f_ref| per contact present in both dicts."""
    return np.array([np.linalg.norm(got[k] - ref[k]) / np.linalg.norm(ref[k])
                     for k in ref if k in got and np.linalg.norm(ref[k]) > 0])


def contact_scale(n, id0, id1, f):
    """Sum over each particle's contacts of |f_ic| (the per-particle error
    normaliser: |dF_i| / sum_c |f_ic|)."""
    s = np.zeros(n)
    m = np.linalg.norm(f, axis=1)
    np.add.at(s, id0, m)
    np.add.at(s, id1[id1 >= 0], m[id1 >= 0])
    return s


def force_errors(o_state, g_state, scale, radius):
    """Per-particle normalised force and torque errors."""
    eps = 1e-300
    dF = np.linalg.norm(o_state["F"] - g_state["F"], axis=1)
    dT = np.linalg.norm(o_state["T"] - g_state["T"], axis=1)
    W = np.linalg.norm(o_state["F"], axis=1)
    fe = dF / (scale + eps)
    te = dT / (radius * scale + eps)
    fe[scale == 0] = dF[scale == 0] / np.maximum(W[scale == 0], eps)
    te[scale == 0] = 0.0 if np.all(dT[scale == 0] == 0) else dT[scale == 0].max()
    return fe, te


def oracle_for(sc, xml_path):
    o = Oracle(xml_path)
    assert o.set_particles(sc.type, sc.x, sc.v, sc.w, sc.q) == 0
    return o


def gpu_from_oracle(xml_path, sc, o, precision):
    """A GPU system holding exactly the oracle's current state (positions,
    velocities, both angular velocities, quaternion, forces, torques and
    contact memory), as a Format2024 reload would."""
    s = o.state()
    g = Grains(xml_path, precision)
    g.upload_state(sc.type, s["x"], s["v"], s["w"], s["q"], wbf=s["wbf"])
    g.upload_forces(s["F"], s["T"])
    own, par, kd, pn, sp = o.history()
    g.upload_history(own, par, kd, pn, sp)
    return g


def radii_of(sc):
    return np.array([t["radius"] for t in sc.types])[sc.type]


def reference_contact_set(ref):
    """Contact set of the reference's contact memory after a step (each
    contact as (lower index, higher index) or (particle, -(k + 2)) for wall
    k); the memory holds the contacts of the last evaluation only."""
    own, par = ref["hist_owner"], ref["hist_partner"]
    return contact_set(own, par)


def periodic_contact_particles(n, id0, id1, x, period):
    """Particles with a contact across a periodic boundary (a pair whose
    centres are more than half a period apart along a periodic axis).  For
    such a pair the reference translates one partner's clone by the period
    while the minimum image here translates the other: the positions entering
    the contact differ by the rounding of x + L, about 1e-17 m, which against
    a contact's overlap (1e-9 to 1e-6 m) is a relative force difference of up
    to 1e-8 in FP64.  Returns a boolean mask."""
    out = np.zeros(n, bool)
    if period is None:
        return out
    L = np.asarray(period, float)
    m = id1 >= 0
    a, b = id0[m], id1[m]
    d = np.abs(x[b] - x[a])
    cross = np.any((L > 0) & (d > 0.5 * L), axis=1)
    out[a[cross]] = True
    out[b[cross]] = True
    return out


def step_parity(xml, particle_file, n, radius, precisions, steps=1, period=None):
    """One leapfrog step (or `steps`) from the state of a Format2024 particle
    file, by the Grains3D reference itself (oracle/_ref, in its own process,
    through its reload path) and by the GPU in each precision from the same
    file.  Per precision: whether the cells and the contact set equal the
    reference's, the per-particle force and torque errors (normaliser: the
    particle's sum of contact-force magnitudes, from the GPU FP64 contacts),
    split into the particles with a contact across a periodic boundary
    (period: the periodic translation per axis, 0 where not periodic) and the
    others, and the largest position difference.  The first precision must be
    FP64 (it gives the normaliser)."""
    from oracle import ref_reload_step
    from pacific_b200 import FP64
    assert precisions[0] == FP64
    ref = ref_reload_step.run(xml, particle_file, n, steps)
    rset = reference_contact_set(ref)
    out = {"reference": {"load_s": float(ref["load_s"]), "step_s": float(ref["step_s"]),
                         "contacts": len(rset)}}
    scale = None
    for prec in precisions:
        g = Grains(xml, prec)
        g.read_reload_particles(particle_file)
        g.set_diagnostics(True)
        g.step(steps)
        s = g.download_state()
        cells = g.download_cells()
        id0, id1, dl, f = g.download_contacts(forces=True)
        if scale is None:
            scale = contact_scale(n, id0, id1, f)
            per = periodic_contact_particles(n, id0, id1, s["x"], period)
        fe, te = force_errors(ref, s, scale, radius)
        gset = contact_set(id0, id1)
        m = scale > 0
        out[prec] = {
            "force_max_interior": float(fe[m & ~per].max(initial=0.0)),
            "torque_max_interior": float(te[m & ~per].max(initial=0.0)),
            "force_max_periodic": float(fe[m & per].max(initial=0.0)),
            "particles_periodic": int((m & per).sum()),
            "cells_equal": bool(np.array_equal(cells, ref["cells"])),
            "contacts_equal": gset == rset, "contacts": len(gset),
            "contacts_missing": len(rset - gset), "contacts_extra": len(gset - rset),
            "force_max": float(fe[m].max(initial=0.0)), "torque_max": float(te[m].max(initial=0.0)),
            "force_max_contact_free": float(fe[~m].max(initial=0.0)),
            "position_max_abs": float(np.abs(s["x"] - ref["x"]).max()),
            "particles_in_contact": int(m.sum()), "status": g.status()}
        g.close()
    return out
