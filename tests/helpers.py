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
