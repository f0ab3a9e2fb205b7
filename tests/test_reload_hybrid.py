"""The hybrid (binary) form of the Format2024 reload particle file
(gdem_read_reload_particles_hybrid, gdem_write_reload_particles_hybrid),
against the file the Grains3D reference writes with its own
Particle::write2014_binary after the same 600 steps as the text fixture
(tests/golden/reload_settling.npz, key "particles_hybrid").

* CPU: parsed with the record layout (byte count as a size_t, then class,
  ID, tag, activity, origin, basis, transform type, v, q with its scalar
  first, omega, F, T, the contact map), the binary file holds the text
  file's values (the text prints 16 significant digits) and every record's
  byte count is 248 + 88 per contact-map entry (Particle::get_numberOfBytes).
* GPU: read and stepped once, it reproduces the reference's next state as
  the text file does (positions 1e-15, cells and contact set exact); written
  right after reading, the file is the reference's byte for byte except the
  spheres' orientation matrices (R(q) here, a composed rotation there; 1e-12).
"""
import struct
from pathlib import Path

import numpy as np
import pytest

from pacific_b200 import FP64, Grains

GOLDEN = Path(__file__).resolve().parent / "golden" / "reload_settling.npz"


def parse_hybrid(data):
    """[(ints (cls, id, tag), active, doubles (x3 B9 | v3 q4 w3 F3 T3),
    ttype, [(key triple, active, 9 doubles)])] of a hybrid particle file."""
    out, p = [], 0
    while p < len(data):
        (nb,) = struct.unpack_from("<Q", data, p)
        p += 8
        rec = data[p:p + nb]
        p += nb
        cls, pid, tag, act = struct.unpack_from("<iiiI", rec, 0)
        geo = struct.unpack_from("<12d", rec, 16)
        (ttype,) = struct.unpack_from("<I", rec, 112)
        kin = struct.unpack_from("<16d", rec, 116)
        (nm,) = struct.unpack_from("<i", rec, 244)
        entries, q = [], 248
        for _ in range(nm):
            k0, partner, k1, ea = struct.unpack_from("<iiii", rec, q)
            vals = struct.unpack_from("<9d", rec, q + 16)
            entries.append(((k0, partner, k1), ea, vals))
            q += 88
        assert q == nb == 248 + 88 * nm
        out.append(((cls, pid, tag), act, geo, ttype, kin, entries))
    return out


def test_hybrid_fixture_holds_the_text_fixture():
    g = np.load(GOLDEN)
    recs = parse_hybrid(g["particles_hybrid"].tobytes())
    lines = [ln.split() for ln in str(g["particles"]).splitlines() if ln.strip()]
    assert len(recs) == len(lines) == 200
    for (ints, act, geo, ttype, kin, entries), tok in zip(recs, lines):
        assert list(ints) == [int(t) for t in tok[0:3]] and act == int(tok[3])
        assert ttype == int(tok[16])
        text_vals = [float(t) for t in tok[4:16] + tok[17:33]]
        assert np.allclose(list(geo) + list(kin), text_vals, rtol=1e-15, atol=1e-300)
        nm = int(tok[33])
        assert nm == len(entries)
        k = 34
        for key, ea, vals in entries:
            assert list(key) + [ea] == [int(t) for t in tok[k:k + 4]]
            assert np.allclose(vals, [float(t) for t in tok[k + 4:k + 13]], rtol=1e-15,
                               atol=1e-300)
            k += 13


@pytest.mark.gpu
def test_hybrid_reference_file_then_step(tmp_path, lib):
    g = np.load(GOLDEN)
    xml = tmp_path / "reload.xml"
    xml.write_text(str(g["xml"]))
    bf = tmp_path / "reload_Particles.bin"
    bf.write_bytes(g["particles_hybrid"].tobytes())
    sim = Grains(str(xml), FP64)
    sim.read_reload_particles_hybrid(bf)
    out = tmp_path / "again_Particles.bin"
    sim.write_reload_particles_hybrid(out)
    mine, ref = parse_hybrid(out.read_bytes()), parse_hybrid(bf.read_bytes())
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        assert a[0] == b[0] and a[1] == b[1] and a[3] == b[3] and a[4] == b[4] and a[5] == b[5]
        assert a[2][:3] == b[2][:3]
        assert np.max(np.abs(np.array(a[2][3:]) - np.array(b[2][3:]))) <= 1e-12
    sim.set_diagnostics(True)
    sim.step(1)
    s = sim.download_state()
    assert sim.status() == 0
    assert np.array_equal(sim.download_cells(), g["s1_cells"])
    assert np.max(np.abs(s["x"] - g["s1_x"])) <= 1e-15
    id0, id1, _ = sim.download_contacts()
    ref_set = {(min(a, b), max(a, b)) if b >= 0 else (a, b)
               for a, b in zip(g["s1_hist_owner"].tolist(), g["s1_hist_partner"].tolist())}
    got = {(min(a, b), max(a, b)) if b >= 0 else (a, b) for a, b in zip(id0.tolist(), id1.tolist())}
    assert got == ref_set and len(ref_set) > 0
    sim.close()
