"""RawData post-processing output and the _VelocityMaxMean.dat line
(gdem_rawdata_start / write / end, gdem_write_velocity_max_mean,
gdem_download_coordination), pinned on files written by the reference's own
RawDataPostProcessingWriter (tests/golden/rawdata_settling_{text,binary}.npz,
made by tests/golden/make_golden.py).

The fixtures: 200 spheres settled for 6,000 steps by the reference, which
writes a Format2024 reload there; its writer starts at that time and writes
after 10 and 100 more steps.  The GPU run reads the same reload file and
writes at the same times.

* CPU: the text and the binary fixture hold the same run, so formatting the
  binary fixture's doubles as GrainsExec::doubleToString(ios::scientific, 6)
  ("%.6e", zero as "0") reproduces the text fixture line for line; this pins
  the file layouts (time first, none in the coordination file, the time
  twice in the binary angular_velocity_z file).
* GPU (FP64): the files written from device state match the reference's:
  times, classes and coordination numbers exactly (the first output comes
  before any force evaluation, whose coordination numbers a reloaded
  reference run also writes as zeros), positions and velocities to their
  printed digits (one unit in the 7th digit: the trajectories agree to
  about 1e-12 after 100 steps, so a value next to a rounding boundary may
  print one unit apart; values below 1e-9 of the quantity's largest, such
  as the round-off velocity of a particle at rest, to that bound), the
  binary doubles to 1e-9 of each quantity's largest value, the velocity
  max/mean to 1e-6.
* GPU (both modes): the text written equals the restated format applied to
  the state and coordination numbers downloaded at the same time.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from pacific_b200 import FP32_SPLIT, FP64, Grains

GOLDEN = Path(__file__).resolve().parent / "golden"
QUANT = ("position_x", "position_y", "position_z", "translational_velocity_x",
         "translational_velocity_y", "translational_velocity_z", "angular_velocity_x",
         "angular_velocity_y", "angular_velocity_z")
N = 200


def fmt(x):
    """GrainsExec::doubleToString(ios::scientific, 6, x)."""
    x = float(x)
    if x != 0.0:
        return f"{x:.6e}"
    return "-0" if math.copysign(1.0, x) < 0 else "0"


def _fixture(mode):
    return np.load(GOLDEN / f"rawdata_settling_{mode}.npz")


def _binary_columns(z):
    """{quantity: (times (k,), values (k, N))}, coordination (k, N), classes (N,)."""
    out = {}
    k = len(z["times"])
    for q in QUANT:
        raw = np.frombuffer(z[q].tobytes(), np.float64)
        head = 2 if q == "angular_velocity_z" else 1
        rec = raw.reshape(k, head + N)
        assert np.all(rec[:, :head] == z["times"][:, None])
        out[q] = rec[:, head:]
    coord = np.frombuffer(z["coordinationNumber"].tobytes(), np.int32).reshape(k, N)
    cls = np.frombuffer(z["particleType"].tobytes(), np.int32)
    assert cls.shape == (N,)
    return out, coord, cls


def _text_lines(times, cols, coord, cls):
    """The text files of one run, restated: {quantity: [lines]}."""
    out = {q: [fmt(t) + "".join(" " + fmt(v) for v in cols[q][i]) + "\n"
               for i, t in enumerate(times)] for q in QUANT}
    out["coordinationNumber"] = ["".join(f" {c}" for c in row) + "\n" for row in coord]
    out["particleType"] = ["".join(f"{c} " for c in cls) + "\n"]
    return out


def test_text_fixture_is_binary_fixture_formatted():
    zt, zb = _fixture("text"), _fixture("binary")
    assert np.array_equal(zt["times"], zb["times"])
    cols, coord, cls = _binary_columns(zb)
    want = _text_lines(zt["times"], cols, coord, cls)
    for name, lines in want.items():
        assert str(zt[name]) == "".join(lines), name
    assert coord[0].sum() > 100          # the settled bed touches


def _gpu_run(tmp_path, precision, binary):
    zt = _fixture("text")
    xml = tmp_path / "raw.xml"
    xml.write_text(str(zt["xml"]))
    pfile = tmp_path / "raw_Particles"
    pfile.write_text(str(zt["particles"]))
    g = Grains(str(xml), precision)
    g.read_reload_particles(pfile)
    root = tmp_path / ("bin" if binary else "txt")
    vfile = tmp_path / "res_VelocityMaxMean.dat"
    times = zt["times"]
    seen = []      # (state, coordination) downloaded at each output time
    done = 0
    for k, m in enumerate(zt["marks"]):
        if k == 0:
            g.rawdata_start(root, binary=binary, append=False, time=times[0])
            g.write_velocity_max_mean(vfile, times[0], append=False)
        else:
            g.step(m - done - 1)
            g.set_diagnostics(True)
            g.step(1)
            g.set_diagnostics(False)
            done = m
            g.rawdata_write(times[k])
            g.write_velocity_max_mean(vfile, times[k])
        seen.append((g.download_state(), g.download_coordination()))
    g.rawdata_end()
    assert g.status() == 0
    g.close()
    return root, vfile, seen


def _read_files(root, binary):
    names = list(QUANT) + ["coordinationNumber", "particleType"]
    return {q: Path(f"{root}_{q}.dat").read_bytes() if binary
            else Path(f"{root}_{q}.dat").read_text() for q in names}


def _cols_of(seen):
    comp = {"position": ("x", 0), "translational_velocity": ("v", 0), "angular_velocity": ("w", 0)}
    cols = {}
    for q in QUANT:
        base, axis = q[:-2], "xyz".index(q[-1])
        key = comp[base][0]
        cols[q] = np.array([s[key][:, axis] for s, _ in seen])
    coord = np.array([c for _, c in seen])
    return cols, coord


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [FP64, FP32_SPLIT], ids=["fp64", "fp32split"])
def test_text_written_is_state_formatted(tmp_path, lib, precision):
    root, _, seen = _gpu_run(tmp_path, precision, binary=False)
    got = _read_files(root, binary=False)
    cols, coord = _cols_of(seen)
    zt = _fixture("text")
    cls = np.zeros(N, np.int32)
    want = _text_lines(zt["times"], cols, coord, cls)
    for name, lines in want.items():
        assert got[name] == "".join(lines), name
    assert np.all(coord[0] == 0) and coord[-1].sum() > 100


def _close_tokens(a, b, scale):
    """Equal strings, or one unit apart in the 7th digit, or apart by less
    than 1e-9 of the quantity's largest value (a velocity of a particle at
    rest is round-off, e.g. 5e-15 m/s, whose digits are not comparable)."""
    if a == b:
        return True
    x, y = float(a), float(b)
    return abs(x - y) <= max(1.0000001e-6 * max(abs(x), abs(y)), 1e-9 * scale)


@pytest.mark.gpu
def test_text_matches_reference(tmp_path, lib):
    root, vfile, _ = _gpu_run(tmp_path, FP64, binary=False)
    got = _read_files(root, binary=False)
    zt = _fixture("text")
    for q in QUANT:
        ref_lines = str(zt[q]).splitlines()
        got_lines = got[q].splitlines()
        assert len(ref_lines) == len(got_lines) == 3, q
        for rl, gl in zip(ref_lines, got_lines):
            rt, gt = rl.split(" "), gl.split(" ")
            assert len(rt) == len(gt) == N + 1 and rt[0] == gt[0], q
            scale = max(abs(float(r)) for r in rt[1:])
            bad = [(r, g) for r, g in zip(rt[1:], gt[1:]) if not _close_tokens(r, g, scale)]
            assert not bad, (q, bad[:5])
    ref_c = str(zt["coordinationNumber"]).splitlines()
    got_c = got["coordinationNumber"].splitlines()
    assert got_c[0] == " 0" * N
    assert got_c[1:] == ref_c[1:]
    assert got["particleType"] == str(zt["particleType"])
    # the _VelocityMaxMean.dat lines
    lines = vfile.read_text().splitlines()
    assert len(lines) == 3
    for line, t, (vmax, vmean) in zip(lines, zt["times"], zt["velocity_max_mean"]):
        tok = line.split("\t")
        assert tok[0] == fmt(t)
        assert abs(float(tok[1]) - vmax) <= 1e-6 * vmax and abs(float(tok[2]) - vmean) <= 1e-6 * vmean


@pytest.mark.gpu
def test_binary_matches_reference(tmp_path, lib):
    root, _, seen = _gpu_run(tmp_path, FP64, binary=True)
    got = _read_files(root, binary=True)
    zb = _fixture("binary")
    ref_cols, ref_coord, ref_cls = _binary_columns(zb)
    # the same parser reads the files written here
    mine = {q: np.frombuffer(got[q], np.uint8) for q in got}
    mine["times"] = zb["times"]
    got_cols, got_coord, got_cls = _binary_columns(mine)
    for q in QUANT:
        scale = np.abs(ref_cols[q]).max()
        err = np.abs(got_cols[q] - ref_cols[q]).max()
        assert err <= 1e-9 * scale, (q, err, scale)
    assert np.all(got_coord[0] == 0)
    assert np.array_equal(got_coord[1:], ref_coord[1:])
    assert np.array_equal(got_cls, ref_cls)
    # and the record holds exactly the downloaded state
    cols, coord = _cols_of(seen)
    for q in QUANT:
        assert np.array_equal(got_cols[q], cols[q])


@pytest.mark.gpu
def test_writer_refuses_a_batch(tmp_path, lib):
    from pacific_b200 import GrainsError, scenarios
    inst = scenarios.batched_boxes(n_inst=2, nmin=50, nmax=80, seed=7)
    xmls = [str(s.write_xml(tmp_path / f"i{k}.xml")) for k, s in enumerate(inst)]
    ins, typ, x, v, w, q = scenarios.concat_state(inst)
    g = Grains(xmls, FP64)
    g.upload_state(typ, x, v, w, q, inst=ins)
    with pytest.raises(GrainsError, match="batch"):
        g.rawdata_start(tmp_path / "out")
    g.close()
