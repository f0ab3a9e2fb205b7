"""The drop-in boundary under the reference's own driver.

oracle/_ref/grains_b200 is the Grains3D executable built from the
reference's unmodified sources and main() (GRAINS_V1/Main/src/main.cpp) with
the GrainsB200 application added (pacific_b200/integration: the factory's
"B200" branch, reached by a link-time wrap of GrainsBuilderFactory::create).
The same input file -- 200 spheres inserted at the initial time from a
positions file with seeded random velocities, settling in the walled box,
outputs every 100 steps: RawData writer, reload files, velocity max/mean --
is run once as Type="Standard" (the reference's serial CPU step) and once as
Type="B200" (the time loop on the GPU, FP64).  Everything the reference's
writers produce must agree: output times, coordination numbers and particle
classes exactly, the printed positions and velocities (%.6e) to their last
digit, the velocity max/mean lines, the contact memory of the final reload
file (pairs exactly, values to round-off) and its positions to 1e-12.

A second input pours particles over time (Mode Type="OverTime": one attempt
every 20 steps at a random point of a box window, seeded random velocities):
the reference picks each particle, point and velocity in both runs, the
overlap test runs on the reference's host particles in one and on the device
(gdem_insert_particle) in the other, so the same particles must go in at the
same steps and end at the same positions.
"""
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from pacific_b200 import scenarios

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "oracle" / "_ref" / "grains_b200"

RAW = ("position_x", "position_y", "position_z", "translational_velocity_x",
       "translational_velocity_y", "translational_velocity_z", "angular_velocity_x",
       "angular_velocity_y", "angular_velocity_z")


def _input(d, kind, n=200, seed=11, steps=400, every=100, dt=1e-5):
    """A complete Grains3D input: construction of the walled settling box,
    insertion at the initial time from a positions file with seeded random
    velocities, outputs every `every` steps."""
    d.mkdir(parents=True, exist_ok=True)
    sc = scenarios.settling_box(n=n, seed=seed)
    np.savetxt(d / "positions.txt", sc.x, fmt="%.17g")
    end = steps * dt
    text = sc.xml().replace('<Grains3D Type="Standard">', f'<Grains3D Type="{kind}">')
    text = re.sub(r"<TimeInterval[^>]*/>", f'<TimeInterval Start="0." End="{end!r}"/>', text)
    sim = (f'    <RestartFile Name="{d}/res" WritingMode="Text"/>\n'
           f'    <TimeSave Start="0." End="{end!r}" Every="{every * dt!r}"/>\n'
           "    <ParticleInsertion>\n"
           '      <Mode Type="InitialTime"/>\n'
           '      <Order Type="Ordered"/>\n'
           '      <RandomGeneratorSeed Type="UserDefined" Value="7"/>\n'
           f'      <ParticlePosition>\n        <File Name="{d}/positions.txt"/>\n'
           "      </ParticlePosition>\n"
           '      <InitialVelocity Mode="Random">\n'
           '        <Translational Amplitude="0.3"/>\n'
           '        <Angular Amplitude="0."/>\n'
           "      </InitialVelocity>\n"
           "    </ParticleInsertion>\n"
           "    <PostProcessing>\n      <Writers>\n"
           f'        <RawData Name="{d}/raw" WritingMode="Text"/>\n'
           "      </Writers>\n    </PostProcessing>\n")
    (d / "input.xml").write_text(text.replace("  </Simulation>", sim + "  </Simulation>"))
    return d / "input.xml"


def _input_overtime(d, kind, n=120, seed=5, steps=3000, every=1000, dt=1e-5):
    """The walled box filled over time: n spheres, one insertion attempt every
    20 steps at a random point of a window in the upper part of the box."""
    d.mkdir(parents=True, exist_ok=True)
    sc = scenarios.settling_box(n=n, seed=seed)
    end = steps * dt
    text = sc.xml().replace('<Grains3D Type="Standard">', f'<Grains3D Type="{kind}">')
    text = re.sub(r"<TimeInterval[^>]*/>", f'<TimeInterval Start="0." End="{end!r}"/>', text)
    sim = (f'    <RestartFile Name="{d}/res" WritingMode="Text"/>\n'
           f'    <TimeSave Start="0." End="{end!r}" Every="{every * dt!r}"/>\n'
           "    <ParticleInsertion>\n"
           '      <Mode Type="OverTime"/>\n'
           '      <Order Type="Ordered"/>\n'
           '      <RandomGeneratorSeed Type="UserDefined" Value="3"/>\n'
           '      <Frequency TryEvery="20"/>\n'
           "      <ParticlePosition>\n        <Windows>\n"
           '          <Window Type="Box">\n'
           '            <Point X="0.004" Y="0.004" Z="0.030"/>\n'
           '            <Point X="0.026" Y="0.026" Z="0.056"/>\n'
           "          </Window>\n        </Windows>\n"
           "      </ParticlePosition>\n"
           '      <InitialVelocity Mode="Random">\n'
           '        <Translational Amplitude="0.2"/>\n'
           '        <Angular Amplitude="0."/>\n'
           "      </InitialVelocity>\n"
           "    </ParticleInsertion>\n"
           "    <PostProcessing>\n      <Writers>\n"
           f'        <RawData Name="{d}/raw" WritingMode="Text"/>\n'
           "      </Writers>\n    </PostProcessing>\n")
    (d / "input.xml").write_text(text.replace("  </Simulation>", sim + "  </Simulation>"))
    return d / "input.xml"


def _run(xml):
    env = dict(os.environ, GRAINS_HOME=str(xml.parent), GRAINS_B200_PRECISION="fp64")
    r = subprocess.run([str(EXE), xml.name], cwd=str(xml.parent), capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


def _reload_particles(path):
    """Per particle ID: position (3) and the contact memory {partner: 9 values}
    of a Format2024 text particle file (Particle::write2014)."""
    out = {}
    for line in path.read_text().splitlines():
        tok = line.split()
        # class ID tag activity | x (3) | basis (9) | transform type | v (3)
        # | q (4) | omega (3) | F (3) | T (3) | map size, entries of 13
        if len(tok) < 34:
            continue
        pid = int(tok[1])
        x = np.array(tok[4:7], float)
        nmap = int(tok[33])
        mem = {}
        k = 34
        for _ in range(nmap):
            partner = int(tok[k + 1])
            mem[partner] = np.array(tok[k + 4:k + 13], float)
            k += 13
        out[pid] = (x, mem)
    return out


@pytest.mark.skipif(not EXE.exists(), reason="oracle/_ref/grains_b200 was not built")
def test_type_b200_under_reference_driver_matches_standard(tmp_path, lib):
    std = _input(tmp_path / "std", "Standard")
    b200 = _input(tmp_path / "b200", "B200")
    _run(std)
    out = _run(b200)
    assert "GrainsB200" not in out or "stopped" not in out
    sd, bd = std.parent, b200.parent
    # coordination numbers and classes exactly
    for name in ("coordinationNumber", "particleType"):
        a = (sd / f"raw_{name}.dat").read_text().split()
        b = (bd / f"raw_{name}.dat").read_text().split()
        assert a == b, name
    coord = np.array((sd / "raw_coordinationNumber.dat").read_text().split(), int)
    assert coord.sum() > 0
    # printed values: the same text, or (a value on a rounding boundary of its
    # 7 printed digits) one unit of the last digit apart
    exact = total = 0
    for name in RAW:
        la = (sd / f"raw_{name}.dat").read_text().split()
        lb = (bd / f"raw_{name}.dat").read_text().split()
        assert len(la) == len(lb), name
        fa, fb = np.array(la, float), np.array(lb, float)
        same = np.array([x == y for x, y in zip(la, lb)])
        exact += int(same.sum())
        total += same.size
        assert np.all(np.abs(fa - fb) <= 1e-6 * np.maximum(np.abs(fa), 1e-300) + 1e-300), name
    assert exact >= total - 2, (exact, total)
    # velocity max/mean lines
    va = np.loadtxt(sd / "res_VelocityMaxMean.dat")
    vb = np.loadtxt(bd / "res_VelocityMaxMean.dat")
    assert va.shape == vb.shape and np.allclose(va, vb, rtol=1e-6, atol=0)
    # the last reload: positions and contact memory
    ra = sorted(sd.glob("res*_Particles.result"), key=lambda p: p.stat().st_mtime)[-1]
    rb = bd / ra.name
    pa, pb = _reload_particles(ra), _reload_particles(rb)
    assert pa.keys() == pb.keys()
    nmem = 0
    for pid, (xa, ma) in pa.items():
        xb, mb = pb[pid]
        assert np.abs(xa - xb).max() <= 1e-12, pid
        assert ma.keys() == mb.keys(), pid
        for partner, va_ in ma.items():
            nmem += 1
            assert np.allclose(va_, mb[partner], rtol=1e-7, atol=1e-15), (pid, partner)
    assert nmem > 0


@pytest.mark.skipif(not EXE.exists(), reason="oracle/_ref/grains_b200 was not built")
def test_type_b200_insertion_over_time_matches_standard(tmp_path, lib):
    std = _input_overtime(tmp_path / "std", "Standard")
    b200 = _input_overtime(tmp_path / "b200", "B200")
    _run(std)
    _run(b200)
    sd, bd = std.parent, b200.parent
    ra = sorted(sd.glob("res*_Particles.result"), key=lambda p: p.stat().st_mtime)[-1]
    pa, pb = _reload_particles(ra), _reload_particles(bd / ra.name)
    # the same particles inserted, at the same places
    assert pa.keys() == pb.keys() and len(pa) > 40, (len(pa), len(pb))
    for pid, (xa, ma) in pa.items():
        xb, mb = pb[pid]
        assert np.abs(xa - xb).max() <= 1e-12, pid
        assert ma.keys() == mb.keys(), pid
    for name in ("coordinationNumber", "particleType"):
        assert (sd / f"raw_{name}.dat").read_text().split() == \
            (bd / f"raw_{name}.dat").read_text().split(), name
