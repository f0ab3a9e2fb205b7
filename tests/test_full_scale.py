"""Parity at scale against the Grains3D reference itself.

The GPU FP64 system is advanced to a state with contacts and writes its
Format2024 particle file; the reference (oracle/_ref, in its own process,
through its own reload path: AllComponents::read_particles, Link,
checkClonesReload) and the GPU in both precision modes read that file and
take one step.  Checked: the reference's cells and contact set exactly, the
per-particle force error (normaliser: the particle's sum of contact-force
magnitudes) within 1e-10 in FP64 and 1e-5 in FP32-split, positions after
the step to round-off.

* 108,000 polydisperse spheres of the periodic gas (FCC n = 30), the state
  after 600 steps;
* 20,000 cubes and tetrahedra of the convex pour launched at up to 2 m/s,
  the state after 150 steps (GJK contacts), every particle within 1e-10 in
  FP64: the pair is oriented as the reference orients it (p0 the particle of
  the lower reference cell number) and each polyhedron's support search
  starts from the vertex its previous call ended on (Polyhedron::
  m_curr_vertex; after reading a particle file, on both sides, the class's
  starting vertex), so that even face-to-face contacts, whose closest points
  are not unique, find the reference's witness points.
"""
import numpy as np
import pytest

from oracle import reference
from pacific_b200 import FP32_SPLIT, FP64, Grains, scenarios
from tests.helpers import radii_of, step_parity

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference.available(),
                                 reason="oracle/_ref (the reference build) is absent")]


def _advance(xml, sc, steps, path):
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    g.step(steps)
    _, contacts = g.pair_counts()
    assert g.status() == 0
    g.write_reload_particles(path)
    g.close()
    return contacts


def test_periodic_gas_108k_one_step_vs_reference(tmp_path, lib):
    sc = scenarios.periodic_gas(n_fcc=30, seed=1236)
    assert sc.n >= 100_000
    xml = str(sc.write_xml(tmp_path / "gas.xml"))
    pfile = tmp_path / "state_Particles"
    assert _advance(xml, sc, 600, pfile) > 100
    period = np.subtract(sc.maxc, sc.origin) * np.asarray(sc.periodic, float)
    r = step_parity(xml, pfile, sc.n, radii_of(sc), (FP64, FP32_SPLIT), period=period)
    print(r)
    assert r["reference"]["contacts"] > 100
    for prec, tol in ((FP64, 1e-10), (FP32_SPLIT, 1e-5)):
        e = r[prec]
        assert e["status"] == 0
        assert e["cells_equal"], prec
        assert e["contacts_equal"], (prec, e)
        assert e["force_max_contact_free"] == 0.0, (prec, e)
        assert e["force_max_interior"] <= tol, (prec, e)
        # across the periodic boundary the reference translates the other
        # partner (periodic_contact_particles): a rounding of x + L against
        # the overlap
        assert e["force_max_periodic"] <= max(tol, 1e-7), (prec, e)
    assert r[FP64]["position_max_abs"] <= 1e-15
    assert r[FP32_SPLIT]["position_max_abs"] <= 1e-13


def test_convex_20k_one_step_vs_reference(tmp_path, lib):
    poly = scenarios.write_tetrahedron(tmp_path / "tet.poly")
    sc = scenarios.convex_pour(n=20_000, seed=1238, poly_path=poly, vmax=2.0)
    xml = str(sc.write_xml(tmp_path / "convex.xml"))
    pfile = tmp_path / "state_Particles"
    assert _advance(xml, sc, 150, pfile) > 50
    r = step_parity(xml, pfile, sc.n, radii_of(sc), (FP64, FP32_SPLIT))
    print(r)
    for prec in (FP64, FP32_SPLIT):
        e = r[prec]
        assert e["status"] == 0
        assert e["cells_equal"], prec
        assert e["contacts_equal"], (prec, e)
        assert e["force_max"] <= (1e-10 if prec == FP64 else 1e-5), (prec, e)
