"""Contact features (gdem_contact_features) against the reference's own
AppCollision statistics (Base/src/AppCollision.cpp:159-179), recorded by
tests/golden/make_golden.py in contact_features.npz: 300 spheres settling in
the walled box from the reference's inserted state, features after the
leapfrog start and after 400 and 1,200 steps.

The largest and the mean overlap over every contact of every evaluation
must agree to 1e-9 relative in FP64 mode and 1e-5 in FP32-split mode (the
trajectories themselves agree to round-off over these steps), and the step
at which the largest overlap was first reached is the reference's."""
from pathlib import Path

import numpy as np
import pytest

from pacific_b200 import FP32_SPLIT, FP64, Grains

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "contact_features.npz"


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-9), (FP32_SPLIT, 1e-5)])
def test_contact_features_match_reference(tmp_path, lib, precision, tol):
    d = np.load(GOLDEN)
    xml = tmp_path / "features.xml"
    xml.write_text(str(d["xml"]))
    g = Grains(xml, precision)
    g.upload_state(d["type"], d["x0"], d["v0"], d["w0"], d["q0"])
    g.do_before_time_stepping()
    dt = 1e-5
    done = 0
    for m in d["marks"]:
        if m > done:
            g.step(int(m) - done)
        done = int(m)
        ref = d[f"s{m}_features"]
        got = g.contact_features()
        if ref[0] == 0.0:
            assert got["overlap_max"] == 0.0 and got["evaluation_of_max"] == -1
            continue
        assert abs(got["overlap_max"] - ref[0]) <= tol * ref[0], (m, got, ref)
        assert abs(got["overlap_mean"] - ref[1]) <= tol * ref[1], (m, got, ref)
        assert abs(got["evaluation_of_max"] * dt - ref[2]) <= 1e-3 * dt, (m, got, ref)
        # the trajectory still agrees with the reference's
        assert np.abs(g.download_state()["x"] - d[f"s{m}_x"]).max() <= (1e-12 if precision == FP64 else 1e-9)
    g.close()
