"""Long chaotic runs compared statistically: kinetic energy, mean
coordination number and packing fraction of an ensemble of seeded settling
boxes, the CPU FP64 restatement (oracle/) against the GPU in both precision
modes.

Over thousands of steps the trajectories of the two implementations part
(the contact sums run in different orders, and a granular gas amplifies
round-off), so single runs are not compared; instead the ensemble means
must not differ significantly: Welch's t-test with p > 1e-3 on each
quantity (quantities that are equal to within 1e-9 relative across the
ensembles, such as the kinetic energy before the first collisions, are
compared directly).  8 seeds, 400 spheres thrown at up to 0.3 m/s into the
walled 0.03 x 0.03 x 0.06 m box, 12,000 steps of 1e-5 s (the bed has
settled by then: its kinetic energy is down by two orders of magnitude).
"""
import numpy as np
import pytest
from scipy import stats

from oracle.oracle import Oracle
from pacific_b200 import FP32_SPLIT, FP64, Grains, scenarios

pytestmark = pytest.mark.gpu

SEEDS = range(101, 109)
MARKS = (1000, 4000, 12000)
N = 400


def _observables(x, v, w, pairs, radius, density):
    m = density * 4.0 / 3.0 * np.pi * radius ** 3
    inertia = 0.4 * m * radius ** 2
    ke = 0.5 * m * np.sum(v * v) + 0.5 * inertia * np.sum(w * w)
    coord = 2.0 * pairs / len(x)
    # bulk packing fraction: the spheres' volume over the box section times
    # the height of the highest sphere top
    top = x[:, 2].max() + radius
    phi = len(x) * 4.0 / 3.0 * np.pi * radius ** 3 / (0.03 * 0.03 * top)
    return ke, coord, phi


def _run_oracle(sc, xml):
    o = Oracle(xml)
    assert o.set_particles(sc.type, sc.x, sc.v, sc.w, sc.q) == 0
    assert o.init() == 0
    out, done = [], 0
    for m in MARKS:
        assert o.step(m - done) == 0
        done = m
        s = o.state()
        id0, id1, _, _, _ = o.contacts()
        pairs = int(np.sum(id1 >= 0))
        out.append(_observables(s["x"], s["v"], s["w"], pairs, 1e-3, 2500.0))
    return out


def _run_gpu(sc, xml, precision):
    g = Grains(xml, precision)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    out, done = [], 0
    for m in MARKS:
        g.step(m - done - 1)
        g.set_diagnostics(True)
        g.step(1)
        g.set_diagnostics(False)
        done = m
        s = g.download_state()
        id0, id1, _ = g.download_contacts()
        pairs = int(np.sum(id1 >= 0))
        out.append(_observables(s["x"], s["v"], s["w"], pairs, 1e-3, 2500.0))
    assert g.status() == 0
    g.close()
    return out


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(abs(a.mean()), abs(b.mean()), 1e-300)
    if a.std() + b.std() <= 1e-9 * scale:
        return abs(a.mean() - b.mean()) <= 1e-9 * scale, None
    p = stats.ttest_ind(a, b, equal_var=False).pvalue
    return p > 1e-3, p


@pytest.fixture(scope="module")
def ensembles(tmp_path_factory, lib, oracle_lib):
    d = tmp_path_factory.mktemp("stats")
    runs = {"oracle": [], FP64: [], FP32_SPLIT: []}
    for seed in SEEDS:
        sc = scenarios.settling_box(n=N, seed=seed, vmax=0.3)
        xml = str(sc.write_xml(d / f"s{seed}.xml"))
        runs["oracle"].append(_run_oracle(sc, xml))
        runs[FP64].append(_run_gpu(sc, xml, FP64))
        runs[FP32_SPLIT].append(_run_gpu(sc, xml, FP32_SPLIT))
    return {k: np.array(v) for k, v in runs.items()}   # (seed, mark, quantity)


@pytest.mark.parametrize("precision", [FP64, FP32_SPLIT], ids=["fp64", "fp32split"])
def test_ensembles_agree(ensembles, precision):
    ref, got = ensembles["oracle"], ensembles[precision]
    names = ("kinetic energy", "coordination", "packing fraction")
    for k, m in enumerate(MARKS):
        for q, name in enumerate(names):
            ok, p = _same(ref[:, k, q], got[:, k, q])
            assert ok, (m, name, ref[:, k, q].mean(), got[:, k, q].mean(), p)
    # the runs did settle: kinetic energy fell and contacts formed
    assert got[:, -1, 0].mean() < 0.2 * got[:, 0, 0].mean()
    assert got[:, -1, 1].mean() > 1.0
