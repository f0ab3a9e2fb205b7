"""Launch tuning and the autotuner (gdem_set_tuning, gdem_autotune).

The pair-list skin sets the pair-list cell size and how often the list is
rebuilt; the force kernels' grid sets how the work is spread over the
multiprocessors.  Neither may change a result: the contact set is exact for
any skin (the list is a superset, every kept pair is decided in FP64) and
each particle sums its contacts in partner-ID order.  So trajectories under
any tuning are equal to the byte, in both precision modes, and the autotuner
only picks among candidates and leaves the trajectory as it was."""
import numpy as np
import pytest

from pacific_b200 import FP32_SPLIT, FP64, Grains, GrainsError, scenarios

pytestmark = pytest.mark.gpu

SKINS = (0.1, 0.175, 0.25, 0.4, 0.6)
BLOCKS = (2, 4, 8)


@pytest.fixture(scope="module")
def dense(tmp_path_factory, lib):
    sc = scenarios.periodic_gas(n_fcc=8, seed=77, spacing=2.35e-3, sigma=0.3)
    xml = str(sc.write_xml(tmp_path_factory.mktemp("tune") / "dense.xml"))
    return sc, xml


def _run(sc, xml, precision, steps, tuning=None, autotune=None):
    g = Grains(xml, precision)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    chosen = None
    if tuning is not None:
        g.set_tuning(*tuning)
    if autotune is not None:
        chosen = g.autotune(trial_steps=autotune)
    g.do_before_time_stepping()
    g.step(steps)
    s = g.download_state()
    counts = g.step_counts()
    st = g.status()
    g.close()
    return s, counts, st, chosen


@pytest.mark.parametrize("precision", [FP64, FP32_SPLIT], ids=["fp64", "fp32split"])
def test_tuning_does_not_change_the_trajectory(dense, precision):
    sc, xml = dense
    ref, ref_counts, st, _ = _run(sc, xml, precision, 80)
    assert st == 0 and ref_counts[1] >= 1
    for tuning in ((0.0, 1), (0.1, 2), (0.6, 8), (None, 3)):
        s, counts, st, _ = _run(sc, xml, precision, 80, tuning=tuning)
        assert st == 0
        for k in ("x", "v", "w", "q", "F", "T"):
            assert np.array_equal(s[k], ref[k]), (tuning, k)
        if tuning[0] == 0.0:
            # no skin: the list is rebuilt before every force evaluation
            assert counts[1] == counts[0]


def test_autotune_picks_a_candidate(dense):
    sc, xml = dense
    ref, _, _, _ = _run(sc, xml, FP32_SPLIT, 60)
    s, _, st, chosen = _run(sc, xml, FP32_SPLIT, 60, autotune=10)
    assert st == 0
    assert chosen["skin_factor"] in SKINS and chosen["blocks_per_sm"] in BLOCKS
    assert chosen["ms_per_step"] > 0.0
    for k in ("x", "v", "w", "q", "F", "T"):
        assert np.array_equal(s[k], ref[k]), k


def test_tuning_is_refused_after_init(dense):
    sc, xml = dense
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    with pytest.raises(GrainsError):
        g.set_tuning(0.2, 4)
    with pytest.raises(GrainsError):
        g.autotune(5)
    g.close()
