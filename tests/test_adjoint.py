"""Adjoint of the DEM step (calibration gradients) against forward-mode dual
numbers and central finite differences.

Both the reverse sweep and the dual-number forward run differentiate the same
discrete FP64 trajectory exactly, so they agree to round-off (1e-8 relative
here), for the parameters and for single initial-velocity components.
Central differences (h = 1e-6 relative) agree with the parameter gradient to
1e-4; for initial velocities, where one particle's perturbation can move a
stick/slip switch of its own contacts inside the difference interval, they
are a coarse check (5 %)."""
import numpy as np
import pytest

from pacific_b200 import scenarios
from pacific_b200.adjoint import Adjoint, trajectory_loss_function

pytestmark = pytest.mark.gpu

P_TARGET = np.array([2.0e4, 0.6, 0.35])
P_START = P_TARGET * np.array([1.05, 0.95, 1.05])


def _case(tmp_path, n=200, steps=200):
    sc = scenarios.adjoint_box(n=n, box=(0.008, 0.008, 0.04), seed=41)
    xml = sc.write_xml(tmp_path / "adj.xml")
    ref = Adjoint(xml)
    ref.set_particles(sc.type, sc.x, sc.v)
    tx, tv, _ = ref.run(P_TARGET, steps)
    ref.close()
    return sc, xml, tx, tv, steps


def test_adjoint_matches_forward_mode_and_differences(tmp_path, lib):
    sc, xml, tx, tv, steps = _case(tmp_path)
    adj = Adjoint(xml)
    adj.set_particles(sc.type, sc.x, sc.v)
    loss, gp, gv = adj.gradients(P_START, tx, tv, steps, every=50)
    loss_f, gp_f = adj.forward_mode(P_START, tx, tv, steps)
    assert loss > 0 and abs(loss - loss_f) <= 1e-12 * loss
    assert np.all(np.abs(gp - gp_f) <= 1e-8 * np.abs(gp_f) + 1e-12 * np.abs(gp_f).max())
    # central differences in each parameter
    for k in range(3):
        h = 1e-6 * P_START[k]
        pp, pm = P_START.copy(), P_START.copy()
        pp[k] += h
        pm[k] -= h
        lp = adj.run(pp, steps, tx, tv)[2]
        lm = adj.run(pm, steps, tx, tv)[2]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - gp[k]) <= 1e-4 * abs(gp[k]), (k, fd, gp[k])
    adj.close()
    # initial velocities: forward mode seeded on single components (exact),
    # and central differences as a coarse check (a contact that switches
    # between stick and slip inside the perturbation makes the loss kinked
    # there, which a difference quotient averages)
    adj = Adjoint(xml)
    adj.set_particles(sc.type, sc.x, sc.v)
    rng = np.random.default_rng(3)
    scale = np.abs(gv).max()
    for i, d in zip(rng.integers(0, sc.n, 4), rng.integers(0, 3, 4)):
        _, gfm = adj.forward_mode(P_START, tx, tv, steps, v0_component=(i, d))
        assert abs(gfm - gv[i, d]) <= 1e-8 * abs(gfm) + 1e-12 * scale, (i, d, gfm, gv[i, d])
        h = 1e-6
        out = []
        for sgn in (1, -1):
            v0 = sc.v.copy()
            v0[i, d] += sgn * h
            a = Adjoint(xml)
            a.set_particles(sc.type, sc.x, v0)
            out.append(a.run(P_START, steps, tx, tv)[2])
            a.close()
        fd = (out[0] - out[1]) / (2 * h)
        assert abs(fd - gv[i, d]) <= 5e-2 * abs(gv[i, d]) + 1e-6 * scale, (i, d, fd, gv[i, d])
    adj.close()


def test_forward_model_follows_the_production_step(tmp_path, lib):
    """The adjoint's forward model (linked-cell search, space-frame sphere
    leapfrog) against the production FP64 step from the same start: the two
    differ only in the rounding of the sums and of the angular update, so
    after 200 steps of collisions the states agree to far below the crust."""
    from pacific_b200 import FP64, Grains
    sc, xml, tx, tv, steps = _case(tmp_path)
    g = Grains(str(xml), FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    g.do_before_time_stepping()
    g.step(steps)
    s = g.download_state()
    g.close()
    assert np.abs(tx - s["x"]).max() <= 1e-12
    assert np.abs(tv - s["v"]).max() <= 1e-9 * np.abs(s["v"]).max()


def test_checkpoint_interval_does_not_change_gradients(tmp_path, lib):
    sc, xml, tx, tv, steps = _case(tmp_path, n=120, steps=120)
    res = []
    for every in (1, 7, 120):
        adj = Adjoint(xml)
        adj.set_particles(sc.type, sc.x, sc.v)
        res.append(adj.gradients(P_START, tx, tv, steps, every=every))
        adj.close()
    for r in res[1:]:
        assert r[0] == res[0][0]
        assert np.array_equal(r[1], res[0][1]) and np.array_equal(r[2], res[0][2])


def test_torch_function(tmp_path, lib):
    import torch
    sc, xml, tx, tv, steps = _case(tmp_path, n=120, steps=100)
    TL = trajectory_loss_function()
    p = torch.tensor(P_START, dtype=torch.float64, requires_grad=True)
    v0 = torch.tensor(sc.v, dtype=torch.float64, requires_grad=True)
    loss = TL.apply(p, v0, Adjoint(xml), sc.type, sc.x, tx, tv, steps, 50)
    loss.backward()
    adj = Adjoint(xml)
    adj.set_particles(sc.type, sc.x, sc.v)
    l2, gp, gv = adj.gradients(P_START, tx, tv, steps, 50)
    assert float(loss.detach()) == l2
    assert np.array_equal(p.grad.numpy(), gp) and np.array_equal(v0.grad.numpy(), gv)
