"""Calibration harness: gradients of a trajectory loss through the adjoint of
the DEM step (C ABI gdem_adjoint_*, pacific_b200/csrc/gdem_adjoint.cu).

    adj = Adjoint(xml_path)
    adj.set_particles(type, x0, v0)
    loss, g_params, g_v0 = adj.gradients(params, target_x, target_v, nsteps=500, every=50)

`TrajectoryLoss` wraps the same call as a torch.autograd.Function whose
inputs are the parameter vector (kn, en, muc) and the initial velocities, so
that a calibration loop can use a torch optimiser.  The loss is
L = sum_i |x_i(N) - x*_i|^2 + |v_i(N) - v*_i|^2.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .grains import GrainsError, _dp, _ip, library

_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_ready = False


def _lib():
    global _ready
    lib = library()
    if not _ready:
        sig = {
            "gdem_adjoint_create": ([ctypes.c_char_p, ctypes.POINTER(_P)], ctypes.c_int),
            "gdem_adjoint_set_particles": ([_P, ctypes.c_int64, _IP, _DP, _DP, _DP], ctypes.c_int),
            "gdem_adjoint_run": ([_P, ctypes.c_int, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _DP,
                                  _DP, _DP], ctypes.c_int),
            "gdem_adjoint_forward_dual": ([_P, ctypes.c_int, _DP, _DP, _DP, ctypes.c_int,
                                           ctypes.c_int, _DP, _DP], ctypes.c_int),
            "gdem_adjoint_destroy": ([_P], None),
        }
        for name, (args, res) in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        _ready = True
    return lib


def _f64(a, shape):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=np.float64).reshape(shape)


class Adjoint:
    """Adjoint engine for one walled box of spheres (FP64)."""

    def __init__(self, xml_path):
        lib = _lib()
        h = _P()
        self._check(lib.gdem_adjoint_create(str(xml_path).encode(), ctypes.byref(h)))
        self._h = h
        self.n = 0

    @staticmethod
    def _check(rc):
        if rc != 0:
            raise GrainsError(library().gdem_last_error().decode())

    def close(self):
        if self._h:
            _lib().gdem_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_particles(self, type, x0, v0, w0=None):
        n = len(type)
        t = np.ascontiguousarray(type, dtype=np.int32)
        self._x0 = _f64(x0, (n, 3))
        self._v0 = _f64(v0, (n, 3))
        w = _f64(w0, (n, 3))
        self._check(_lib().gdem_adjoint_set_particles(self._h, n, _ip(t), _dp(self._x0),
                                                      _dp(self._v0), _dp(w)))
        self.n = n

    def run(self, params, nsteps, target_x=None, target_v=None):
        """Forward only: (final x, final v, loss or None)."""
        p = _f64(params, (3,))
        xo = np.empty((self.n, 3))
        vo = np.empty((self.n, 3))
        tx, tv = _f64(target_x, (self.n, 3)), _f64(target_v, (self.n, 3))
        loss = ctypes.c_double(0.0)
        self._check(_lib().gdem_adjoint_run(
            self._h, nsteps, max(nsteps, 1), _dp(p), _dp(tx), _dp(tv),
            ctypes.byref(loss) if tx is not None else None, _dp(xo), _dp(vo), None, None))
        return xo, vo, (loss.value if tx is not None else None)

    def gradients(self, params, target_x, target_v, nsteps, every=50):
        """(loss, dL/d(kn, en, muc), dL/dv0) by the reverse sweep."""
        p = _f64(params, (3,))
        tx, tv = _f64(target_x, (self.n, 3)), _f64(target_v, (self.n, 3))
        loss = ctypes.c_double(0.0)
        gp = np.zeros(3)
        gv = np.zeros((self.n, 3))
        self._check(_lib().gdem_adjoint_run(self._h, nsteps, every, _dp(p), _dp(tx), _dp(tv),
                                            ctypes.byref(loss), None, None, _dp(gp), _dp(gv)))
        return loss.value, gp, gv

    def forward_mode(self, params, target_x, target_v, nsteps, v0_component=None):
        """(loss, dL/d(kn, en, muc)) by dual numbers through the whole run; with
        v0_component = (particle, axis): (loss, dL/dv0[particle, axis])."""
        p = _f64(params, (3,))
        tx, tv = _f64(target_x, (self.n, 3)), _f64(target_v, (self.n, 3))
        loss = ctypes.c_double(0.0)
        gp = np.zeros(3)
        i, d = v0_component if v0_component is not None else (-1, 0)
        self._check(_lib().gdem_adjoint_forward_dual(self._h, nsteps, _dp(p), _dp(tx), _dp(tv),
                                                     int(i), int(d), ctypes.byref(loss),
                                                     _dp(gp)))
        return (loss.value, gp) if v0_component is None else (loss.value, gp[0])


def trajectory_loss_function():
    """torch.autograd.Function over (params, v0) for one Adjoint instance;
    built lazily so that importing this module needs no torch."""
    import torch

    class TrajectoryLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, v0, adj, type_, x0, target_x, target_v, nsteps, every):
            adj_ = adj
            if adj_.n == 0:
                adj_.set_particles(type_, x0, v0.detach().cpu().numpy())
            else:
                raise GrainsError("TrajectoryLoss needs a fresh Adjoint per initial state")
            loss, gp, gv = adj_.gradients(params.detach().cpu().numpy(), target_x, target_v,
                                          nsteps, every)
            ctx.save_for_backward(torch.as_tensor(gp, dtype=params.dtype),
                                  torch.as_tensor(gv, dtype=v0.dtype))
            return params.new_tensor(loss)

        @staticmethod
        def backward(ctx, g):
            gp, gv = ctx.saved_tensors
            return g * gp, g * gv, None, None, None, None, None, None, None

    return TrajectoryLoss
