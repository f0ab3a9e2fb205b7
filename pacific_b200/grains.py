"""Python binding of the C ABI in include/grains_b200.h.

The class mirrors the reference's application object (GRAINS_V1/Grains/Base/
include/Grains.hh): construction from the XML input, the leapfrog start
(``do_before_time_stepping``, Grains.cpp:95-173) and the time loop
(``Simulation``, Grains.cpp:271-452), plus the state accessors that the
reference's reload/post-processing files carry.  Errors that the reference
throws as C++ exceptions (ContactError, MotionError, SimulationError,
Base/include/Error.hh) are reported by :meth:`status` and raised by
:meth:`Simulation` as :class:`SimulationError` subclasses.

There is no CPU path: loading fails when the CUDA library is missing, and
creating a system fails without a CUDA device.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libgrains_b200.so"
_lib = None

FP64 = 0
FP32_SPLIT = 1

ST_CONTACT_OVERLAP = 0x01
ST_MOTION = 0x02
ST_OUT_OF_GRID = 0x04
ST_HASH_FULL = 0x08
ST_GJK_MAXITER = 0x10
ST_TIMEOUT = 0x20
ST_PAIRS_FULL = 0x40


class GrainsError(RuntimeError):
    """A C-ABI call failed (invalid input, CUDA error, call out of sequence)."""


class SimulationError(RuntimeError):
    """Base of the step errors (Base/include/Error.hh)."""


class ContactError(SimulationError):
    """Overlap reached the sum of the crust thicknesses."""


class MotionError(SimulationError):
    """A particle moved more than its crust thickness in one step."""


class OutOfGridError(SimulationError):
    """A particle left the linked-cell grid."""


_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def library() -> ctypes.CDLL:
    """Loads libgrains_b200.so (built by pacific_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise GrainsError(f"{_LIB_PATH} is missing: run `python -m pacific_b200.build` "
                          "(the DEM step has no CPU fallback)")
    lib = ctypes.CDLL(str(_LIB_PATH))
    i64 = ctypes.c_int64
    sig = {
        "gdem_create": ([ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_P)], ctypes.c_int),
        "gdem_create_batch": ([ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                               ctypes.POINTER(_P)], ctypes.c_int),
        "gdem_upload_state": ([_P, i64, _IP, _IP, _DP, _DP, _DP, _DP, _DP], ctypes.c_int),
        "gdem_upload_forces": ([_P, _DP, _DP], ctypes.c_int),
        "gdem_reserve": ([_P, i64], ctypes.c_int),
        "gdem_insert_particle": ([_P, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, _IP, _IP], ctypes.c_int),
        "gdem_upload_history": ([_P, i64, _IP, _IP, _DP, _DP, _DP], ctypes.c_int),
        "gdem_write_reload_particles": ([_P, ctypes.c_char_p], ctypes.c_int),
        "gdem_write_reload_particles_hybrid": ([_P, ctypes.c_char_p], ctypes.c_int),
        "gdem_read_reload_particles_hybrid": ([_P, ctypes.c_char_p], ctypes.c_int),
        "gdem_read_reload_particles": ([_P, ctypes.c_char_p], ctypes.c_int),
        "gdem_set_fluid": ([_P, ctypes.c_double, ctypes.c_int], ctypes.c_int),
        "gdem_set_time_step": ([_P, ctypes.c_double], ctypes.c_int),
        "gdem_set_velocities": ([_P, _DP, _DP], ctypes.c_int),
        "gdem_set_hydro_forces": ([_P, _DP, _DP], ctypes.c_int),
        "gdem_init": ([_P], ctypes.c_int),
        "gdem_set_tuning": ([_P, ctypes.c_double, ctypes.c_int], ctypes.c_int),
        "gdem_autotune": ([_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)],
                          ctypes.c_int),
        "gdem_step": ([_P, ctypes.c_int], ctypes.c_int),
        "gdem_download_state": ([_P, _DP, _DP, _DP, _DP, _DP, _DP, _DP], ctypes.c_int),
        "gdem_download_cells": ([_P, _IP], ctypes.c_int),
        "gdem_download_coordination": ([_P, _IP], ctypes.c_int),
        "gdem_download_classes": ([_P, _IP], ctypes.c_int),
        "gdem_download_ids": ([_P, _IP], ctypes.c_int),
        "gdem_upload_support_vertices": ([_P, _IP], ctypes.c_int),
        "gdem_download_support_vertices": ([_P, _IP], ctypes.c_int),
        "gdem_contact_features": ([_P, _DP, _DP, ctypes.POINTER(ctypes.c_int64), _DP, ctypes.c_int],
                                  ctypes.c_int),
        "gdem_num_instances": ([_P], ctypes.c_int),
        "gdem_rawdata_start": ([_P, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double],
                               ctypes.c_int),
        "gdem_rawdata_write": ([_P, ctypes.c_double], ctypes.c_int),
        "gdem_rawdata_end": ([_P], ctypes.c_int),
        "gdem_write_velocity_max_mean": ([_P, ctypes.c_char_p, ctypes.c_int, ctypes.c_double],
                                         ctypes.c_int),
        "gdem_upload_basis": ([_P, _DP], ctypes.c_int),
        "gdem_download_basis": ([_P, _DP], ctypes.c_int),
        "gdem_set_diagnostics": ([_P, ctypes.c_int], ctypes.c_int),
        "gdem_download_history": ([_P, i64, ctypes.POINTER(i64), _IP, _IP, _DP, _DP, _DP],
                                  ctypes.c_int),
        "gdem_download_contacts": ([_P, i64, ctypes.POINTER(i64), _IP, _IP, _DP, _DP],
                                   ctypes.c_int),
        "gdem_status": ([_P, _IP, ctypes.c_int], ctypes.c_int),
        "gdem_grid": ([_P, ctypes.c_int, _IP, _DP, _DP], ctypes.c_int),
        "gdem_num_particles": ([_P], i64),
        "gdem_last_step_ms": ([_P], ctypes.c_double),
        "gdem_use_graphs": ([_P, ctypes.c_int], ctypes.c_int),
        "gdem_set_contact_memory_pruning": ([_P, ctypes.c_int], ctypes.c_int),
        "gdem_set_state": ([_P, _DP, _DP, _DP, _DP, _DP, _DP, _DP], ctypes.c_int),
        "gdem_velocity_stats": ([_P, _DP, _DP], ctypes.c_int),
        "gdem_set_profiling": ([_P, ctypes.c_int], ctypes.c_int),
        "gdem_law_counts": ([_P, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.c_int],
                            ctypes.c_int),
        "gdem_gjk_counts": ([_P, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64),
                             ctypes.c_int], ctypes.c_int),
        "gdem_step_counts": ([_P, ctypes.POINTER(i64), ctypes.POINTER(i64)], ctypes.c_int),
        "gdem_pair_counts": ([_P, ctypes.POINTER(i64), ctypes.POINTER(i64)], ctypes.c_int),
        "gdem_kernel_times": ([_P, ctypes.c_int, _IP, ctypes.c_char_p, _DP,
                               ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "gdem_last_error": ([], ctypes.c_char_p),
        "gdem_destroy": ([_P], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_DP)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_IP)


def _f64(a, shape):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape)


class Grains:
    """A Grains3D system (or a batch of independent systems) on one B200."""

    def __init__(self, xml, precision: int = FP64):
        lib = library()
        h = _P()
        if isinstance(xml, (list, tuple)):
            arr = (ctypes.c_char_p * len(xml))(*[os.fsencode(str(p)) for p in xml])
            rc = lib.gdem_create_batch(len(xml), arr, precision, ctypes.byref(h))
        else:
            rc = lib.gdem_create(os.fsencode(str(xml)), precision, ctypes.byref(h))
        self._check(rc)
        self._h = h
        self.precision = precision
        self.n = 0

    # -------------------------------------------------------------- helpers
    @staticmethod
    def _check(rc):
        if rc != 0:
            raise GrainsError(library().gdem_last_error().decode())

    def close(self):
        if getattr(self, "_h", None):
            library().gdem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ----------------------------------------------------------------- state
    def upload_state(self, type, x, v, w, q, inst=None, wbf=None):
        n = len(type)
        t = np.ascontiguousarray(type, dtype=np.int32)
        ins = None if inst is None else np.ascontiguousarray(inst, dtype=np.int32)
        arrs = [_f64(x, (n, 3)), _f64(v, (n, 3)), _f64(w, (n, 3)), _f64(wbf, (n, 3)),
                _f64(q, (n, 4))]
        self._check(library().gdem_upload_state(self._h, n, _ip(ins), _ip(t), _dp(arrs[0]),
                                                 _dp(arrs[1]), _dp(arrs[2]), _dp(arrs[3]),
                                                 _dp(arrs[4])))
        self.n = n

    # ---- fluid coupling (GrainsCoupledWithFluid) ----
    def set_fluid(self, fluid_density, corrected_acceleration=True):
        """Buoyant weight m (1 - rho_f / rho) g and, with corrected
        acceleration, the coupling factor c = 1 - rho_f / rho of the kicks."""
        self._check(library().gdem_set_fluid(self._h, float(fluid_density),
                                             1 if corrected_acceleration else 0))

    def set_time_step(self, dt):
        self._check(library().gdem_set_time_step(self._h, float(dt)))

    def set_velocities(self, v, w):
        """Velocities and space-frame angular velocities from the fluid, by ID."""
        v = _f64(v, (self.n, 3))
        w = _f64(w, (self.n, 3))
        self._check(library().gdem_set_velocities(self._h, _dp(v), _dp(w)))

    def set_hydro_forces(self, F=None, T=None):
        """Hydrodynamic force and torque by ID, added at every step (None: clear)."""
        if F is None and T is None:
            self._check(library().gdem_set_hydro_forces(self._h, None, None))
            return
        F = _f64(F, (self.n, 3))
        T = _f64(T, (self.n, 3))
        self._check(library().gdem_set_hydro_forces(self._h, _dp(F), _dp(T)))

    def read_reload_particles(self, path):
        """Loads a Format2024 reload particle file (state, forces, contact
        memory); stepping then continues without do_before_time_stepping."""
        self._check(library().gdem_read_reload_particles(self._h, os.fsencode(str(path))))
        self.n = library().gdem_num_particles(self._h)

    def read_reload_particles_hybrid(self, path):
        """Loads the hybrid (binary) form of a reload particle file."""
        self._check(library().gdem_read_reload_particles_hybrid(self._h, os.fsencode(str(path))))
        self.n = library().gdem_num_particles(self._h)

    def write_reload_particles_hybrid(self, path):
        self._check(library().gdem_write_reload_particles_hybrid(self._h, os.fsencode(str(path))))

    def write_reload_particles(self, path):
        """Writes the state after the last step as a Format2024 reload
        particle file."""
        self._check(library().gdem_write_reload_particles(self._h, os.fsencode(str(path))))

    def upload_basis(self, basis):
        """Orientation matrices (n, 3, 3) or (n, 9), row-major, by particle ID;
        only right after upload_state / set_state.  Without it they follow q."""
        b = _f64(basis, (self.n, 9))
        self._check(library().gdem_upload_basis(self._h, _dp(b)))

    def download_basis(self):
        out = np.empty((self.n, 9))
        self._check(library().gdem_download_basis(self._h, _dp(out)))
        return out

    def reserve(self, extra):
        """Room for `extra` particles inserted after the upload (before
        upload_state)."""
        self._check(library().gdem_reserve(self._h, int(extra)))

    def insert_particle(self, type, x, v=(0., 0., 0.), w=(0., 0., 0.), q=(0., 0., 0., 1.),
                        basis=None, force=False, bv_only=False, ref_id=0):
        """One insertion attempt (Grains::insertParticle): the particle goes in
        unless it touches a particle or a wall (or force).  Returns its
        particle ID, or None when it was not inserted."""
        arr = [_f64(a, (k,)) for a, k in ((x, 3), (v, 3), (w, 3), (q, 4))]
        b = _f64(basis, (9,))
        ins = ctypes.c_int(0)
        pid = ctypes.c_int(-1)
        self._check(library().gdem_insert_particle(
            self._h, int(type), *[_dp(a) for a in arr], _dp(b), 1 if force else 0,
            1 if bv_only else 0, int(ref_id), ctypes.byref(ins), ctypes.byref(pid)))
        if not ins.value:
            return None
        self.n += 1
        return pid.value

    def upload_forces(self, F, T):
        F = _f64(F, (self.n, 3))
        T = _f64(T, (self.n, 3))
        self._check(library().gdem_upload_forces(self._h, _dp(F), _dp(T)))

    def upload_history(self, owner, partner, kdelta, prevn, spring=None):
        m = len(owner)
        o = np.ascontiguousarray(owner, dtype=np.int32)
        p = np.ascontiguousarray(partner, dtype=np.int32)
        kd = _f64(kdelta, (m, 3))
        pn = _f64(prevn, (m, 3))
        sp = _f64(spring, (m, 3))
        self._check(library().gdem_upload_history(self._h, m, _ip(o), _ip(p), _dp(kd), _dp(pn),
                                                  _dp(sp)))

    def set_state(self, x, v, w, q, F=None, T=None, wbf=None):
        """Replaces the state in place (no allocation); arrays by particle ID.
        Pass pinned host arrays for full-speed copies."""
        n = self.n
        arrs = [_f64(x, (n, 3)), _f64(v, (n, 3)), _f64(w, (n, 3)), _f64(wbf, (n, 3)),
                _f64(q, (n, 4)), _f64(F, (n, 3)), _f64(T, (n, 3))]
        self._check(library().gdem_set_state(self._h, *[_dp(a) for a in arrs]))

    def velocity_stats(self):
        """(max |v|, mean |v|) over the particles."""
        a = ctypes.c_double(0.0)
        b = ctypes.c_double(0.0)
        self._check(library().gdem_velocity_stats(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def download_coordination(self):
        """Coordination number of each particle at the last force evaluation
        (which must have run with diagnostics on), by particle ID."""
        c = np.empty(self.n, np.int32)
        self._check(library().gdem_download_coordination(self._h, _ip(c)))
        return c

    def download_classes(self):
        c = np.empty(self.n, np.int32)
        self._check(library().gdem_download_classes(self._h, _ip(c)))
        return c

    def contact_features(self, reset=False):
        """{overlap_max, overlap_mean, evaluation_of_max, gjk_iterations_mean}
        over the evaluations since the last reset (the contact features
        Grains3D prints at the end of a run)."""
        a, b, d = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        c = ctypes.c_int64()
        self._check(library().gdem_contact_features(self._h, ctypes.byref(a), ctypes.byref(b),
                                                    ctypes.byref(c), ctypes.byref(d), int(reset)))
        return {"overlap_max": a.value, "overlap_mean": b.value, "evaluation_of_max": c.value,
                "gjk_iterations_mean": d.value}

    def upload_support_vertices(self, vertex):
        """Current polyhedron support vertex of each particle, by ID."""
        v = np.ascontiguousarray(vertex, dtype=np.int32)
        self._check(library().gdem_upload_support_vertices(self._h, _ip(v)))

    def download_support_vertices(self):
        v = np.empty(self.n, np.int32)
        self._check(library().gdem_download_support_vertices(self._h, _ip(v)))
        return v

    def download_ids(self):
        """Reference particle IDs (1-based) by particle index."""
        c = np.empty(self.n, np.int32)
        self._check(library().gdem_download_ids(self._h, _ip(c)))
        return c

    def rawdata_start(self, root, binary=False, append=False, time=0.0):
        """Opens the RawData post-processing files <root>_*.dat and writes
        the first output time."""
        self._check(library().gdem_rawdata_start(self._h, os.fsencode(str(root)), int(binary),
                                                 int(append), float(time)))

    def rawdata_write(self, time):
        self._check(library().gdem_rawdata_write(self._h, float(time)))

    def rawdata_end(self):
        self._check(library().gdem_rawdata_end(self._h))

    def write_velocity_max_mean(self, path, time, append=True):
        """Appends (or, append=False, starts) a line of <root>_VelocityMaxMean.dat."""
        self._check(library().gdem_write_velocity_max_mean(self._h, os.fsencode(str(path)),
                                                           int(append), float(time)))

    def pair_counts(self):
        """(directed pair-list entries, live contact-memory entries) of the
        last force evaluation."""
        a = ctypes.c_int64(0)
        b = ctypes.c_int64(0)
        self._check(library().gdem_pair_counts(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def gjk_counts(self, reset=False):
        """(calls, iterations, most iterations of one call) of the GJK narrow
        phase since the last reset (convex bodies)."""
        c, it, mx = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        self._check(library().gdem_gjk_counts(self._h, ctypes.byref(c), ctypes.byref(it),
                                              ctypes.byref(mx), 1 if reset else 0))
        return c.value, it.value, mx.value

    def step_counts(self):
        """(force evaluations, pair-list rebuilds) since the state was created."""
        a = ctypes.c_int64(0)
        b = ctypes.c_int64(0)
        self._check(library().gdem_step_counts(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def law_counts(self, reset=False):
        """(contact-law evaluations, FP64 re-evaluations) of FP32-split mode."""
        a = ctypes.c_int64(0)
        b = ctypes.c_int64(0)
        self._check(library().gdem_law_counts(self._h, ctypes.byref(a), ctypes.byref(b),
                                              1 if reset else 0))
        return a.value, b.value

    def set_profiling(self, on=True):
        self._check(library().gdem_set_profiling(self._h, 1 if on else 0))

    def kernel_times(self):
        """{phase: (total_ms, launches)} accumulated while profiling."""
        lib = library()
        cnt = ctypes.c_int(0)
        self._check(lib.gdem_kernel_times(self._h, 0, ctypes.byref(cnt), None, None, None))
        k = cnt.value
        names = ctypes.create_string_buffer(32 * max(k, 1))
        ms = np.zeros(max(k, 1))
        nl = np.zeros(max(k, 1), np.int64)
        self._check(lib.gdem_kernel_times(self._h, k, ctypes.byref(cnt), names, _dp(ms),
                                          nl.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        raw = names.raw
        return {raw[32 * i:32 * (i + 1)].split(b"\0")[0].decode(): (float(ms[i]), int(nl[i]))
                for i in range(k)}

    def download_state(self):
        n = self.n
        out = {k: np.empty((n, 3)) for k in ("x", "v", "w", "wbf", "F", "T")}
        out["q"] = np.empty((n, 4))
        self._check(library().gdem_download_state(
            self._h, _dp(out["x"]), _dp(out["v"]), _dp(out["w"]), _dp(out["wbf"]),
            _dp(out["q"]), _dp(out["F"]), _dp(out["T"])))
        return out

    def download_cells(self):
        ijk = np.empty((self.n, 3), dtype=np.int32)
        self._check(library().gdem_download_cells(self._h, _ip(ijk)))
        return ijk

    def set_diagnostics(self, on=True):
        self._check(library().gdem_set_diagnostics(self._h, 1 if on else 0))

    def download_contacts(self, forces=False):
        """(id0, id1, overlap) of the last force evaluation's contacts, plus
        the force on id0 (m, 3) when forces=True."""
        lib = library()
        cnt = ctypes.c_int64(0)
        self._check(lib.gdem_download_contacts(self._h, 0, ctypes.byref(cnt), None, None, None,
                                               None))
        m = cnt.value
        id0 = np.empty(m, np.int32)
        id1 = np.empty(m, np.int32)
        dl = np.empty(m)
        f = np.empty((m, 3)) if forces else None
        self._check(lib.gdem_download_contacts(self._h, m, ctypes.byref(cnt), _ip(id0), _ip(id1),
                                               _dp(dl), _dp(f)))
        return (id0, id1, dl, f) if forces else (id0, id1, dl)

    def download_history(self):
        """The contact memory of the last force evaluation (both views of a
        pair): owner and partner IDs (a wall k as -(k + 2)), kdelta, previous
        normal and spring torque (m, 3) each."""
        lib = library()
        cnt = ctypes.c_int64(0)
        self._check(lib.gdem_download_history(self._h, 0, ctypes.byref(cnt), None, None, None,
                                              None, None))
        m = cnt.value
        own = np.empty(m, np.int32)
        par = np.empty(m, np.int32)
        kd, pn, sp = np.empty((m, 3)), np.empty((m, 3)), np.empty((m, 3))
        self._check(lib.gdem_download_history(self._h, m, ctypes.byref(cnt), _ip(own), _ip(par),
                                              _dp(kd), _dp(pn), _dp(sp)))
        return {"owner": own, "partner": par, "kdelta": kd, "prevn": pn, "spring": sp}

    def grid(self, k=0):
        nb = np.empty(3, np.int32)
        edge = np.empty(3)
        org = np.empty(3)
        self._check(library().gdem_grid(self._h, k, _ip(nb), _dp(edge), _dp(org)))
        return nb, edge, org

    def status(self, reset=False) -> int:
        bits = ctypes.c_int(0)
        self._check(library().gdem_status(self._h, ctypes.byref(bits), 1 if reset else 0))
        return bits.value

    def use_graphs(self, on=True):
        self._check(library().gdem_use_graphs(self._h, 1 if on else 0))

    def set_contact_memory_pruning(self, prune=True):
        """Whether the memory of ended contacts is dropped (the plain step,
        the default) or kept (GrainsCoupledWithFluid's step); before the
        particles are uploaded or read."""
        self._check(library().gdem_set_contact_memory_pruning(self._h, 1 if prune else 0))

    @property
    def last_step_ms(self) -> float:
        return library().gdem_last_step_ms(self._h)

    # ------------------------------------------------------------- stepping
    def set_tuning(self, skin_factor=None, blocks_per_sm=None):
        """Pair-list skin (multiple of rmax) and force-kernel blocks per
        multiprocessor, before do_before_time_stepping; None keeps the default."""
        self._check(library().gdem_set_tuning(
            self._h, -1.0 if skin_factor is None else float(skin_factor),
            0 if blocks_per_sm is None else int(blocks_per_sm)))

    def autotune(self, trial_steps=50):
        """Times copies of the uploaded system over the candidate launch
        settings and applies the fastest; returns
        {"skin_factor", "blocks_per_sm", "ms_per_step"}."""
        sf = ctypes.c_double(0.0)
        bps = ctypes.c_int(0)
        ms = ctypes.c_double(0.0)
        self._check(library().gdem_autotune(self._h, int(trial_steps), ctypes.byref(sf),
                                            ctypes.byref(bps), ctypes.byref(ms)))
        return {"skin_factor": sf.value, "blocks_per_sm": bps.value, "ms_per_step": ms.value}

    def do_before_time_stepping(self):
        """Leapfrog start: forces at t0, zeroed cumulative contact memory."""
        self._check(library().gdem_init(self._h))

    def step(self, nsteps=1):
        self._check(library().gdem_step(self._h, int(nsteps)))

    def Simulation(self, nsteps, raise_on_error=True):
        """Runs nsteps leapfrog steps (Grains::Simulation) and raises the
        reference's exception types on a status bit."""
        self.step(nsteps)
        st = self.status()
        if raise_on_error and st:
            if st & ST_CONTACT_OVERLAP:
                raise ContactError(f"max overlap exceeded (status {st:#x})")
            if st & ST_MOTION:
                raise MotionError(f"motion over one step exceeds the crust (status {st:#x})")
            if st & ST_OUT_OF_GRID:
                raise OutOfGridError(f"particle outside the linked cell (status {st:#x})")
            raise SimulationError(f"simulation status {st:#x}")
        return st
