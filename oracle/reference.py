"""ctypes front end of the Grains3D reference built by oracle/build_ref.sh.

TEST INFRASTRUCTURE: available only where the reference tree was present at
build time (oracle/_ref/ is not committed).  Used to pin the CPU
restatement and to generate the golden vectors in tests/golden/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libgrains_ref.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def tree_present() -> bool:
    """The reference's sources are where build_ref.sh looks for them."""
    root = Path(os.environ.get("GRAINS_REFERENCE", "/root/reference"))
    return (root / "GRAINS_V1" / "Grains").is_dir()


def build() -> Path:
    subprocess.run(["sh", str(HERE / "build_ref.sh")], check=True)
    return LIB


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(LIB))
        V = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        I = ctypes.POINTER(ctypes.c_int)
        lib.ref_create.argtypes = [ctypes.c_char_p]
        lib.ref_create.restype = V
        lib.ref_set_particles.argtypes = [V, ctypes.c_int, I, D, D, D, D]
        lib.ref_set_particles.restype = ctypes.c_int
        lib.ref_load_particles.argtypes = [V, ctypes.c_char_p, ctypes.c_int]
        lib.ref_load_particles.restype = ctypes.c_int
        lib.ref_init.argtypes = [V]
        lib.ref_init.restype = ctypes.c_int
        lib.ref_step.argtypes = [V, ctypes.c_int]
        lib.ref_step.restype = ctypes.c_int
        lib.ref_get_state.argtypes = [V, D, D, D, D, D, D]
        lib.ref_get_cells.argtypes = [V, I]
        lib.ref_get_basis.argtypes = [V, D]
        lib.ref_num_history.argtypes = [V]
        lib.ref_num_history.restype = ctypes.c_int
        lib.ref_get_history.argtypes = [V, I, I, D, D, D]
        lib.ref_write_particles.argtypes = [V, ctypes.c_char_p]
        lib.ref_write_particles.restype = ctypes.c_int
        lib.ref_write_particles_hybrid.argtypes = [V, ctypes.c_char_p]
        lib.ref_write_particles_hybrid.restype = ctypes.c_int
        lib.ref_rawdata_start.argtypes = [V, ctypes.c_char_p, ctypes.c_double]
        lib.ref_rawdata_start.restype = ctypes.c_int
        lib.ref_rawdata_write.argtypes = [V, ctypes.c_double]
        lib.ref_rawdata_write.restype = ctypes.c_int
        lib.ref_rawdata_end.argtypes = [V]
        lib.ref_velocity_max_mean.argtypes = [V, D, D]
        lib.ref_contact_features.argtypes = [V, D]
        lib.ref_destroy.argtypes = [V]
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Reference:
    """The unmodified Grains3D serial step driven from a given state."""

    def __init__(self, xml_path, quiet=True):
        lib = _load()
        self._h = lib.ref_create(os.fsencode(str(xml_path)))
        if not self._h:
            raise RuntimeError(f"reference could not read {xml_path}")
        self.n = 0

    def set_particles(self, type, x, v, w, q):
        n = len(type)
        self._t = np.ascontiguousarray(type, np.int32)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (x, v, w, q)]
        rc = _load().ref_set_particles(self._h, n, _ip(self._t), *[_dp(a) for a in arrs])
        self.n = n
        return rc

    def load_particles(self, stem, n):
        """Reads <stem>_Particles.result (a Format2024 particle file) through
        the reference's own reload path; stem must hold no '.'."""
        if "." in str(stem):
            raise ValueError("the reference cuts the reload name at its first '.'")
        self.n = n
        return _load().ref_load_particles(self._h, os.fsencode(str(stem) + ".reload"), n)

    def init(self):
        return _load().ref_init(self._h)

    def step(self, nsteps=1):
        return _load().ref_step(self._h, nsteps)

    def state(self):
        n = self.n
        out = {k: np.empty((n, 3)) for k in ("x", "v", "w", "F", "T")}
        out["q"] = np.empty((n, 4))
        _load().ref_get_state(self._h, _dp(out["x"]), _dp(out["v"]), _dp(out["w"]),
                              _dp(out["q"]), _dp(out["F"]), _dp(out["T"]))
        return out

    def basis(self):
        b = np.empty((self.n, 9))
        _load().ref_get_basis(self._h, _dp(b))
        return b

    def cells(self):
        ijk = np.empty((self.n, 3), np.int32)
        _load().ref_get_cells(self._h, _ip(ijk))
        return ijk

    def write_particles(self, path):
        """The particle file of a Format2024 reload, by Particle::write2014."""
        return _load().ref_write_particles(self._h, os.fsencode(str(path)))

    def write_particles_hybrid(self, path):
        """The same particle file in the hybrid binary form (Particle::write2014_binary)."""
        return _load().ref_write_particles_hybrid(self._h, os.fsencode(str(path)))

    def rawdata_start(self, root, binary, time):
        """Registers the reference's RawDataPostProcessingWriter with output
        root `root` and writes its first output time (PostProcessing_start)."""
        root = Path(root)
        spec = root.parent / (root.name + "_writer.xml")
        mode = "Binary" if binary else "Text"
        spec.write_text(f'<RawData Name="{root}" WritingMode="{mode}"/>\n')
        return _load().ref_rawdata_start(self._h, os.fsencode(str(spec)), time)

    def rawdata_write(self, time):
        return _load().ref_rawdata_write(self._h, time)

    def rawdata_end(self):
        _load().ref_rawdata_end(self._h)

    def velocity_max_mean(self):
        a, b = np.zeros(1), np.zeros(1)
        _load().ref_velocity_max_mean(self._h, _dp(a), _dp(b))
        return float(a[0]), float(b[0])

    def contact_features(self):
        """(overlap max, overlap mean, time of the max, mean GJK iterations)
        over every evaluation of this process."""
        out = np.zeros(4)
        _load().ref_contact_features(self._h, _dp(out))
        return out

    def history(self):
        lib = _load()
        m = lib.ref_num_history(self._h)
        own = np.empty(m, np.int32)
        par = np.empty(m, np.int32)
        kd = np.empty((m, 3))
        pn = np.empty((m, 3))
        sp = np.empty((m, 3))
        lib.ref_get_history(self._h, _ip(own), _ip(par), _dp(kd), _dp(pn), _dp(sp))
        return own, par, kd, pn, sp
