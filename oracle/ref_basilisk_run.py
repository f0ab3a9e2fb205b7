"""TEST INFRASTRUCTURE: the reference's Basilisk coupling interface
(oracle/_ref/libgrains_ref_basilisk.so, built by oracle/build_ref.sh from
GRAINS_V1/Grains/InterfaceCBasilisk/src unmodified over the reference
objects) driven through its C ABI, in a process of its own (the interface
keeps its application in a file-static pointer and the reference its
configuration in static members).

    python -m oracle.ref_basilisk_run <lib.so> <xml> <rho_f> <dt_fluid> <rows.npy> <out.json>

runs Init_Grains(xml, rho_f, restart = false, fluid-corrected acceleration
= true), Simu_Grains(dt_fluid), GrainsToBasilisk, UpdateVelocityGrains(rows),
Simu_Grains(dt_fluid), GrainsToBasilisk, NumberOfRigidBodiesInBasilisk, and
saves the two streams and the counts.  The same driver runs the library of
this repository (libgrains_b200_basilisk.so) for the comparison in
tests/test_coupling.py.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
REF_LIB = Path(__file__).resolve().parent / "_ref" / "libgrains_ref_basilisk.so"


def _stream(lib):
    size = ctypes.c_int(0)
    ptr = lib.GrainsToBasilisk(ctypes.byref(size))
    return ctypes.string_at(ptr).decode()


def main(so, xml, rho, dt_fluid, rows_path, out):
    os.chdir(Path(xml).parent)
    lib = ctypes.CDLL(str(so))
    lib.Init_Grains.argtypes = [ctypes.c_char_p, ctypes.c_double, ctypes.c_bool, ctypes.c_bool]
    lib.Simu_Grains.argtypes = [ctypes.c_double]
    lib.GrainsToBasilisk.argtypes = [ctypes.POINTER(ctypes.c_int)]
    lib.GrainsToBasilisk.restype = ctypes.c_void_p
    lib.UpdateVelocityGrains.argtypes = [ctypes.POINTER(ctypes.POINTER(ctypes.c_double)),
                                         ctypes.c_int]
    lib.NumberOfRigidBodiesInBasilisk.argtypes = [ctypes.POINTER(ctypes.c_size_t)] * 2
    lib.Init_Grains(str(xml).encode(), rho, False, True)
    lib.Simu_Grains(dt_fluid)
    s1 = _stream(lib)
    rows = np.ascontiguousarray(np.load(rows_path), dtype=np.float64)
    arr = (ctypes.POINTER(ctypes.c_double) * len(rows))(
        *[rows[i].ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for i in range(len(rows))])
    lib.UpdateVelocityGrains(arr, len(rows))
    lib.Simu_Grains(dt_fluid)
    s2 = _stream(lib)
    npart, nobs = ctypes.c_size_t(0), ctypes.c_size_t(0)
    lib.NumberOfRigidBodiesInBasilisk(ctypes.byref(npart), ctypes.byref(nobs))
    Path(out).write_text(json.dumps({"streams": [s1, s2], "particles": npart.value,
                                     "obstacles": nobs.value}))


def run(so, xml, rho, dt_fluid, rows, timeout=600):
    """Runs the driver above on library `so` in a subprocess; returns its
    results (streams after the first and the second fluid step)."""
    xml = Path(xml)
    rows_path = xml.parent / f"rows_{Path(so).stem}.npy"
    out = xml.parent / f"streams_{Path(so).stem}.json"
    np.save(rows_path, np.asarray(rows, dtype=np.float64))
    env = dict(os.environ, GRAINS_HOME=str(xml.parent))
    r = subprocess.run([sys.executable, "-m", "oracle.ref_basilisk_run", str(so), str(xml),
                        repr(float(rho)), repr(float(dt_fluid)), str(rows_path), str(out)],
                       cwd=str(ROOT), capture_output=True, text=True, timeout=timeout, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"Basilisk run of {so} failed: {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return json.loads(out.read_text())


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], float(sys.argv[3]), float(sys.argv[4]), sys.argv[5],
         sys.argv[6])
