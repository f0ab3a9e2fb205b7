"""gdem_speed_stats_static, the entry point that allocates nothing, through
the C ABI.

Who needs it: a caller that cannot allocate device memory at the point where
it wants the particles' speed statistics -- a fluid solver that has reserved
the rest of the GPU's memory for its own fields, or code running while a
stream is being captured -- and that holds the velocities in its own device
buffer.  The entry point reduces them with the library's fixed scratch array.

Checked here against gdem_velocity_stats (the handle path) on the same
velocities: the maximum must agree exactly, the mean to 1e-12 relative (the
two reductions sum in different orders: cell order on the handle, particle-ID
order here), on two calls in a row (the scratch keeps the previous call's
contents and needs no reset).  Also: several calls leave the device's free
memory unchanged, sizes above the fixed capacity are refused, and in a fresh
process the entry point still gives the right answer after cudaDeviceReset
has replaced the device's context (the scratch address is looked up again).
"""
import ctypes
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

from pacific_b200 import FP64, Grains, scenarios

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _static_stats(lib, v_dev, n, out_dev):
    fn = lib.gdem_speed_stats_static
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn(ctypes.c_void_p(v_dev), n, ctypes.c_void_p(out_dev), None)


def test_speed_stats_static_matches_handle(tmp_path, lib):
    import torch
    sc = scenarios.periodic_gas(n_fcc=20, seed=91)
    xml = str(sc.write_xml(tmp_path / "gas.xml"))
    g = Grains(xml, FP64)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    vmax, vmean = g.velocity_stats()
    g.close()

    v = torch.from_numpy(np.ascontiguousarray(sc.v, dtype=np.float64)).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        assert _static_stats(lib, v.data_ptr(), sc.n, out.data_ptr()) == 0
        torch.cuda.synchronize()
        smax, smean = out.cpu().tolist()
        assert smax == vmax
        assert abs(smean - vmean) <= 1e-12 * vmean


def test_speed_stats_static_allocates_nothing(lib):
    """After the first call (which looks up the scratch address), further
    calls change neither the device's free memory (cudaMemGetInfo) nor
    torch's reserved pool."""
    import torch
    rng = np.random.default_rng(7)
    v = torch.from_numpy(rng.normal(0.0, 0.1, (200_000, 3))).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _static_stats(lib, v.data_ptr(), 200_000, out.data_ptr()) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(5):
        assert _static_stats(lib, v.data_ptr(), 200_000, out.data_ptr()) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_reserved() == reserved0
    vh = v.cpu().numpy()
    s = np.sqrt(vh[:, 0] * vh[:, 0] + vh[:, 1] * vh[:, 1] + vh[:, 2] * vh[:, 2])
    assert out[0].item() == s.max()


def test_speed_stats_static_rejects_oversize(lib):
    import torch
    v = torch.zeros(3, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _static_stats(lib, v.data_ptr(), 1_048_577, out.data_ptr()) == -1
    assert b"capacity" in lib.gdem_last_error()


_RESET_SCRIPT = textwrap.dedent("""
    import ctypes, sys
    import numpy as np
    lib = ctypes.CDLL(sys.argv[1])
    rt = ctypes.CDLL("libcudart.so.12")   # the runtime the library itself loaded
    lib.gdem_speed_stats_static.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_void_p]
    n = 5000
    v = np.random.default_rng(3).normal(0.0, 0.2, (n, 3))
    s = np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])

    def once():
        dv, dout = ctypes.c_void_p(), ctypes.c_void_p()
        assert rt.cudaMalloc(ctypes.byref(dv), ctypes.c_size_t(v.nbytes)) == 0
        assert rt.cudaMalloc(ctypes.byref(dout), ctypes.c_size_t(16)) == 0
        assert rt.cudaMemcpy(dv, v.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(v.nbytes), 1) == 0
        assert lib.gdem_speed_stats_static(dv, n, dout, None) == 0
        out = np.zeros(2)
        assert rt.cudaMemcpy(out.ctypes.data_as(ctypes.c_void_p), dout, ctypes.c_size_t(16), 2) == 0
        assert rt.cudaDeviceSynchronize() == 0
        assert out[0] == s.max(), (out, s.max())
        assert abs(out[1] - s.mean()) <= 1e-12 * s.mean(), (out, s.mean())
        rt.cudaFree(dv)
        rt.cudaFree(dout)

    once()
    assert rt.cudaDeviceReset() == 0   # ends this process's context on the device
    once()
    print("reset ok")
""")


def test_speed_stats_static_after_device_reset(lib, tmp_path):
    """In a fresh process (no torch): a call, cudaDeviceReset, another call."""
    script = tmp_path / "reset_check.py"
    script.write_text(_RESET_SCRIPT)
    so = ROOT / "pacific_b200" / "libgrains_b200.so"
    r = subprocess.run([sys.executable, str(script), str(so)], capture_output=True, text=True,
                       timeout=300, env=dict(os.environ))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "reset ok" in r.stdout
