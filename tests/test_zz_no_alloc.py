"""gdem_speed_stats_static (the allocation-free entry point) against
gdem_velocity_stats on the same velocities, through the C ABI.

Both compute max |v| and mean |v|; max must agree exactly, the mean to 1e-12
relative (the two reductions sum in different orders: cell order on the
handle, particle-ID order here).  Two calls in a row must both agree (the
scratch needs no reset between calls)."""
import ctypes

import numpy as np
import pytest

from pacific_b200 import FP64, Grains, scenarios

pytestmark = pytest.mark.gpu


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


def test_speed_stats_static_rejects_oversize(lib):
    import torch
    v = torch.zeros(3, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _static_stats(lib, v.data_ptr(), 1_048_577, out.data_ptr()) == -1
    assert b"capacity" in lib.gdem_last_error()
