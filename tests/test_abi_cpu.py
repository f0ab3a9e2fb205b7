"""CPU-side checks of the C ABI library: it loads, exports every entry point
that include/grains_b200.h declares, and refuses to run without a device."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(gdem_[a-z0-9_]+)\s*\(", txt))
    return names


def test_exports_every_declared_symbol(lib):
    declared = _declared()
    assert "gdem_step" in declared and len(declared) >= 15
    for name in sorted(declared):
        assert hasattr(lib, name), name


def test_create_without_device_fails_cleanly(lib, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from pacific_b200 import Grains, GrainsError, scenarios
    p = scenarios.settling_box(n=10).write_xml(tmp_path / "s.xml")
    with pytest.raises(GrainsError, match="CUDA|device"):
        Grains(p)


def test_bad_xml_is_rejected_before_device(lib, tmp_path):
    """XML errors surface as GDEM_ERR_INVALID / GDEM_ERR_CUDA, never a crash."""
    from pacific_b200 import Grains, GrainsError
    p = tmp_path / "bad.xml"
    p.write_text("<Grains3D><Construction><LinkedCell MX='1'/></Construction>")
    with pytest.raises(GrainsError):
        Grains(p)


# InterfaceGrains3DBasilisk.h (GRAINS_V1/Grains/InterfaceCBasilisk/include)
BASILISK_SYMBOLS = ("Init_Grains", "Simu_Grains", "GrainsToBasilisk", "SetInitialTime",
                    "SaveResults_Grains", "checkParaviewPostProcessing_Grains",
                    "UpdateVelocityGrains", "SetInitialCycleNumber",
                    "NumberOfRigidBodiesInBasilisk")


def test_basilisk_library_exports_the_coupling_abi(lib):
    """libgrains_b200_basilisk.so loads over libgrains_b200.so and exports the
    reference's Basilisk coupling entry points, so a DLMFD build can link it
    in place of the reference's interface library."""
    b = ctypes.CDLL(str(ROOT / "pacific_b200" / "libgrains_b200_basilisk.so"))
    for name in BASILISK_SYMBOLS:
        assert hasattr(b, name), name
    # with no system, the rigid-body count is zero (no crash without a device)
    n, m = ctypes.c_size_t(7), ctypes.c_size_t(7)
    b.NumberOfRigidBodiesInBasilisk(ctypes.byref(n), ctypes.byref(m))
    assert n.value == 0 and m.value == 0


def test_output_entry_points_reject_bad_arguments(lib, tmp_path):
    """The RawData writer, the velocity line and the reload readers check
    their arguments before touching a device: a null handle or a missing
    file is GDEM_ERR_INVALID with a message, never a crash."""
    import ctypes
    lib.gdem_rawdata_start.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_double]
    lib.gdem_write_velocity_max_mean.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                                 ctypes.c_double]
    lib.gdem_rawdata_write.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.gdem_rawdata_end.argtypes = [ctypes.c_void_p]
    lib.gdem_read_reload_particles_hybrid.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    lib.gdem_last_error.restype = ctypes.c_char_p
    root = str(tmp_path / "out").encode()
    assert lib.gdem_rawdata_start(None, root, 0, 0, 0.0) == -1
    assert lib.gdem_write_velocity_max_mean(None, root, 0, 0.0) == -1
    assert lib.gdem_rawdata_write(None, 0.0) == -1
    assert b"gdem_rawdata_start" in lib.gdem_last_error()
    assert lib.gdem_rawdata_end(None) == 0            # nothing open: nothing to close
    assert lib.gdem_read_reload_particles_hybrid(None, root) == -1
    assert not list(tmp_path.iterdir())
