"""The C-ABI library loads and exports every symbol include/kf.h declares (CPU only)."""
import ctypes as C
import os
import re

import pytest

from oglfusionkinectv2_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "kf.h")).read()
    return sorted(set(re.findall(r"^KF_API\s+[\w\s\*]+?\b(kf_\w+)\s*\(", text, re.M)))


def test_header_declares_the_api():
    names = declared_symbols()
    assert len(names) >= 40
    assert set(names) == set(L.SIGNATURES), set(names) ^ set(L.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    L.load()  # binds every signature


def test_host_only_entry_points():
    lib = L.load()
    assert lib.kf_abi_version() == 2
    c = L.kf_config()
    assert lib.kf_config_default(C.byref(c)) == L.KF_OK
    # gFusionConfig() defaults (gFusion.h:56-69)
    assert (c.nx, c.mu, c.max_weight, c.near_plane, c.far_plane) == (256, pytest.approx(0.05), 100.0,
                                                                     pytest.approx(0.1), 3.0)
    assert list(c.iterations) == [5, 5, 5] and c.quirks == L.KF_QUIRKS_DEFAULT
    assert lib.kf_status_string(L.KF_ERR_TIMEOUT) == b"device wait timed out"
    b = C.c_uint64()
    i = L.kf_intrinsics(365, 365, 256, 212, 512, 424)
    assert lib.kf_session_device_bytes(C.byref(c), C.byref(i), C.byref(b)) == L.KF_OK
    assert b.value > 256 ** 3 * 8
    bad = L.kf_config.from_buffer_copy(c)
    bad.mu = 0
    assert lib.kf_session_device_bytes(C.byref(bad), C.byref(i), C.byref(b)) == L.KF_ERR_INVALID_ARGUMENT


def test_quirk_presets_match_header():
    text = open(os.path.join(ROOT, "include", "kf.h")).read()
    for name in ["KF_Q1_LAST_GROUP_ONLY", "KF_Q3_DOWN_FROM_LEFT", "KF_Q4_SAME_PIXEL", "KF_Q6_SDF_D2_TWICE",
                 "KF_Q7_SDF_LAST_COLUMN", "KF_Q8_NARROW_BAND", "KF_Q13_MC_FIRST_SEVEN",
                 "KF_Q15_MC_BORDER_SKIP", "KF_Q18_STL_COUNT_X4", "KF_Q19_EIG_TRANSLATION",
                 "KF_Q23_SDF_XY_OFFSET", "KF_Q24_MC_SHADER_UNITS"]:
        m = re.search(r"#define " + name + r" \(1u << (\d+)\)", text)
        assert m and getattr(L, name) == 1 << int(m.group(1)), name


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = L.load()
    c = L.kf_config()
    lib.kf_config_default(C.byref(c))
    c.nx = c.ny = c.nz = 32
    i = L.kf_intrinsics(365, 365, 256, 212, 512, 424)
    h = C.c_void_p()
    assert lib.kf_create(C.byref(c), C.byref(i), C.byref(h)) == L.KF_ERR_NO_DEVICE
    from oglfusionkinectv2_b200 import GFusion
    with pytest.raises(L.KfError):
        GFusion()


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors of the ABI structs have the C compiler's sizes and offsets."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    structs = {"kf_config": L.kf_config, "kf_intrinsics": L.kf_intrinsics, "kf_volume_view": L.kf_volume_view,
               "kf_server_config": L.ServerConfig, "kf_server_stats_t": L.ServerStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "kf.h"', "int main(void) {"]
    for name, py in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for name, py in structs.items():
        assert int(got[name]) == C.sizeof(py), name
        for f, _ in py._fields_:
            assert int(got[f"{name}.{f}"]) == getattr(py, f).offset, f"{name}.{f}"


def test_batch_and_server_without_device_fail_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = L.load()
    h = C.c_void_p()
    assert lib.kf_batch_create(4, C.byref(h)) == L.KF_ERR_NO_DEVICE
    assert lib.kf_batch_create(0, C.byref(h)) == L.KF_ERR_INVALID_ARGUMENT
    assert lib.kf_batch_create(L.KF_BATCH_MAX_SESSIONS + 1, C.byref(h)) == L.KF_ERR_INVALID_ARGUMENT
    cfg = L.ServerConfig()
    assert lib.kf_server_config_default(C.byref(cfg)) == L.KF_OK
    assert (cfg.max_sessions, cfg.max_batch, cfg.storage, cfg.jtj) == (128, 64, L.KF_STORAGE_F16U16,
                                                                      L.KF_JTJ_SPLIT_BF16)
    assert lib.kf_server_create(C.byref(cfg), C.byref(h)) != L.KF_OK
    t0 = lib.kf_server_now()
    assert lib.kf_server_now() >= t0


@pytest.mark.parametrize("field,value", [
    ("nx", 3), ("ny", 4097), ("nz", 0),
    ("mu", 0.0), ("mu", float("nan")), ("dim_x", -1.0), ("max_weight", 0.0),
    ("near_plane", 3.0), ("storage", 7), ("jtj", 2), ("tracking", 5),
])
def test_invalid_configs_are_rejected(field, value):
    """Every bad configuration is refused with KF_ERR_INVALID_ARGUMENT before any device work
    (checked through kf_session_device_bytes, which needs no device)."""
    lib = L.load()
    c = L.kf_config()
    lib.kf_config_default(C.byref(c))
    setattr(c, field, value)
    i = L.kf_intrinsics(365, 365, 256, 212, 512, 424)
    b = C.c_uint64()
    assert lib.kf_session_device_bytes(C.byref(c), C.byref(i), C.byref(b)) == L.KF_ERR_INVALID_ARGUMENT


def test_volume_and_image_limits():
    lib = L.load()
    c = L.kf_config()
    lib.kf_config_default(C.byref(c))
    i = L.kf_intrinsics(365, 365, 256, 212, 512, 424)
    b = C.c_uint64()
    # 32-bit plane offsets: fewer than 2^31 voxels
    c.nx, c.ny, c.nz = 2048, 1024, 1024
    assert lib.kf_session_device_bytes(C.byref(c), C.byref(i), C.byref(b)) == L.KF_ERR_INVALID_ARGUMENT
    c.nx, c.ny, c.nz = 1024, 1024, 1024
    assert lib.kf_session_device_bytes(C.byref(c), C.byref(i), C.byref(b)) == L.KF_OK
    # 16-bit weights cannot hold a larger maximum weight
    c.storage, c.max_weight = L.KF_STORAGE_RG16I, 40000.0
    assert lib.kf_session_device_bytes(C.byref(c), C.byref(i), C.byref(b)) == L.KF_ERR_INVALID_ARGUMENT
    c.storage, c.max_weight = L.KF_STORAGE_F32F32, 100.0
    # three exact mip halvings
    for w, h in ((510, 424), (512, 8), (8200, 424)):
        bad = L.kf_intrinsics(365, 365, 256, 212, w, h)
        assert lib.kf_session_device_bytes(C.byref(c), C.byref(bad), C.byref(b)) == L.KF_ERR_INVALID_ARGUMENT
    iterations_bad = L.kf_config.from_buffer_copy(c)
    iterations_bad.iterations[1] = -1
    assert lib.kf_session_device_bytes(C.byref(iterations_bad), C.byref(i), C.byref(b)) == L.KF_ERR_INVALID_ARGUMENT
