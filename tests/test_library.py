"""The C-ABI library: it loads without a GPU, exports every symbol include/kf_api.h declares,
and its host-only entry points (defaults, validation, footprint) behave.  CPU only."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "kf_api.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:kf_status|int|void|double|const\s+char\s*\*)\s*\**\s*(kf_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_parses():
    names = declared_functions()
    assert len(names) >= 50
    assert "kf_process_frame" in names and "kf_server_step" in names


def test_every_declared_symbol_is_exported(kf):
    from kfb200 import _lib
    so = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(so, n)]
    assert not missing, missing
    # and the Python mirror binds every one of them with a signature
    unbound = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not unbound, unbound


def test_api_version(kf):
    assert kf.lib.kf_api_version() == 1


def test_default_config_is_the_reference_main(kf):
    c = kf.default_config()
    # project/src/main.cpp:11-59 (dataset configuration) and the compile-time constants
    assert (c.width, c.height) == (640, 480)
    assert c.fx == 525.0 and c.fy == 525.0 and c.cx == 319.5 and c.cy == 239.5
    assert c.depth_scale == np.float32(1.0 / 5000.0)
    assert list(c.iters) == [10, 5, 3] and c.levels == 3
    assert abs(c.dist_thresh - 0.4) < 1e-7 and abs(c.angle_thresh - 4 * math.pi / 18) < 1e-6
    assert abs(c.stop_angle - math.radians(0.1)) < 1e-9 and abs(c.stop_dist - 0.01) < 1e-9
    assert c.bilateral_sigma_s == 4.0 and c.bilateral_sigma_r == 0.25 and c.bilateral_radius == 3
    assert c.volume_n == 256 and c.volume_width == 8.0 and abs(c.mu - 3 * 8 / 255) < 1e-6
    assert c.min_depth == pytest.approx(0.4) and c.max_depth == 6.0
    assert c.step_large == pytest.approx(1.99) and c.step_small == pytest.approx(0.1)
    assert c.keep_on_miss == 1 and c.max_weight == 0.0 and c.tsdf_format == kf.KF_TSDF_F32F32
    assert list(c.initial_pose) == [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]
    # the visualization grid: 512^3 over 5 m, mu = 2 voxels (project/src/main.cpp:25-26,
    # project/src/kinect_fusion.cpp:19)
    assert c.vis_volume_n == 512 and c.vis_volume_width == 5.0 and abs(c.vis_mu - 2 * 5 / 511) < 1e-7


def test_visualization_volume_counts_in_the_footprint(kf):
    n = ctypes.c_size_t()
    c = kf.config_small()
    assert c.vis_volume_n == 0
    kf.lib.kf_session_footprint(ctypes.byref(c), ctypes.byref(n))
    base = n.value
    cv = kf.config_small(vis_volume_n=256, vis_volume_width=5.0, vis_mu=2 * 5 / 255)
    kf.lib.kf_session_footprint(ctypes.byref(cv), ctypes.byref(n))
    assert n.value - base >= 256 ** 3 * 8
    bad = kf.config_small(vis_volume_n=100, vis_volume_width=5.0, vis_mu=0.04)   # not a multiple of 8
    assert kf.lib.kf_session_footprint(ctypes.byref(bad), ctypes.byref(n)) == kf.KF_ERR_ARG


def test_status_strings(kf):
    for s in range(9):
        assert kf.lib.kf_status_string(s)


def test_footprint(kf):
    c = kf.config_full()
    n = ctypes.c_size_t()
    assert kf.lib.kf_session_footprint(ctypes.byref(c), ctypes.byref(n)) == kf.KF_OK
    assert n.value > 512 ** 3 * 8
    c16 = kf.config_full(tsdf_format=kf.KF_TSDF_F16U16)
    n16 = ctypes.c_size_t()
    kf.lib.kf_session_footprint(ctypes.byref(c16), ctypes.byref(n16))
    assert n.value - n16.value == 512 ** 3 * 4


@pytest.mark.parametrize("field,value,status", [
    ("width", 322, 2),          # not divisible by 2^(levels-1): KF_ERR_SHAPE
    ("levels", 4, 1),
    ("volume_n", 100, 1),       # volume edge must be a multiple of 8
    ("bilateral_radius", 9, 1),
    ("mu", 0.0, 1),
    ("tsdf_format", 7, 1),
])
def test_invalid_configs_rejected_before_any_device_work(kf, field, value, status):
    c = kf.config_small(**{field: value})
    h = ctypes.c_void_p()
    assert kf.lib.kf_session_create(ctypes.byref(c), ctypes.byref(h)) == status
    n = ctypes.c_size_t()
    assert kf.lib.kf_session_footprint(ctypes.byref(c), ctypes.byref(n)) == status


def test_too_many_icp_iterations_rejected(kf):
    c = kf.config_small(iters=(30, 30, 30))
    n = ctypes.c_size_t()
    assert kf.lib.kf_session_footprint(ctypes.byref(c), ctypes.byref(n)) == kf.KF_ERR_ARG


def test_null_arguments(kf):
    assert kf.lib.kf_session_create(None, None) == kf.KF_ERR_ARG
    assert kf.lib.kf_process_frame(None, None, 0, None, None) == kf.KF_ERR_ARG
    assert kf.lib.kf_pose_error(None, None, None) == kf.KF_ERR_ARG


def test_pose_error_host(kf, orc):
    import numpy as np
    a = np.eye(4, dtype=np.float32)
    b = np.eye(4, dtype=np.float32)
    b[:3, 3] = [0.3, 0.0, 0.4]
    c = np.cos(0.01); s = np.sin(0.01)
    b[:3, :3] = [[c, -s, 0], [s, c, 0], [0, 0, 1]]
    got = kf.poseError(a, b)
    want = orc.pose_error(a, b)
    assert abs(got[0] - want[0]) < 1e-7 and abs(got[1] - 0.5) < 1e-6


@pytest.mark.parametrize("level", [0, 1, 2])
def test_level_inverse_intrinsics(kf, level):
    """The Python mirror of the library's K_l^-1 (float32 adjugate over determinant) inverts
    K_l to float rounding, for the full-size and small configurations."""
    for cfg in (kf.config_full(), kf.config_small()):
        k = kf.level_intrinsics(cfg, level).astype(np.float64)
        ik = kf.level_inverse_intrinsics(cfg, level)
        assert ik.dtype == np.float32
        np.testing.assert_allclose(ik.astype(np.float64) @ k, np.eye(3), atol=2e-6)
