"""Host checks of the build of the reference's own pipeline (oracle/Makefile, oracle/refshim,
oracle/ref_harness.cpp, oracle/refpipe.py), no GPU:
  - the glm subset the reference's sources compile against computes what glm's documented
    functions compute (inverse, transpose, orientate3 = Ry(yaw) Rx(pitch) Rz(roll), normalize,
    cross, column-major products), checked against numpy;
  - the harness library, where it is built, exports every entry point refpipe binds;
  - its host-only entries pin the library's host code to the reference's own functions:
    the level intrinsics and their inverse to Sensor, kf_pose_error to poseError, and the
    TUM reader (kf_tum_*) to RgbdDataset;
  - refpipe.matching_config gives the reference's hard-coded constants."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import refpipe

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "refshim")

_SRC = r"""
#include <glm/glm.hpp>
#include <glm/gtx/euler_angles.hpp>
extern "C" {
void inv3(const float* a, float* o) {   // a, o column-major
    glm::mat3 m; for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) m[c][r] = a[c * 3 + r];
    glm::mat3 i = glm::inverse(m); for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) o[c * 3 + r] = i[c][r];
}
void inv4(const float* a, float* o) {
    glm::mat4 m; for (int c = 0; c < 4; ++c) for (int r = 0; r < 4; ++r) m[c][r] = a[c * 4 + r];
    glm::mat4 i = glm::inverse(m); for (int c = 0; c < 4; ++c) for (int r = 0; r < 4; ++r) o[c * 4 + r] = i[c][r];
}
void orient(float x, float y, float z, float* o) {
    glm::mat3 m = glm::orientate3(glm::vec3(x, y, z));
    for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) o[c * 3 + r] = m[c][r];
}
void mulv(const float* a, const float* v, float* o) {
    glm::mat3 m; for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) m[c][r] = a[c * 3 + r];
    glm::mat4 m4(m); glm::vec4 w = m4 * glm::vec4(glm::vec3(v[0], v[1], v[2]), 1.0f);
    glm::vec3 x = glm::transpose(m) * glm::vec3(v[0], v[1], v[2]);
    glm::vec3 n = glm::normalize(glm::cross(glm::vec3(v[0], v[1], v[2]), glm::vec3(1.0f, 2.0f, 3.0f)));
    o[0] = w.x; o[1] = w.y; o[2] = w.z; o[3] = w.w; o[4] = x.x; o[5] = x.y; o[6] = x.z;
    o[7] = n.x; o[8] = n.y; o[9] = n.z; o[10] = glm::length(glm::vec3(v[0], v[1], v[2]));
}
}
"""


@pytest.fixture(scope="module")
def glmlib(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("glm")
    src, so = d / "g.cpp", d / "libg.so"
    src.write_text(_SRC)
    inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", SHIM, "-I", inc, str(src), "-o", str(so)],
                   check=True, capture_output=True)
    return ctypes.CDLL(str(so))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _cm(m):
    return np.ascontiguousarray(np.asarray(m, np.float32).T).ravel()


def _uncm(a, n):
    return a.reshape(n, n).T


def test_glm_inverse(glmlib):
    rng = np.random.default_rng(5)
    k = np.array([[525.0, 0, 319.5], [0, 525.0, 239.5], [0, 0, 1]], np.float32)
    for m3 in (k, rng.normal(size=(3, 3)).astype(np.float32) + 3 * np.eye(3, dtype=np.float32)):
        out = np.zeros(9, np.float32)
        glmlib.inv3(_p(_cm(m3)), _p(out))
        np.testing.assert_allclose(_uncm(out, 3), np.linalg.inv(m3.astype(np.float64)), rtol=1e-5, atol=1e-6)
    a = rng.normal(size=(3,))
    c, s = np.cos(a), np.sin(a)
    rx = np.array([[1, 0, 0], [0, c[0], -s[0]], [0, s[0], c[0]]])
    ry = np.array([[c[1], 0, s[1]], [0, 1, 0], [-s[1], 0, c[1]]])
    pose = np.eye(4)
    pose[:3, :3] = rx @ ry
    pose[:3, 3] = rng.normal(size=3)
    out = np.zeros(16, np.float32)
    glmlib.inv4(_p(_cm(pose)), _p(out))
    np.testing.assert_allclose(_uncm(out, 4), np.linalg.inv(pose), rtol=1e-5, atol=2e-6)


def test_glm_orientate3(glmlib):
    """orientate3(a) = yawPitchRoll(a.z, a.x, a.y) = Ry(a.z) Rx(a.x) Rz(a.y), the rotation the
    reference's ICP update builds (project/src/icp.cpp:82)."""
    x, y, z = 0.11, -0.23, 0.37
    out = np.zeros(9, np.float32)
    glmlib.orient(ctypes.c_float(x), ctypes.c_float(y), ctypes.c_float(z), _p(out))

    def rx(t):
        return np.array([[1, 0, 0], [0, np.cos(t), -np.sin(t)], [0, np.sin(t), np.cos(t)]])

    def ry(t):
        return np.array([[np.cos(t), 0, np.sin(t)], [0, 1, 0], [-np.sin(t), 0, np.cos(t)]])

    def rz(t):
        return np.array([[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]])
    np.testing.assert_allclose(_uncm(out, 3), ry(z) @ rx(x) @ rz(y), atol=1e-6)


def test_glm_products_and_geometry(glmlib):
    m = np.array([[1, 2, 3], [4, 5, 6], [7, 8, 10]], np.float32)
    v = np.array([0.5, -1.5, 2.0], np.float32)
    out = np.zeros(11, np.float32)
    glmlib.mulv(_p(_cm(m)), _p(v), _p(out))
    np.testing.assert_allclose(out[:3], m @ v, rtol=1e-6)
    assert out[3] == 1.0
    np.testing.assert_allclose(out[4:7], m.T @ v, rtol=1e-6)
    n = np.cross(v.astype(np.float64), [1, 2, 3])
    np.testing.assert_allclose(out[7:10], n / np.linalg.norm(n), rtol=1e-6)
    np.testing.assert_allclose(out[10], np.linalg.norm(v), rtol=1e-6)


def test_harness_exports_every_entry_point():
    if not refpipe.available():
        pytest.skip("the reference harness is built only where a reference checkout exists")
    lib = refpipe.lib()   # binds every name in refpipe._SIG, AttributeError when one is missing
    for name in refpipe._SIG:
        assert getattr(lib, name) is not None


def test_matching_config_has_the_reference_constants(kf):
    c = refpipe.matching_config(kf, volume_n=512, volume_width=3.0, depth_scale=1e-3)
    res = np.float32(3.0) / np.float32(511)
    assert np.float32(c.mu) == np.float32(np.float32(3.0) * res)
    assert refpipe.mue_scale_for(c) == pytest.approx(3.0, rel=1e-6)
    assert (c.width, c.height, c.levels) == (640, 480, 3)
    assert (c.fx, c.fy, c.cx, c.cy) == (525.0, 525.0, 319.5, 239.5)
    assert (c.bilateral_sigma_s, c.bilateral_sigma_r, c.bilateral_radius) == (4.0, 0.25, 3)
    assert list(c.iters)[:3] == [10, 5, 3]
    assert (c.min_depth, c.max_depth) == (np.float32(0.4), np.float32(6.0))


def test_pose_error_equals_the_reference_function(kf, orc):
    """kf_pose_error (library, host) and the oracle's pose error against the reference's own
    poseError (project/src/general_helper.cpp:11-21, compiled from its sources over the glm
    subset), bit for bit on random poses: rotations about random axes up to 0.5 rad and
    translations up to 2 m, identity and equal poses included."""
    if not refpipe.available():
        pytest.skip("the reference harness is built only where a reference checkout exists")
    rng = np.random.default_rng(17)

    def pose():
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        ang = rng.uniform(0.0, 0.5)
        k = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        m = np.eye(4)
        m[:3, :3] = np.eye(3) + np.sin(ang) * k + (1 - np.cos(ang)) * k @ k
        m[:3, 3] = rng.uniform(-2.0, 2.0, size=3)
        return m.astype(np.float32)

    pairs = [(np.eye(4, dtype=np.float32), np.eye(4, dtype=np.float32))]
    p = pose()
    pairs.append((p, p.copy()))
    pairs += [(pose(), pose()) for _ in range(200)]
    for a, b in pairs:
        want = refpipe.pose_error(a, b)
        assert tuple(np.float32(kf.poseError(a, b))) == tuple(np.float32(want))
        assert tuple(np.float32(orc.pose_error(a, b))) == tuple(np.float32(want))


def _write_tum(d, gt_t, trans, quats, depth_t):
    with open(os.path.join(d, "groundtruth.txt"), "w") as f:
        f.write("# ground truth trajectory\n# file: 'x.bag'\n# timestamp tx ty tz qx qy qz qw\n")
        for t, tr, q in zip(gt_t, trans, quats):
            f.write("%.4f %.4f %.4f %.4f %.4f %.4f %.4f %.4f\n" % (t, *tr, *q))
    with open(os.path.join(d, "depth.txt"), "w") as f:
        f.write("# depth maps\n# file: 'x.bag'\n# timestamp filename\n")
        for t in depth_t:
            f.write("%.6f depth/%.6f.png\n" % (t, t))


@pytest.mark.parametrize("case", ["regular", "edges_and_ties", "out_of_order"])
def test_tum_reader_equals_the_reference_reader(kf, case):
    """The library's TUM reader (kf_tum_*) against the reference's own RgbdDataset
    (project/src/rgbd_dataset.cpp:6-96, compiled from its sources): the same frame count, the
    same ground-truth pose for every depth frame, bit for bit (the nearest-timestamp search
    forward from the last match and the quaternion-to-matrix conversion), and the same initial
    pose inverse to float rounding (the reference inverts in float, the library in double).
    Cases: a regular 100 Hz trajectory; depth stamps before the first and after the last pose,
    repeated stamps and exact ties between two poses; depth stamps out of order, where the
    forward search keeps a later pose.  Quaternions are written with 4 decimals, so they are
    not exactly of unit length."""
    import tempfile
    if not refpipe.available():
        pytest.skip("the reference harness is built only where a reference checkout exists")
    rng = np.random.default_rng({"regular": 21, "edges_and_ties": 22, "out_of_order": 23}[case])
    gt_t = np.round(np.arange(0.0, 2.0, 0.01) + 1305031102.0, 4)
    trans = rng.normal(size=(gt_t.size, 3))
    quats = rng.normal(size=(gt_t.size, 4))
    quats /= np.linalg.norm(quats, axis=1, keepdims=True)
    if case == "regular":
        depth_t = gt_t[3::7][:25] + 0.0031
    elif case == "edges_and_ties":
        depth_t = np.concatenate([[gt_t[0] - 0.5, gt_t[0]], gt_t[10:14] + 0.005,   # midway: ties
                                  [gt_t[20], gt_t[20], gt_t[57] + 0.004],
                                  [gt_t[-1], gt_t[-1] + 0.3, gt_t[-1] + 7.0]])
    else:
        depth_t = np.concatenate([gt_t[[40, 80, 60, 20, 90, 89, 150, 5, 199]] + 0.002])
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "depth"))
        _write_tum(d, gt_t, trans, quats, depth_t)
        ref_frames, ref_inv = refpipe.tum_sequence(d)
        ds = kf.RgbdDataset(d)
        try:
            assert len(ds) == len(ref_frames) == len(depth_t)
            for k, (path, ref_pose) in enumerate(ref_frames):
                assert path == os.path.join(d, "depth/%.6f.png" % depth_t[k])
                pose = np.asarray(ds.getCurrentPose(), np.float32)
                np.testing.assert_array_equal(pose, ref_pose.astype(np.float32), err_msg="frame %d" % k)
                ds.m_current_index += 1
            if case == "out_of_order":
                # the stamp near pose 60 after the one near pose 80: the forward search stops at
                # pose 80 again (a global nearest search would take pose 60)
                np.testing.assert_array_equal(ref_frames[2][1], ref_frames[1][1])
            np.testing.assert_allclose(np.asarray(ds.getInitialPoseInverse(), np.float32), ref_inv,
                                       rtol=1e-6, atol=2e-6)
        finally:
            ds.close()


@pytest.mark.parametrize("fov", [525.0, 517.3, 481.2])
def test_level_intrinsics_equal_the_reference_sensor(kf, fov):
    """The library's level intrinsics and the K^-1 it forms for its rays (kfb200's mirror of
    it) against the reference's own Sensor (project/src/sensor.h:10-52, compiled from its
    sources): bit for bit at every level, for a 640 x 480 frame with fx = fy = fov, the only
    frame the reference's fixed principal points describe."""
    if not refpipe.available():
        pytest.skip("the reference harness is built only where a reference checkout exists")
    cfg = kf.default_config(width=640, height=480, fx=fov, fy=fov, cx=319.5, cy=239.5, levels=3)
    for level in range(3):
        ref_k, ref_ik = refpipe.sensor_intrinsics(fov, level)
        np.testing.assert_array_equal(kf.level_intrinsics(cfg, level).astype(np.float32), ref_k)
        np.testing.assert_array_equal(kf.level_inverse_intrinsics(cfg, level), ref_ik)
