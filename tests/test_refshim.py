"""Host checks of the build of the reference's own pipeline (oracle/Makefile, oracle/refshim,
oracle/ref_harness.cpp, oracle/refpipe.py), no GPU:
  - the glm subset the reference's sources compile against computes what glm's documented
    functions compute (inverse, transpose, orientate3 = Ry(yaw) Rx(pitch) Rz(roll), normalize,
    cross, column-major products), checked against numpy;
  - the harness library, where it is built, exports every entry point refpipe binds;
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
