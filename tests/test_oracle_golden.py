"""Pins the CPU oracle (oracle/kf_oracle.cpp) to the reference's own known-answer tests and to
hand-derived answers for the stages no reference test covers.  CPU only.

Reference tests restated here (values copied from the reference test files):
    test/icp_tests.cpp:55-80    TestComputeCorrespondence
    test/icp_tests.cpp:82-98    TestNormalsAreTooDifferent
    test/icp_tests.cpp:100-114  TestComputeAndFillA
    test/icp_tests.cpp:116-127  TestComputeAndFillB
    test/icp_tests.cpp:129-157  TestSolveLinearSystem
    test/icp_tests.cpp:159-231  TestConstructIcpResiduals
    test/transformation_tests.cpp:41-59  TestComputeNormal (all three components)
    test/example_test.cpp:36-50 TestGlmToArray (column-major layout)
The golden values also live in tests/golden/reference_known_answers.json, which the GPU
tests use for the same cases through the C ABI.
"""
import json
import math
import os

import numpy as np

from conftest import ROOT

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_known_answers.json")))

PI = 3.14159265358979323846
# glm::mat3(vec3 c0, vec3 c1, vec3 c2) builds columns; these are [row, col] arrays
K_TEST = np.array(GOLDEN["intrinsics_rows"], np.float32)          # [[2,0,1],[0,2,1],[0,0,1]]
ROT90 = np.array(GOLDEN["rotation_90_rows"], np.float32)


def test_compute_correspondence(orc):
    g = GOLDEN["compute_correspondence"]
    for v, want in zip(g["vertices"], g["pixels"]):
        assert orc.compute_correspondence(v, ROT90, [0, 0, 0], K_TEST) == tuple(want)


def test_normals_are_too_different(orc):
    g = GOLDEN["normals_too_different"]
    assert not orc.normals_too_different(g["close"], g["target"], ROT90, PI / 2)
    assert orc.normals_too_different(g["far"], g["target"], ROT90, PI / 2)


def test_compute_and_fill_a_b(orc):
    g = GOLDEN["fill_a_b"]
    a, b = orc.fill_a_b(g["vertex"], g["normal"], g["target_vertex"])
    np.testing.assert_array_equal(a, np.array(g["a"], np.float32))
    assert b == g["b"]


def test_solve_linear_system(orc):
    g = GOLDEN["solve_linear_system"]
    A = np.array(g["A"], np.float32)
    b = np.array(g["b"], np.float32)
    for prec in (0, 1):
        x = orc.solve_lls(A, b, prec=prec)
        np.testing.assert_allclose(x, np.ones(6), atol=1e-4)


def test_construct_icp_residuals(orc):
    g = GOLDEN["construct_icp_residuals"]
    tv = np.array(g["target_vertices"], np.float32).reshape(2, 2, 4)
    tn = np.array(g["target_normals"], np.float32).reshape(2, 2, 4)
    v = np.array(g["vertices"], np.float32).reshape(2, 2, 4)
    eye = np.eye(3, dtype=np.float32)
    A, b, mask, count = orc.icp_residuals(v, tv, tn, eye, [0, 0, 0], eye, [0, 0, 0], K_TEST,
                                          g["distance_threshold"], PI)
    np.testing.assert_array_equal(A, np.array(g["A"], np.float32))
    np.testing.assert_array_equal(b, np.array(g["b"], np.float32))
    assert count == 1 and mask.reshape(-1).tolist() == [1, 0, 0, 0]


def test_compute_normal(orc):
    g = GOLDEN["compute_normal"]
    v = np.array(g["vertices"], np.float32).reshape(2, 2, 4)
    # the reference's map uses w = 0 for these entries; validity needs the tag -1
    v[..., 3] = -1.0
    n = orc.compute_normal(v, 0, 0)
    np.testing.assert_array_equal(n[:3], np.array(g["normal"], np.float32))
    assert n[3] == -1.0


def test_column_major_layout(kf):
    # glm::mat3(vec3(0,1,0), vec3(-1,42,0), vec3(0,0,1)): flat[4] is m[1][1]
    cols = np.array([[0, 1, 0], [-1, 42, 0], [0, 0, 1]], np.float32)
    flat = kf.to_colmajor(cols.T)
    assert flat[4] == 42.0


# ---- hand-derived known answers (stages no reference test pins) ----

def test_half_rounding(orc):
    # __half2float of an unsigned short converts the value, round to nearest even
    for u, want in [(0, 0.0), (1, 1.0), (2047, 2047.0), (2048, 2048.0), (2049, 2048.0), (2051, 2052.0),
                    (4097, 4096.0), (10001, 10000.0), (65504, 65504.0), (65519, 65504.0)]:
        assert orc.half_value(u) == want, u
    assert math.isinf(orc.half_value(65520)) and math.isinf(orc.half_value(65535))


def test_convert_unmirror(orc):
    raw = np.arange(32, dtype=np.uint16).reshape(4, 8) * 100
    d = orc.convert(raw, 1e-3)
    np.testing.assert_array_equal(d, raw.astype(np.float32) * np.float32(1e-3))
    m = orc.convert(raw, 1e-3, unmirror=True)
    np.testing.assert_array_equal(m, d[:, ::-1])


def test_bilateral_constant_plane(orc):
    d = np.full((16, 20), 1.5, np.float32)
    for prec in (0, 1):
        out = orc.bilateral(d, 4.0, 0.25, 3, prec=prec)
        np.testing.assert_allclose(out, 1.5, rtol=1e-6)


def test_bilateral_edge_preserving(orc):
    # a 1 m step: with sigma_r = 30 mm the other side's weight is exp(-1/0.0009) = 0
    d = np.full((16, 16), 1.0, np.float32)
    d[:, 8:] = 2.0
    out = orc.bilateral(d, 4.5, 0.03, 2)
    np.testing.assert_allclose(out[:, :8], 1.0, rtol=1e-6)
    np.testing.assert_allclose(out[:, 8:], 2.0, rtol=1e-6)


def test_bilateral_known_value(orc):
    # 3x1 neighbourhood by hand: radius 1 on a 1-row image = clamped rows
    d = np.array([[1.0, 1.1, 1.0]], np.float32)
    out = orc.bilateral(d, 1.0, 0.5, 1, prec=1)
    # centre pixel: offsets x in {-1,0,1}, y rows all clamp to the same row
    num = den = 0.0
    for x in (-1, 0, 1):
        for y in (-1, 0, 1):
            cur = d[0, 1 + x]
            e = math.exp(-(x * x + y * y) / 1.0 - (1.1 - cur) ** 2 / 0.25)
            num += e * cur
            den += e
    assert abs(out[0, 1] - num / den) < 1e-6


def test_down_sample_rules(orc):
    d = np.array([[1.0, 1.2, 3.0, 3.0],
                  [1.1, 5.0, 3.0, 0.0]], np.float32)
    out = orc.down_sample(d, 0.25)
    # block 0: f1 = 1.0; 1.2 and 1.1 within 0.75, 5.0 not -> (1.0 + 1.2 + 1.1) / 3
    assert abs(out[0, 0] - np.float32((np.float32(1.0) + np.float32(1.2)) + np.float32(1.1)) / np.float32(3)) < 1e-7
    # block 1: zeros are not excluded when close to f1 -- here 0 is 3 m away, so excluded
    assert out[0, 1] == np.float32(3.0)


def test_trunc8_covers_the_reference_launch_grids(orc):
    """compat_trunc8 processes only the pixels the reference's launches reach: blocks =
    dims / 8 of 8 x 8 threads (project/src/measurement.cu:150-151, 171-172, 192-193, 213-214),
    so at 80 x 60 (level 2 of 320 x 240) rows 56-59 keep the output's initial contents; 640 x
    480 and 320 x 240 divide by 8 and are covered whole."""
    rng = np.random.default_rng(5)
    raw = rng.integers(500, 4000, size=(60, 80)).astype(np.uint16)
    full = orc.convert(raw, 1e-3)
    part = orc.convert(raw, 1e-3, trunc8=True)
    assert np.all(full > 0)
    np.testing.assert_array_equal(part[:56], full[:56])
    assert np.all(part[56:] == 0)           # never written: the initial zeros stay
    # the same for the 2x2 downsample into 80 x 60 and for the vertex map of that level
    d = rng.uniform(0.5, 4.0, size=(120, 160)).astype(np.float32)
    ds_full = orc.down_sample(d, 0.03)
    ds_part = orc.down_sample(d, 0.03, trunc8=True)
    np.testing.assert_array_equal(ds_part[:56], ds_full[:56])
    assert np.all(ds_part[56:] == 0) and np.all(ds_full[56:] > 0)
    inv_k = np.linalg.inv(np.array([[131.25, 0, 39.5], [0, 131.25, 29.5], [0, 0, 1]], np.float32))
    vm_full = orc.vertex_map(ds_full, inv_k)
    vm_part = orc.vertex_map(ds_full, inv_k, trunc8=True)
    np.testing.assert_array_equal(vm_part[:56], vm_full[:56])
    assert np.all(vm_part[56:] == 0) and np.all(vm_full[56:, :, 3] == -1.0)
    # sizes that divide by 8 are unaffected
    raw2 = rng.integers(500, 4000, size=(240, 320)).astype(np.uint16)
    np.testing.assert_array_equal(orc.convert(raw2, 1e-3, trunc8=True), orc.convert(raw2, 1e-3))


def test_vertex_map_constant_depth(orc, kf):
    cfg = kf.default_config(width=8, height=4, fx=2.0, fy=2.0, cx=3.5, cy=1.5, levels=1)
    k = kf.level_intrinsics(cfg, 0)
    d = np.full((4, 8), 2.0, np.float32)
    d[1, 2] = 0.0          # invalid
    d[2, 3] = 0.005        # below cMinDepth
    v = orc.vertex_map(d, np.linalg.inv(k), prec=1)
    assert v[0, 0, 3] == -1.0 and v[1, 2, 3] == -2.0 and v[2, 3, 3] == -2.0
    # (i + .5 - cx) / fx * d
    np.testing.assert_allclose(v[0, 0, :3], [(0.5 - 3.5) / 2 * 2, (0.5 - 1.5) / 2 * 2, 2.0], atol=1e-6)


def test_voxel_axes_accumulate_in_float(orc):
    xs, zs = orc.voxel_axes(512, 3.0)
    res = np.float32(3.0) / np.float32(511)
    z = np.float32(-1.5) + np.float32(-res)
    ref = []
    for _ in range(512):
        z = np.float32(z + res)
        ref.append(z)
    np.testing.assert_array_equal(zs, np.array(ref, np.float32))
    np.testing.assert_array_equal(xs, np.float32(-1.5) + np.arange(512, dtype=np.float32) * res)


def test_fuse_single_voxel_known_answer(orc, kf):
    # camera at the origin looking +z, 8^3 volume 1.4 m wide; depth 1 m everywhere
    n, width, mu = 8, 1.4, 0.1
    cfg = kf.default_config(width=64, height=64, fx=50.0, fy=50.0, cx=31.5, cy=31.5, levels=1)
    k = kf.level_intrinsics(cfg, 0)
    depth = np.full((64, 64), 1.0, np.float32)
    f = np.full((n, n, n), 2.0, np.float32)
    w = np.zeros((n, n, n), np.float32)
    pose = np.eye(4, dtype=np.float32)
    pose[2, 3] = -0.5   # volume z range [-0.7, 0.7] -> camera depth [-0.2, 1.2]
    orc.fuse(depth, k, f, w, width, mu, pose, prec=1)
    xs, zs = orc.voxel_axes(n, width)
    i = j = 4
    for kk in range(n):
        z_eye = zs[kk] + 0.5
        px = 50.0 * xs[i] / z_eye + 31.5 if z_eye > 0 else -1
        inside = 0.4 <= z_eye < 6.0 and 0 <= px < 64
        diff = 1.0 - z_eye
        if inside and diff >= -mu:
            assert abs(f[kk, j, i] - min(1.0, diff / mu)) < 1e-5
            assert abs(w[kk, j, i] - 1.0) < 1e-6
        else:
            assert f[kk, j, i] == 2.0 and w[kk, j, i] == 0.0
    # second identical frame: same f, weight doubles
    f2, w2 = f.copy(), w.copy()
    orc.fuse(depth, k, f2, w2, width, mu, pose, prec=1)
    upd = w > 0
    np.testing.assert_allclose(f2[upd], f[upd], atol=1e-6)
    np.testing.assert_allclose(w2[upd], 2.0 * w[upd], atol=1e-6)


def test_raycast_plane_known_answer(orc, kf):
    # fuse a fronto-parallel plane at 1.0 m depth repeatedly and raycast it back
    n, width, mu = 64, 2.0, 0.06
    cfg = kf.default_config(width=32, height=24, fx=30.0, fy=30.0, cx=15.5, cy=11.5, levels=1)
    k = kf.level_intrinsics(cfg, 0)
    depth = np.full((24, 32), 1.0, np.float32)
    f = np.full((n, n, n), 2.0, np.float32)
    w = np.zeros((n, n, n), np.float32)
    pose = np.eye(4, dtype=np.float32)
    pose[2, 3] = -0.6
    for _ in range(2):
        orc.fuse(depth, k, f, w, width, mu, pose, prec=1)
    v, nrm, samples = orc.raycast(f, width, mu, pose, np.linalg.inv(k), 32, 24, keep_on_miss=False, prec=1)
    hit = v[..., 3] == -1
    assert hit.mean() > 0.9 and samples > 0
    # Where the model is seen: the raycast's texel mapping (uvw * n - 0.5) scales the fused
    # model by (n - 1) / n about the origin, so the plane at world z = 0.4 appears at
    # 0.4 (n - 1) / n.  The reference's refinement t - step * f_prev / (f - f_prev)
    # (project/src/raycast.cu:106) extrapolates from the current sample, one small step
    # (0.1 mu) beyond the interpolated crossing.  Interior pixels (away from the frustum
    # edge, where unobserved voxels enter the interpolation) show exactly that.
    z_model = 0.4 * (n - 1) / n + 0.1 * mu
    inner = np.zeros_like(hit)
    inner[3:-3, 3:-3] = True
    dz = np.abs(v[hit & inner][:, 2] - z_model)
    assert dz.max() < 1e-4
    # normals point away from the camera (-grad f), along +z
    assert np.all(nrm[hit & inner][:, 2] > 0.99)


def test_euler_yxz_small_angles(orc):
    # to first order every Euler order gives I + [w]x
    w = np.array([1e-3, -2e-3, 1.5e-3])
    R = orc.euler_yxz(*w)
    skew = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    np.testing.assert_allclose(R, np.eye(3) + skew, atol=5e-6)
    # Y * X * Z composition for a pure rotation about each axis
    b = 0.3
    np.testing.assert_allclose(orc.euler_yxz(b, 0, 0), [[1, 0, 0], [0, np.cos(b), -np.sin(b)], [0, np.sin(b), np.cos(b)]],
                               atol=1e-6)
    np.testing.assert_allclose(orc.euler_yxz(0, b, 0), [[np.cos(b), 0, np.sin(b)], [0, 1, 0], [-np.sin(b), 0, np.cos(b)]],
                               atol=1e-6)
    np.testing.assert_allclose(orc.euler_yxz(0, 0, b), [[np.cos(b), -np.sin(b), 0], [np.sin(b), np.cos(b), 0], [0, 0, 1]],
                               atol=1e-6)


def test_update_pose_and_pose_error(orc):
    pose = np.eye(4, dtype=np.float32)
    st, p2 = orc.update_pose(pose, [0, 0, 0, 0.1, -0.2, 0.3])
    assert st == 0
    np.testing.assert_allclose(p2[:3, 3], [0.1, -0.2, 0.3], atol=1e-7)
    a, d = orc.pose_error(pose, p2)
    assert a == 0.0 and abs(d - math.sqrt(0.14)) < 1e-6
    st, _ = orc.update_pose(pose, [float("nan"), 0, 0, 0, 0, 0])
    assert st == 4  # KF_ERR_NONFINITE: the reference throws here (icp.cpp:67-73)


def test_pipeline_frame0_fuses_only(orc, kf):
    from kfb200 import synth
    cfg = kf.config_small()
    frames, _ = synth.sequence(cfg, 2, seed=3)
    P = orc.Pipeline(cfg, prec=0)
    st, pose = P.process_frame(frames[0])
    assert st == 0 and P.iters() == [0, 0, 0]
    np.testing.assert_allclose(pose, kf.start_pose(2.0), atol=0)
    assert P.last_fused() > 0
    st, _ = P.process_frame(frames[1])
    assert st == 0 and sum(P.iters()) > 0


# ---- the fixture against the reference's test sources it was transcribed from ----

# a checkout of the reference project, given by the environment; without one the two checks
# below are skipped
REFERENCE_ROOT = os.environ.get("KF_REFERENCE_ROOT", "")


def _transcription():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "check_transcription", os.path.join(ROOT, "tests", "golden", "check_transcription.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_golden_transcription_matches_reference_sources():
    """Every number of every fixture entry appears among the numeric literals of the test lines
    it cites (runs where KF_REFERENCE_ROOT names a reference checkout)."""
    import pytest
    if not REFERENCE_ROOT or not os.path.isdir(os.path.join(REFERENCE_ROOT, "test")):
        pytest.skip("no reference checkout on this machine")
    assert _transcription().check(REFERENCE_ROOT) == []


def test_golden_transcription_check_catches_a_changed_value():
    """A planted transcription mistake (b of TestComputeAndFillB changed from -7 to -7.5) is
    reported for that entry alone."""
    import copy
    import pytest
    if not REFERENCE_ROOT or not os.path.isdir(os.path.join(REFERENCE_ROOT, "test")):
        pytest.skip("no reference checkout on this machine")
    fx = copy.deepcopy(GOLDEN)
    fx["fill_a_b"]["b"] = -7.5
    bad = _transcription().check(REFERENCE_ROOT, fx)
    assert [(k, m) for k, _, m in bad] == [("fill_a_b", [-7.5])]


# ---- TestComputePose (test/icp_tests.cpp:233-326) on synthetic frames ----

def two_frame_case(kf, orc, kind, seed, a, b, prec=1):
    """The reference's TestComputePose set-up with two synthetic frames instead of TUM
    fr1/xyz (absent): ICP {8, 4, 2} fine to coarse, distance 0.5 m, angle 6 pi / 18; frame a's
    measured vertex and normal maps are the target (its camera is the world frame, so the
    previous pose is the identity), frame b's vertex maps the source.  Returns the ground-truth
    relative pose inverse(P_a) P_b, the cfg and the maps."""
    from kfb200 import synth
    cfg = kf.config_full(iters=(8, 4, 2), dist_thresh=0.5, angle_thresh=float(6.0 * PI / 18.0))
    imgs, poses = synth.sequence(cfg, max(a, b) + 1, seed=seed, kind=kind)

    def pyramid(img):
        d = orc.convert(img, cfg.depth_scale)
        ds = [orc.bilateral(d, cfg.bilateral_sigma_s, cfg.bilateral_sigma_r, cfg.bilateral_radius, prec=prec)]
        for _ in (1, 2):
            ds.append(orc.down_sample(ds[-1], cfg.bilateral_sigma_r, prec=prec))
        vs = [orc.vertex_map(ds[l], kf.level_inverse_intrinsics(cfg, l), prec=prec) for l in range(3)]
        return vs, [orc.normal_map(v, prec=prec) for v in vs]

    (va, na), (vb, _) = pyramid(imgs[a]), pyramid(imgs[b])
    true = np.linalg.inv(poses[a].astype(np.float64)) @ poses[b].astype(np.float64)
    return cfg, true, vb, va, na


def rotated_diagonal_angle(r_true, r_est):
    """The reference's rotation check: the angle between R v for v = (1, 1, 1) / sqrt(3)."""
    v = np.ones(3) / np.sqrt(3.0)
    x = np.asarray(r_true, np.float64) @ v
    y = np.asarray(r_est, np.float64) @ v
    x /= np.linalg.norm(x)
    y /= np.linalg.norm(y)
    return float(np.arccos(np.clip(x @ y, -1.0, 1.0)))


def test_compute_pose_two_synthetic_frames(kf, orc):
    """Ground-truth relative motion recovered within the reference's bounds (angle <= pi / 90,
    translation within 0.01 m per axis), here for a small hand-held-like motion and for a
    0.15 rad / 0.32 m step of the loop trajectory; FP64 and float oracle alike."""
    from kfb200 import synth
    for kind, seed, a, b in ((synth.WOBBLE, 5, 4, 5), (synth.LOOP, 3, 10, 11)):
        for prec in (1, 0):
            cfg, true, vb, va, na = two_frame_case(kf, orc, kind, seed, a, b, prec)
            st, est, iters = orc.compute_pose(cfg, vb, va, na, np.eye(4, dtype=np.float32), prec=prec)
            assert st == 0
            assert rotated_diagonal_angle(true[:3, :3], est[:3, :3]) <= PI / 90.0
            assert np.max(np.abs(true[:3, 3] - est[:3, 3])) <= 0.01
            # and far tighter in practice (measured: <= 6.1e-4 rad, <= 4.2e-4 m)
            assert rotated_diagonal_angle(true[:3, :3], est[:3, :3]) <= 2e-3
            assert np.max(np.abs(true[:3, 3] - est[:3, 3])) <= 2e-3
