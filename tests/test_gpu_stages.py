"""Per-stage parity: each CUDA stage (through the C ABI) against the CPU oracle on identical
inputs, plus the reference's own known answers on the device.

Tolerances (floating point, stated per test): values from the fused/fast-exp kernels agree
with the float oracle to ~1e-6 relative; masks and integer decisions agree exactly except
where stated; raycast depths agree within 1 mm where both hit."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_known_answers.json")))
PI = 3.14159265358979323846


def dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        return torch.from_numpy(a.view(np.int16)).cuda()
    return torch.from_numpy(a).cuda()


def host(t, dtype=None):
    a = t.cpu().numpy()
    return a.view(dtype) if dtype is not None else a


@pytest.fixture(scope="module")
def frames_small(kf):
    from kfb200 import synth
    cfg = kf.config_small()
    imgs, poses = synth.sequence(cfg, 6, seed=21)
    return cfg, imgs, poses


# ---- preprocessing ----

def test_convert_bit_exact(kf, orc, cuda, frames_small):
    cfg, imgs, _ = frames_small
    raw = imgs[1].copy()
    raw[0, :6] = [2049, 4097, 10001, 65504, 65519, 65535]   # fp16 rounding and inf
    out = cuda.zeros((cfg.height, cfg.width), dtype=cuda.float32, device="cuda")
    for unmirror in (False, True):
        kf.kernel.convertToDepthMeters(dev(cuda, raw), out, cfg.depth_scale, unmirror)
        want = orc.convert(raw, cfg.depth_scale, unmirror)
        np.testing.assert_array_equal(host(out), want)


def test_shape_mismatch_raises(kf, cuda):
    a = cuda.zeros((8, 8), dtype=cuda.float32, device="cuda")
    b = cuda.zeros((8, 16), dtype=cuda.float32, device="cuda")
    with pytest.raises(kf.KfError) as e:
        kf.kernel.applyBilateralFilter(a, b)
    assert e.value.status == kf.KF_ERR_SHAPE
    with pytest.raises(kf.KfError):
        kf.kernel.downSample(a, a)


@pytest.mark.parametrize("ss,sr,r", [(4.0, 0.25, 3), (4.5, 0.03, 2)])
def test_bilateral_vs_oracle(kf, orc, cuda, frames_small, ss, sr, r):
    cfg, imgs, _ = frames_small
    d = orc.convert(imgs[2], cfg.depth_scale)
    out = cuda.zeros_like(dev(cuda, d))
    ms = kf.kernel.applyBilateralFilter(dev(cuda, d), out, ss, sr, r)
    assert ms >= 0.0
    got = host(out)
    want = orc.bilateral(d, ss, sr, r, prec=1)
    np.testing.assert_array_equal(got > 0.01, want > 0.01)
    valid = want > 0.01
    # fast exponential (the reference's -use_fast_math build) vs FP64: 2e-6 relative
    np.testing.assert_allclose(got[valid], want[valid], rtol=2e-6)


def test_down_sample_vs_oracle(kf, orc, cuda, frames_small):
    """The same gating and sums as the oracle; the mean divides the way the reference's
    fast-math build does (at most 2 ulp from IEEE division, exact for 1, 2 or 4 terms), so the
    oracle's IEEE quotient is matched within 2 ulp.  Bit-exactness is checked against the
    reference's own kernel (test_gpu_reference_pipeline.py)."""
    cfg, imgs, _ = frames_small
    d = orc.bilateral(orc.convert(imgs[3], cfg.depth_scale), 4.5, 0.03, 2)
    out = cuda.zeros((cfg.height // 2, cfg.width // 2), dtype=cuda.float32, device="cuda")
    kf.kernel.downSample(dev(cuda, d), out, 0.03)
    got = np.ascontiguousarray(host(out), np.float32)
    want = np.ascontiguousarray(orc.down_sample(d, 0.03), np.float32)
    np.testing.assert_array_equal(got > 0.01, want > 0.01)
    ulps = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert int(ulps.max()) <= 2, int(ulps.max())


def test_vertex_and_normal_maps(kf, orc, cuda, frames_small):
    cfg, imgs, _ = frames_small
    d = orc.convert(imgs[1], cfg.depth_scale)
    ik = np.linalg.inv(kf.level_intrinsics(cfg, 0).astype(np.float64)).astype(np.float32)
    vm = cuda.zeros((cfg.height, cfg.width, 4), dtype=cuda.float32, device="cuda")
    kf.kernel.createVertexMap(dev(cuda, d), vm, ik)
    got = host(vm)
    want = orc.vertex_map(d, ik, prec=1)
    np.testing.assert_array_equal(got[..., 3], want[..., 3])
    np.testing.assert_allclose(got[..., :3], want[..., :3], rtol=1e-6, atol=1e-7)
    nm = cuda.zeros_like(vm)
    kf.kernel.createNormalMap(vm, nm)
    gn = host(nm)
    wn = orc.normal_map(got, prec=1)
    np.testing.assert_array_equal(gn[..., 3], wn[..., 3])
    ok = (wn[..., 3] == -1) & np.all(np.isfinite(wn[..., :3]), axis=-1)
    assert np.max(np.abs(gn[ok][:, :3] - wn[ok][:, :3])) < 2e-4


def test_compute_normal_known_answer(kf, cuda):
    g = GOLDEN["compute_normal"]
    v = np.array(g["vertices"], np.float32).reshape(2, 2, 4)
    v[..., 3] = -1.0
    nm = cuda.zeros((2, 2, 4), dtype=cuda.float32, device="cuda")
    kf.kernel.createNormalMap(dev(cuda, v), nm)
    n = host(nm)
    np.testing.assert_array_equal(n[0, 0, :3], np.array(g["normal"], np.float32))
    assert n[0, 0, 3] == -1.0 and n[0, 1, 3] == -2.0 and n[1, 0, 3] == -2.0


# ---- ICP pieces ----

def test_construct_icp_residuals_known_answer(kf, cuda):
    g = GOLDEN["construct_icp_residuals"]
    K = np.array(GOLDEN["intrinsics_rows"], np.float32)
    eye = np.eye(3, dtype=np.float32)
    tv = dev(cuda, np.array(g["target_vertices"], np.float32).reshape(2, 2, 4))
    tn = dev(cuda, np.array(g["target_normals"], np.float32).reshape(2, 2, 4))
    vm = dev(cuda, np.array(g["vertices"], np.float32).reshape(2, 2, 4))
    A = cuda.full((4, 6), 7.0, dtype=cuda.float32, device="cuda")
    b = cuda.full((4,), 7.0, dtype=cuda.float32, device="cuda")
    kf.kernel.constructIcpResiduals(vm, tv, tn, eye, [0, 0, 0], eye, [0, 0, 0], K, g["distance_threshold"], PI, A, b)
    np.testing.assert_array_equal(host(A), np.array(g["A"], np.float32))
    np.testing.assert_array_equal(host(b), np.array(g["b"], np.float32))


def test_solve_linear_system_known_answer(kf, cuda):
    g = GOLDEN["solve_linear_system"]
    A = dev(cuda, np.array(g["A"], np.float32))
    b = dev(cuda, np.array(g["b"], np.float32))
    x = kf.LinearLeastSquares().solve(A, b, 7)
    np.testing.assert_allclose(x, np.ones(6), atol=1e-4)


def test_solve_linear_system_large_vs_fp64(kf, cuda):
    rng = np.random.default_rng(5)
    n = 307200
    A = rng.normal(size=(n, 6)).astype(np.float32)
    xt = rng.normal(size=6)
    b = (A.astype(np.float64) @ xt + 1e-3 * rng.normal(size=n)).astype(np.float32)
    x = kf.LinearLeastSquares().solve(dev(cuda, A), dev(cuda, b), n)
    Ad = A.astype(np.float64)
    xd = np.linalg.solve(Ad.T @ Ad, Ad.T @ b.astype(np.float64))
    np.testing.assert_allclose(x, xd, rtol=1e-5, atol=1e-6)


# ---- volume stages ----

def fused_oracle_volume(kf, orc, cfg, imgs, poses, nframes):
    n = cfg.volume_n
    f = np.full((n, n, n), 2.0, np.float32)
    w = np.zeros((n, n, n), np.float32)
    k = kf.level_intrinsics(cfg, 0)
    for i in range(nframes):
        d = orc.convert(imgs[i], cfg.depth_scale)
        orc.fuse(d, k, f, w, cfg.volume_width, cfg.mu, poses[i])
    return f, w


def test_fuse_vs_oracle(kf, orc, cuda, frames_small):
    cfg, imgs, poses = frames_small
    n = cfg.volume_n
    f0, w0 = fused_oracle_volume(kf, orc, cfg, imgs, poses, 2)
    d = orc.convert(imgs[2], cfg.depth_scale)
    ft, wt = dev(cuda, f0), dev(cuda, w0)
    vol = kf.kernel.volume(ft, wt, cfg.volume_width, cfg.mu)
    kf.kernel.fuse(dev(cuda, d), vol, poses[2], kf.level_intrinsics(cfg, 0))
    cuda.cuda.synchronize()
    fw, ww = f0.copy(), w0.copy()
    orc.fuse(d, kf.level_intrinsics(cfg, 0), fw, ww, cfg.volume_width, cfg.mu, poses[2], prec=1)
    gf, gw = host(ft), host(wt)
    df = np.abs(gf - fw)
    # float arithmetic vs FP64: a voxel whose projection sits on a pixel edge may pick the
    # neighbouring pixel; everything else agrees to 1e-3 of the truncation distance
    assert np.mean(df <= 1e-3) >= 0.9999
    assert np.mean(np.abs(gw - ww) <= 1e-5 * np.maximum(1.0, ww)) >= 0.9999


def test_fuse_f16u16_vs_oracle(kf, orc, cuda, frames_small):
    """FP16 distance + uint16 weight fusion, three frames.  Against the f32 volume fused by the
    same kernels on the same frames (identical projections), every voxel differs only by the
    storage rounding: fp16 (2^-11 relative) and 1/1024 weight steps, re-rounded on each of the
    three updates.  Against the FP64 oracle, voxels whose projection sits within float rounding
    of a pixel edge may read the neighbouring pixel in some frame; their share is bounded and
    the rest agree."""
    cfg, imgs, poses = frames_small
    n = cfg.volume_n
    f_h = cuda.full((n, n, n), 2.0, dtype=cuda.float16, device="cuda")
    w_h = cuda.zeros((n, n, n), dtype=cuda.int16, device="cuda")
    vol = kf.kernel.volume(f_h, w_h, cfg.volume_width, cfg.mu, fmt=kf.KF_TSDF_F16U16)
    kf.kernel.initializeGrid(vol)
    f_s = cuda.full((n, n, n), 2.0, dtype=cuda.float32, device="cuda")
    w_s = cuda.zeros((n, n, n), dtype=cuda.float32, device="cuda")
    vol32 = kf.kernel.volume(f_s, w_s, cfg.volume_width, cfg.mu)
    f = np.full((n, n, n), 2.0, np.float32)
    w = np.zeros((n, n, n), np.float32)
    k = kf.level_intrinsics(cfg, 0)
    for i in range(3):
        d = orc.convert(imgs[i], cfg.depth_scale)
        kf.kernel.fuse(dev(cuda, d), vol, poses[i], k)
        kf.kernel.fuse(dev(cuda, d), vol32, poses[i], k)
        orc.fuse(d, k, f, w, cfg.volume_width, cfg.mu, poses[i], prec=1)
    gf = host(f_h).astype(np.float32)
    gw = host(w_h, np.uint16).astype(np.float32) / kf.KF_WEIGHT_SCALE
    sf, sw = host(f_s), host(w_s)
    # storage rounding only, against the f32 volume of the same kernels
    assert np.array_equal(gw > 0, sw > 0)
    up = sw > 0
    wq = 3 * 0.5 / kf.KF_WEIGHT_SCALE + 1e-6
    assert np.mean(np.abs(gw[up] - sw[up]) <= wq) >= 0.9999
    # |f| <= 1 after the first update: three fp16 roundings (3 * 2^-11) plus the weighting by
    # rounded weights (below 1e-3 for these depths)
    assert np.mean(np.abs(gf[up] - sf[up]) <= 2.5e-3) >= 0.9999
    assert np.sqrt(np.mean((gf[up] - sf[up]) ** 2)) < 5e-4
    # against the FP64 oracle
    upd = w > 0
    assert np.mean((gw > 0) == upd) > 0.9999
    both = upd & (gw > 0)
    df = np.abs(gf[both] - f[both])
    assert np.mean(df <= 2e-3) > 0.999
    assert np.sqrt(np.mean(df[df <= 0.05] ** 2)) < 1e-3
    dw = np.abs(gw[both] - w[both])
    assert np.mean(dw > wq) < 0.01          # pixel-edge picks differ (about 0.1-0.5 % of voxels)


def test_initialize_grid(kf, cuda):
    n = 16
    f = cuda.zeros((n, n, n), dtype=cuda.float32, device="cuda")
    w = cuda.ones((n, n, n), dtype=cuda.float32, device="cuda")
    kf.kernel.initializeGrid(kf.kernel.volume(f, w, 1.0, 0.1))
    assert float(f.min()) == 2.0 and float(f.max()) == 2.0 and float(w.abs().max()) == 0.0


@pytest.mark.parametrize("fmt", [0, 1])
def test_raycast_vs_oracle(kf, orc, cuda, frames_small, fmt):
    cfg, imgs, poses = frames_small
    f, w = fused_oracle_volume(kf, orc, cfg, imgs, poses, 4)
    if fmt == 1:
        f = f.astype(np.float16).astype(np.float32)   # what the fp16 volume stores
        ft = dev(cuda, f.astype(np.float16))
        wt = dev(cuda, np.zeros(f.shape, np.int16))
    else:
        ft, wt = dev(cuda, f), dev(cuda, w)
    vol = kf.kernel.volume(ft, wt, cfg.volume_width, cfg.mu, fmt=fmt)
    for level in range(3):
        k = kf.level_intrinsics(cfg, level)
        ik = np.linalg.inv(k.astype(np.float64)).astype(np.float32)
        wl, hl = cfg.width >> level, cfg.height >> level
        vt = cuda.zeros((hl, wl, 4), dtype=cuda.float32, device="cuda")
        nt = cuda.zeros_like(vt)
        kf.kernel.raycast(vol, poses[4], ik, vt, nt, step_large=cfg.step_large, step_small=cfg.step_small)
        gv, gn = host(vt), host(nt)
        ov, on, _ = orc.raycast(f, cfg.volume_width, cfg.mu, poses[4], ik, wl, hl, step_l=cfg.step_large,
                                step_s=cfg.step_small, prec=1)
        gh, oh = gv[..., 3] == -1, ov[..., 3] == -1
        assert oh.mean() > 0.1
        assert np.mean(gh == oh) >= 0.999
        both = gh & oh
        cam = poses[4][:3, 3]
        dz = np.abs(np.linalg.norm(gv[both][:, :3] - cam, axis=1) - np.linalg.norm(ov[both][:, :3] - cam, axis=1))
        assert np.mean(dz <= 1e-3) >= 0.999      # raycast depth within 1 mm where both hit
        cosang = np.sum(gn[both][:, :3] * on[both][:, :3], axis=1)
        assert np.mean(cosang > 0.999) >= 0.99


def test_compute_pose_vs_oracle(kf, orc, cuda, frames_small):
    cfg, imgs, poses = frames_small
    P = orc.Pipeline(cfg, prec=1)
    for i in range(4):
        P.process_frame(imgs[i])
    # the maps the oracle used in its last ICP (frame 3)
    vmaps = [P.vertex_map(l) for l in range(3)]
    pvs = [P.raycast_maps(l)[0] for l in range(3)]
    pns = [P.raycast_maps(l)[1] for l in range(3)]
    prev = orc.Pipeline(cfg, prec=1)
    for i in range(3):
        prev.process_frame(imgs[i])
    start = prev.pose()
    st_o, pose_o, it_o = orc.compute_pose(cfg, vmaps, pvs, pns, start, prec=1)
    st_g, pose_g, it_g = kf.ICP(cfg).computePose([dev(cuda, v) for v in vmaps], [dev(cuda, v) for v in pvs],
                                                  [dev(cuda, v) for v in pns], start)
    assert st_o == st_g == 0
    assert it_o == it_g
    a, d = kf.poseError(pose_o, pose_g)
    assert a <= 1e-4 and d <= 1e-4


def test_compute_pose_two_synthetic_frames_device(kf, orc, cuda):
    """TestComputePose (test/icp_tests.cpp:233-326) through the C ABI, on two synthetic frames
    in place of TUM fr1/xyz: a 0.15 rad / 0.32 m step of the loop trajectory, recovered within
    the reference's bounds (angle of R (1,1,1)/sqrt(3) <= pi / 90, translation within 0.01 m
    per axis).  The maps are the oracle's (test_oracle_golden.two_frame_case)."""
    from kfb200 import synth
    from test_oracle_golden import rotated_diagonal_angle, two_frame_case
    cfg, true, vb, va, na = two_frame_case(kf, orc, synth.LOOP, 3, 10, 11)
    st, est, _ = kf.ICP(cfg).computePose([dev(cuda, v) for v in vb], [dev(cuda, v) for v in va],
                                         [dev(cuda, v) for v in na], np.eye(4, dtype=np.float32))
    assert st == 0
    assert rotated_diagonal_angle(true[:3, :3], est[:3, :3]) <= PI / 90.0
    assert np.max(np.abs(true[:3, 3] - est[:3, 3])) <= 0.01


def test_bounded_wait_times_out_and_context_survives(kf, cuda):
    st, waited = kf.selftest_bounded_wait(50)
    assert st == kf.KF_ERR_TIMEOUT
    assert waited < 2000
    # the context is still usable
    x = cuda.ones(16, device="cuda")
    assert float((x * 2).sum()) == 32.0


def test_read_bandwidth_probe(kf):
    """The read-bandwidth probe runs and reports an L2-resident read rate above the HBM copy
    rate (64 MiB fits the L2), and rejects sizes outside its range."""
    import ctypes
    g = ctypes.c_double()
    assert kf.lib.kf_measure_read_bandwidth(64 << 20, 20, ctypes.byref(g)) == kf.KF_OK
    assert g.value > 3000.0, g.value
    assert kf.lib.kf_measure_read_bandwidth(1 << 20, 20, ctypes.byref(g)) == kf.KF_ERR_ARG
    assert kf.lib.kf_measure_read_bandwidth(64 << 20, 0, ctypes.byref(g)) == kf.KF_ERR_ARG
