"""End-to-end parity of the per-frame pipeline (kf_session, graph-replayed) against the CPU
oracle's restatement of KinectFusion::startTracking on the same seeded synthetic frames.

Per frame, the oracle starts from the device's state (TSDF and pose before the frame) and
both process the same frame; that isolates each frame's arithmetic from the way the
reference's algorithm amplifies tiny differences over a sequence (hard ICP rejections and a
1 cm early stop: the reference algorithm's own float and FP64 restatements differ by ~1e-4
after one frame on these scenes).  Free-running sequences are compared with a drift bound.

Bounds: per-frame pose within 1e-4 rad (rotation chord) / 1e-4 m of the FP64 oracle; depth
pyramid and valid-pixel masks equal, values within 2e-6 relative; ICP correspondence masks
agreeing on >= 99.9% of pixels; each frame's fusion within 1e-3 of the truncation distance
on every touched voxel but boundary flips (oracle/parity.py), which are at most 0.5 % of the
touched voxels; raycast depth within 1 mm on
every pixel both hit whose march took the same decisions, with decision flips at most 0.1 %
of the rays."""
import os
import tempfile

import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

NFRAMES = 10


def synced_frame(s, P, img):
    """Run one frame on the device and on the oracle from the device's state."""
    f, w = s.tsdf()
    P.set_tsdf(f, w)
    P.set_pose(s.pose())
    st_o, pose_o = P.process_frame(img)
    st_g, pose_g = s.process_frame(img)
    return st_g, st_o, pose_g, pose_o


@pytest.fixture(scope="module")
def run_small(kf, orc, cuda):
    from kfb200 import synth
    cfg = kf.config_small(export_icp_mask=1)
    imgs, gt = synth.sequence(cfg, NFRAMES, seed=33)
    xs, zs = orc.voxel_axes(cfg.volume_n, cfg.volume_width)
    s = kf.KinectFusion(cfg)
    s.set_debug(kf.KF_DEBUG_RAY_TRACE)
    P = orc.Pipeline(cfg, prec=1)
    rows = []
    for i, img in enumerate(imgs):
        f0, w0 = s.tsdf()
        cam = s.pose()[:3, 3].copy()
        st_g, st_o, pose_g, pose_o = synced_frame(s, P, img)
        # this frame's fusion by the oracle at the device's pose, from the same volume
        f1, w1 = s.tsdf()
        fo, wo = f0.copy(), w0.copy()
        depth_m = orc.convert(img, cfg.depth_scale)
        orc.fuse(depth_m, kf.level_intrinsics(cfg, 0), fo, wo, cfg.volume_width, cfg.mu, pose_g, prec=1)
        fusion = parity.tsdf_frame_parity(cfg, f0, w0, f1, w1, fo, wo, pose_g, depth_m, xs, zs)
        rays = [parity.raycast_parity(s.raycast_maps(l)[0], P.raycast_maps(l)[0], s.ray_trace(l), P.ray_trace(l),
                                      cam) for l in range(cfg.levels)] if i else []
        rows.append((st_g, st_o, pose_g, pose_o, s.frame_stats()["icp_iters"], P.iters(), fusion, rays))
    return cfg, imgs, s, P, rows


def test_pose_per_frame(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    for i, (st_g, st_o, pg, po, ig, io, _, _) in enumerate(rows):
        assert st_g == st_o == kf.KF_OK, i
        a, d = kf.poseError(po, pg)
        assert a <= 1e-4 and d <= 1e-4, (i, a, d, ig, io)


def test_free_running_drift(kf, orc):
    """Without re-synchronisation both runs follow the reference's algorithm; they may take
    a different number of ICP iterations where a step sits near the 1 cm stop threshold."""
    from kfb200 import synth
    cfg = kf.config_small()
    imgs, _ = synth.sequence(cfg, NFRAMES, seed=33)
    s = kf.KinectFusion(cfg)
    P = orc.Pipeline(cfg, prec=0)
    worst = 0.0
    for img in imgs:
        _, pg = s.process_frame(img)
        _, po = P.process_frame(img)
        worst = max(worst, *kf.poseError(po, pg))
    assert worst <= 3e-3, worst
    s.close()


def test_first_frame_fuses_only(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    assert rows[0][4] == [0, 0, 0]
    np.testing.assert_array_equal(rows[0][2], kf.start_pose(cfg.volume_width))


def test_pyramid_and_masks(kf, orc, run_small):
    cfg, imgs, s, P, rows = run_small
    np.testing.assert_array_equal(s.depth(-1), P.depth(-1))     # uint16 -> fp16 -> metres, bit exact
    for level in range(3):
        gd, od = s.depth(level), P.depth(level)
        np.testing.assert_array_equal(gd > 0.01, od > 0.01)
        v = od > 0.01
        np.testing.assert_allclose(gd[v], od[v], rtol=2e-6)
        gv, ov = s.vertex_map(level), P.vertex_map(level)
        np.testing.assert_array_equal(gv[..., 3], ov[..., 3])


def test_icp_masks(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    for level in range(3):
        agree = np.mean(s.icp_mask(level) == P.icp_mask(level))
        assert agree >= 0.999, (level, agree)


def test_raycast_maps(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    for i, row in enumerate(rows[1:], start=1):
        for level, p in enumerate(row[7]):
            assert p["hit_agreement"] >= 0.999, (i, level, p)
            assert p["both_hit_same_trace"] > 0, (i, level, p)
            assert p["max_mm_same_trace"] <= 1.0, (i, level, p)
            assert p["trace_flips"] <= 1e-3 * p["rays"], (i, level, p)


@pytest.mark.parametrize("volume_n,fmt", [(256, 0), (200, 0), (256, 1)], ids=["n256", "n200", "n256f16"])
def test_pipeline_raycast_equals_serial_stage(kf, cuda, volume_n, fmt):
    """The pipeline's march (cell skipping with runs of super-bricks, 40-iteration lane budget,
    long rays marched by a whole warp) takes the same samples as a plain serial march: compare
    with the stage raycast (no skipping, no hand-off) on the same volume and pose, with the
    library's K^-1.  n = 200 is a multiple of 8 but not of 32: its last super-bricks are
    partial, and their far faces are the volume's edges (which bound no skip)."""
    from kfb200 import synth
    cfg = kf.config_full(volume_n=volume_n, tsdf_format=fmt)
    imgs, _ = synth.sequence(cfg, 6, seed=41, kind=synth.LOOP)
    s = kf.KinectFusion(cfg)
    for img in imgs[:5]:
        s.process_frame(img)
    vol = s.volume()
    pose = s.pose()
    # the library's own K^-1 (a K^-1 one ulp apart is a different ray: it can move a sample
    # across 0.99 or 0 near a surface)
    ik = kf.level_inverse_intrinsics(cfg, 0)
    vt = cuda.zeros((cfg.height, cfg.width, 4), dtype=cuda.float32, device="cuda")
    nt = cuda.zeros_like(vt)
    kf.kernel.raycast(vol, pose, ik, vt, nt, cfg.min_depth, cfg.max_depth, cfg.step_large, cfg.step_small)
    sv, sn = vt.cpu().numpy(), nt.cpu().numpy()
    s.process_frame(imgs[5])              # its raycast runs on the same volume and pose
    gv, gn = s.raycast_maps(0)
    written = sv[..., 3] != 0
    assert (sv[..., 3] == -1).mean() > 0.05   # enough hits to compare (8 % at n = 200)
    # the same rays, the same samples: bit for bit wherever the stage raycast wrote
    np.testing.assert_array_equal(gv[written], sv[written])
    np.testing.assert_array_equal(gn[written], sn[written])
    s.close()


def test_tsdf(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    for i, row in enumerate(rows):
        t = row[6]
        assert t["touched"] > 10000, (i, t)
        assert t["max_nonflip"] <= 1e-3, (i, t)
        # the start pose looks straight down the volume's axes, where many voxel centres project
        # onto pixel edges exactly: about 0.13 % boundary flips on frame 0, a handful later
        assert t["boundary_flips"] <= 5e-3 * t["touched"], (i, t)
    gf, gw = s.tsdf()
    of, ow = P.tsdf()
    assert np.mean((gw > 0) == (ow > 0)) >= 0.9999


def test_tsdf_save_load_roundtrip(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    f, w = s.tsdf()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "tsdf.bin")
        s.saveTSDF(path)
        raw = np.fromfile(path, np.float32).reshape(cfg.volume_n, cfg.volume_n, cfg.volume_n, 2)
        np.testing.assert_array_equal(raw[..., 0], f)     # reference .bin layout: {f, w}, x fastest
        other = kf.KinectFusion(cfg)
        other.loadTSDF(path)
        f2, w2 = other.tsdf()
        np.testing.assert_array_equal(f2, f)
        np.testing.assert_array_equal(w2, w)
        other.close()


def test_nonfinite_keeps_pose_and_skips_fusion(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    pose0 = s.pose()
    f0, w0 = s.tsdf()
    st, pose = s.process_frame(np.zeros((cfg.height, cfg.width), np.uint16))   # no correspondences
    assert st == kf.KF_ERR_NONFINITE
    np.testing.assert_array_equal(pose, pose0)
    f1, w1 = s.tsdf()
    np.testing.assert_array_equal(f1, f0)
    assert s.frame_stats()["status"] == kf.KF_ERR_NONFINITE


def test_reset_replays_identically(kf, run_small):
    cfg, imgs, s, P, rows = run_small
    s.reset()
    for i in range(3):
        st, pose = s.process_frame(imgs[i])
        np.testing.assert_array_equal(pose, rows[i][2])


def test_device_input_path(kf, cuda, run_small):
    cfg, imgs, s, P, rows = run_small
    s2 = kf.KinectFusion(cfg)
    for i in range(3):
        d = cuda.from_numpy(imgs[i].view(np.int16)).cuda()
        st, pose = s2.process_frame(d)
        np.testing.assert_array_equal(pose, rows[i][2])
    s2.close()


def test_mixed_host_device_and_async_frames(kf, cuda, run_small):
    """A host frame's copy runs on a stream of its own beside the raycast; device frames
    (synchronous and queued) go through the session's stream.  Mixing them frame by frame
    gives the same poses and volume as host frames alone."""
    cfg, imgs, s, P, rows = run_small
    s2 = kf.KinectFusion(cfg)
    for i in range(6):
        if i % 3 == 0:
            st, pose = s2.process_frame(imgs[i])
        elif i % 3 == 1:
            st, pose = s2.process_frame(cuda.from_numpy(imgs[i].view(np.int16)).cuda())
        else:
            d = cuda.from_numpy(imgs[i].view(np.int16)).cuda()
            s2.process_frame_async(d)
            cuda.cuda.synchronize()
            pose = s2.pose()
        np.testing.assert_array_equal(pose, rows[i][2])
    s2.close()


def test_trunc8_compat_mode(kf, orc):
    from kfb200 import synth
    cfg = kf.config_small(compat_trunc8=1)
    imgs, _ = synth.sequence(cfg, 4, seed=35)
    s = kf.KinectFusion(cfg)
    P = orc.Pipeline(cfg, prec=1)
    for img in imgs:
        _, _, pg, po = synced_frame(s, P, img)
        a, d = kf.poseError(po, pg)
        assert a <= 1e-4 and d <= 1e-4
    # level 2 of 320x240 is 80x60: the reference's 8x8 grid never writes rows 56-59
    assert np.all(s.depth(2)[56:] == 0) and np.all(s.vertex_map(2)[56:, :, 3] == 0)
    s.close()


def test_f16u16_precision_form_vs_fp64(kf, orc):
    """FP16 distance + uint16 weight volume against the FP64 oracle (float volume): per frame
    from the device's state, pose within 1e-4 and the frame's fused TSDF within fp16 / weight
    quantisation (RMS below 1e-3 of the truncation distance)."""
    from kfb200 import synth
    cfg16 = kf.config_small(tsdf_format=kf.KF_TSDF_F16U16)
    cfg = kf.config_small()
    imgs, _ = synth.sequence(cfg, 8, seed=37)
    s = kf.KinectFusion(cfg16)
    P = orc.Pipeline(cfg, prec=1)
    for img in imgs:
        _, _, pg, po = synced_frame(s, P, img)
        a, d = kf.poseError(po, pg)
        assert a <= 1e-4 and d <= 1e-4
    gf, gw = s.tsdf()
    of, ow = P.tsdf()
    obs = (ow > 0) & (gw > 0)
    assert np.mean((ow > 0) == (gw > 0)) >= 0.999
    rms = np.sqrt(np.mean((gf[obs] - of[obs]) ** 2))
    assert rms < 1e-3
    s.close()


def test_bilateral_radius_zero_and_single_level(kf, orc):
    from kfb200 import synth
    cfg = kf.config_small(levels=1, iters=(6, 0, 0), bilateral_radius=0)
    imgs, _ = synth.sequence(cfg, 3, seed=39)
    s = kf.KinectFusion(cfg)
    P = orc.Pipeline(cfg, prec=1)
    for img in imgs:
        _, _, pg, po = synced_frame(s, P, img)
        a, d = kf.poseError(po, pg)
        assert a <= 1e-4 and d <= 1e-4
    np.testing.assert_allclose(s.depth(0), s.depth(-1), rtol=0)   # a 1x1 window is the identity
    s.close()


def test_debug_modes_change_no_result(kf, run_small):
    """Plain launches per stage (KF_DEBUG_NO_GRAPH, the mode for profiling a stage), the
    decision-trace recording and the raycast's counting kernels give the same poses as the
    replayed graph, bit for bit."""
    cfg, imgs, s, P, rows = run_small
    s2 = kf.KinectFusion(cfg)
    s2.set_debug(kf.KF_DEBUG_NO_GRAPH | kf.KF_DEBUG_RAY_TRACE | kf.KF_DEBUG_COUNTERS)
    for i in range(5):
        st, pose = s2.process_frame(imgs[i])
        np.testing.assert_array_equal(pose, rows[i][2])
        c = s2.debug_counts()
        if i == 0:
            assert c["rays"] == 0   # the first frame fuses only
        else:
            # every pixel of every level marches; samples are evaluated, skipped or taken by warps
            assert 0 < c["rays"] <= sum((cfg.width >> l) * (cfg.height >> l) for l in range(cfg.levels))
            assert c["eval_large"] + c["eval_small"] > c["rays"] and c["skips"] > 0 and c["gradient"] % 6 == 0
    s2.set_debug(0)
    st, pose = s2.process_frame(imgs[5])
    np.testing.assert_array_equal(pose, rows[5][2])
    with pytest.raises(kf.KfError):
        s2.ray_trace(0)   # recording is off again
    s2.close()


def test_submitted_frames_equal_synchronous_frames(kf, cuda, run_small):
    """Frames queued with kf_process_frame_submit (host and device frames, up to the in-flight
    limit ahead) give the poses of kf_process_frame, bit for bit, in order; one frame beyond the
    limit is refused, and a synchronous call waits for the queue to be collected."""
    cfg, imgs, s, P, rows = run_small
    s2 = kf.KinectFusion(cfg)
    pinned = [cuda.from_numpy(im.view(np.int16)).pin_memory() for im in imgs]
    host = [p.numpy().view(np.uint16) for p in pinned]
    depth = kf._lib.KF_MAX_FRAMES_IN_FLIGHT
    got, nxt = [], 0
    for _ in range(depth):
        s2.submit_frame(host[nxt] if nxt % 2 == 0 else cuda.from_numpy(imgs[nxt].view(np.int16)).cuda())
        nxt += 1
    with pytest.raises(kf.KfError) as e:
        s2.submit_frame(host[nxt])
    assert e.value.status == kf.KF_ERR_CAPACITY
    with pytest.raises(kf.KfError) as e:
        s2.process_frame(host[nxt])
    assert e.value.status == kf.KF_ERR_STATE
    while len(got) < len(imgs):
        got.append(s2.wait_frame()[1])
        if nxt < len(imgs):
            s2.submit_frame(host[nxt])
            nxt += 1
    for i, pose in enumerate(got):
        np.testing.assert_array_equal(pose, rows[i][2])
    assert s2.frame_stats()["frame"] == len(imgs) - 1
    st, pose = s2.process_frame(host[0])   # the queue is empty again
    s2.close()
