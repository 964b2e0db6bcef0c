"""The plain pipeline at its full size (640x480 frames, a 512^3 volume over 3 m, mu 0.02 m,
ICP 4/5/10) against the FP64 oracle, frame by frame from the device's state, in both volume
formats (f32 + f32, and the precision form's fp16 + uint16), on the start of the full-size
300-frame loop; plus properties that hold at any size: fusing nothing (an all-invalid frame)
leaves the volume bit for bit unchanged.

Bounds:
  - pose within 1e-4 rad / 1e-4 m of the FP64 oracle per frame, with the same ICP iteration
    counts;
  - raycast depth within 1 mm at every level, as a maximum over the pixels both hit whose march
    took the same decisions (equal decision traces); rays whose decisions differ (a sample
    within rounding of 0.99 or 0) are at most 0.1 % of the marched rays;
  - the frame's fusion (the oracle fusing the same frame at the device's pose) within 1e-3 of
    the truncation distance, as a maximum over every voxel the frame touched except boundary
    flips (a projection within rounding of a pixel edge, the depth range or the -mu limit),
    which are at most 1e-4 of the touched voxels."""
import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

NFRAMES = 4


@pytest.fixture(scope="module", params=[0, 1], ids=["f32f32", "f16u16"])
def full_run(request, kf, orc):
    from kfb200 import synth
    cfg = kf.config_full(tsdf_format=request.param)
    imgs, _ = synth.sequence(cfg, NFRAMES, seed=3, kind=synth.LOOP)
    xs, zs = orc.voxel_axes(cfg.volume_n, cfg.volume_width)
    s = kf.KinectFusion(cfg)
    s.set_debug(kf.KF_DEBUG_RAY_TRACE)
    P = orc.Pipeline(cfg, prec=1)
    rows = []
    for img in imgs:
        f0, w0 = s.tsdf()
        P.set_tsdf(f0, w0)
        P.set_pose(s.pose())
        cam = s.pose()[:3, 3].copy()   # the frame's raycast runs at the previous frame's pose
        st_o, pose_o = P.process_frame(img)
        st_g, pose_g = s.process_frame(img)
        f1, w1 = s.tsdf()
        # the frame's fusion alone, at the device's final pose (the two ICPs' poses differ by up
        # to 1e-4 m, i.e. 5e-3 of the 2 cm truncation near surfaces)
        fo, wo = f0.copy(), w0.copy()
        depth_m = orc.convert(img, cfg.depth_scale)
        orc.fuse(depth_m, kf.level_intrinsics(cfg, 0), fo, wo, cfg.volume_width, cfg.mu, pose_g, prec=1)
        tsdf = parity.tsdf_frame_parity(cfg, f0, w0, f1, w1, fo, wo, pose_g, depth_m, xs, zs)
        rays = []
        if len(rows):
            for level in range(cfg.levels):
                gv, _ = s.raycast_maps(level)
                ov, _ = P.raycast_maps(level)
                rays.append(parity.raycast_parity(gv, ov, s.ray_trace(level), P.ray_trace(level), cam))
        rows.append(dict(st=(st_g, st_o), pose=(pose_g, pose_o), iters=(s.frame_stats()["icp_iters"], P.iters()),
                         tsdf=tsdf, rays=rays))
        del f0, w0, f1, w1, fo, wo
    yield cfg, imgs, s, rows
    s.close()
    P.close()


def test_full_size_pose_per_frame(kf, full_run):
    cfg, imgs, s, rows = full_run
    for i, r in enumerate(rows):
        assert r["st"][0] == r["st"][1] == kf.KF_OK, i
        a, d = kf.poseError(r["pose"][1], r["pose"][0])
        assert a <= 1e-4 and d <= 1e-4, (i, a, d)
        assert list(r["iters"][0]) == list(r["iters"][1]), (i, r["iters"])


def test_full_size_tsdf(full_run):
    cfg, imgs, s, rows = full_run
    for i, r in enumerate(rows):
        t = r["tsdf"]
        assert t["touched"] > 100000, (i, t)
        assert t["max_nonflip"] <= 1e-3, (i, t)
        assert t["boundary_flips"] <= 1e-4 * t["touched"], (i, t)


def test_full_size_raycast_depth(full_run):
    cfg, imgs, s, rows = full_run
    for i, r in enumerate(rows[1:], start=1):
        for level, p in enumerate(r["rays"]):
            assert p["hit_agreement"] >= 0.999, (i, level, p)
            assert p["both_hit_same_trace"] > 0.1 * (cfg.width >> level) * (cfg.height >> level), (i, level, p)
            assert p["max_mm_same_trace"] <= 1.0, (i, level, p)
            assert p["trace_flips"] <= 1e-3 * p["rays"], (i, level, p)


def test_full_size_invalid_frame_changes_nothing(kf, full_run):
    """A frame with no valid depth: ICP finds no correspondences (the reference throws on the
    singular system and keeps the pose), nothing is fused, and the volume is unchanged."""
    cfg, imgs, s, rows = full_run
    f0, w0 = s.tsdf()
    pose0 = s.pose()
    st, pose = s.process_frame(np.zeros((cfg.height, cfg.width), np.uint16))
    assert st in (kf.KF_OK, kf.KF_ERR_NONFINITE)
    f1, w1 = s.tsdf()
    np.testing.assert_array_equal(w1, w0)
    np.testing.assert_array_equal(f1, f0)
    if st == kf.KF_ERR_NONFINITE:
        np.testing.assert_array_equal(pose, pose0)
