"""The plain pipeline at its full size (640x480 frames, a 512^3 f32 volume over 3 m, mu 0.02 m,
ICP 4/5/10) against the FP64 oracle, frame by frame from the device's state, plus properties
that hold at any size: fusing nothing (an all-invalid frame) leaves the volume bit for bit
unchanged.

Bounds as for the small configuration: pose within 1e-4 rad / 1e-4 m per frame, the same ICP
iteration counts, raycast depth within 1 mm on >= 99.9 % of pixels where both hit, and the
frame's fusion (the oracle fusing the same frame at the device's pose) within 1e-3 of the
truncation distance on >= 99.9 % of the voxels the frame touched."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NFRAMES = 4


@pytest.fixture(scope="module")
def full_run(kf, orc):
    from kfb200 import synth
    cfg = kf.config_full()
    imgs, _ = synth.sequence(cfg, NFRAMES, seed=3, kind=synth.LOOP)
    s = kf.KinectFusion(cfg)
    P = orc.Pipeline(cfg, prec=1)
    rows = []
    for img in imgs:
        f0, w0 = s.tsdf()
        P.set_tsdf(f0, w0)
        P.set_pose(s.pose())
        st_o, pose_o = P.process_frame(img)
        st_g, pose_g = s.process_frame(img)
        f1, w1 = s.tsdf()
        # the frame's fusion alone, at the device's final pose (the two ICPs' poses differ by up
        # to 1e-4 m, i.e. 5e-3 of the 2 cm truncation near surfaces)
        fo, wo = f0.copy(), w0.copy()
        orc.fuse(orc.convert(img, cfg.depth_scale), kf.level_intrinsics(cfg, 0), fo, wo, cfg.volume_width, cfg.mu,
                 pose_g, prec=1)
        touched = (w1 != w0) | (wo != w0)
        tsdf_ok = float(np.mean(np.abs(f1[touched] - fo[touched]) <= 1e-3)) if touched.any() else 1.0
        rays = []
        for level in range(cfg.levels):
            gv, _ = s.raycast_maps(level)
            ov, _ = P.raycast_maps(level)
            rays.append((gv, ov))
        rows.append(dict(st=(st_g, st_o), pose=(pose_g, pose_o), iters=(s.frame_stats()["icp_iters"], P.iters()),
                         tsdf_ok=tsdf_ok, touched=int(touched.sum()), rays=rays, cam=pose_g[:3, 3].copy()))
        del f0, w0, f1, w1, fo, wo, touched
    yield cfg, imgs, s, rows
    s.close()


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
        assert r["touched"] > 100000, (i, r["touched"])
        assert r["tsdf_ok"] >= 0.999, (i, r["tsdf_ok"])


def test_full_size_raycast_depth(full_run):
    cfg, imgs, s, rows = full_run
    for i, r in enumerate(rows[1:], start=1):
        cam = rows[i - 1]["cam"]   # a frame's raycast runs at the previous frame's pose
        for level, (gv, ov) in enumerate(r["rays"]):
            gh, oh = gv[..., 3] == -1, ov[..., 3] == -1
            assert np.mean(gh == oh) >= 0.999, (i, level)
            both = gh & oh
            assert both.mean() > 0.1, (i, level)
            dz = np.abs(np.linalg.norm(gv[both][:, :3] - cam, axis=1) - np.linalg.norm(ov[both][:, :3] - cam, axis=1))
            assert np.mean(dz <= 1e-3) >= 0.999, (i, level, float(np.percentile(dz, 99.9)))


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
