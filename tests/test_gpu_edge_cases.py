"""Edge cases of the frame pipeline against the FP64 oracle, synced per frame (the oracle starts
from the device's TSDF and pose): frame sizes that are not multiples of the 32-pixel
preprocess tiles or the 8 x 4 ray tiles, volumes that are not multiples of the 32-voxel
lanes and super-bricks, a two-level pyramid, the Kinect unmirror path, a large frame, an
empty first frame, and mixed batches equal to their sessions run alone.

Bounds as in test_gpu_session.py: pose within 1e-4 rad / 1e-4 m per frame, valid-pixel masks
equal, TSDF within 1e-3 of the truncation distance on >= 99.9% of voxels."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def synced_run(kf, orc, cfg, imgs):
    s = kf.KinectFusion(cfg)
    P = orc.Pipeline(cfg, prec=1)
    for img in imgs:
        f, w = s.tsdf()
        P.set_tsdf(f, w)
        P.set_pose(s.pose())
        st_o, _ = P.process_frame(img)
        st_g, _ = s.process_frame(img)
        assert st_g == st_o
        a, d = kf.poseError(P.pose(), s.pose())
        assert a <= 1e-4 and d <= 1e-4, (a, d, s.frame_stats(), P.iters())
    for level in range(cfg.levels):
        np.testing.assert_array_equal(s.depth(level) > 0.01, P.depth(level) > 0.01)
        np.testing.assert_array_equal(s.vertex_map(level)[..., 3], P.vertex_map(level)[..., 3])
    gf, gw = s.tsdf()
    of, ow = P.tsdf()
    assert np.mean(np.abs(gf - of) <= 1e-3) >= 0.999
    return s, P


def small_cfg(kf, w, h, n, **kw):
    return kf.config_small(width=w, height=h, cx=(w - 1) / 2.0, cy=(h - 1) / 2.0, volume_n=n, **kw)


def test_ragged_frame_and_volume(kf, orc):
    from kfb200 import synth
    # 324 x 244: not a multiple of 32 (preprocess tiles) nor of 8 (ray tiles at level 2: 81 x 61);
    # 136^3: x rows of 136 leave 8 lanes of the last fusion warp idle, super-bricks are partial
    cfg = small_cfg(kf, 324, 244, 136)
    imgs, _ = synth.sequence(cfg, 5, seed=71)
    s, P = synced_run(kf, orc, cfg, imgs)
    s.close()


def test_two_level_pyramid(kf, orc):
    from kfb200 import synth
    cfg = kf.config_small(levels=2, iters=(6, 4, 0))
    imgs, _ = synth.sequence(cfg, 5, seed=73)
    s, P = synced_run(kf, orc, cfg, imgs)
    assert s.frame_stats()["icp_iters"][2] == 0
    s.close()


def test_unmirror(kf, orc):
    from kfb200 import synth
    cfg = kf.config_small(unmirror=1)
    imgs, _ = synth.sequence(cfg, 4, seed=75)
    s, P = synced_run(kf, orc, cfg, imgs)
    # the unfiltered metres map is the mirrored fp16-value conversion, bit for bit
    np.testing.assert_array_equal(s.depth(-1), orc.convert(imgs[-1], cfg.depth_scale, unmirror=True))
    s.close()


def test_large_frame(kf, orc):
    from kfb200 import synth
    w, h = 1280, 960
    cfg = kf.config_full(width=w, height=h, fx=1050.0, fy=1050.0, cx=(w - 1) / 2.0, cy=(h - 1) / 2.0,
                         volume_n=256)
    imgs, _ = synth.sequence(cfg, 3, seed=77)
    s, P = synced_run(kf, orc, cfg, imgs)
    s.close()


def test_empty_first_frame(kf):
    """Frame 0 fuses only; an all-zero frame 0 leaves the grid empty, so frame 1 has nothing to
    track against: ICP finds no correspondences, the pose is kept and nothing is fused (the
    reference throws here, project/src/icp.cpp:67-73)."""
    from kfb200 import synth
    cfg = kf.config_small()
    imgs, _ = synth.sequence(cfg, 2, seed=79)
    s = kf.KinectFusion(cfg)
    st, p0 = s.process_frame(np.zeros((cfg.height, cfg.width), np.uint16))
    assert st == kf.KF_OK
    f, w = s.tsdf()
    assert np.all(w == 0) and np.all(f == 2.0)
    st, p1 = s.process_frame(imgs[1])
    assert st == kf.KF_ERR_NONFINITE
    np.testing.assert_array_equal(p1, p0)
    assert np.all(s.tsdf()[1] == 0)
    s.close()


def test_ragged_batch_equals_alone(kf):
    from kfb200 import synth
    cfgs = [small_cfg(kf, 324, 244, 136), kf.config_small(levels=2, iters=(6, 4, 0)),
            small_cfg(kf, 200, 148, 96, tsdf_format=kf.KF_TSDF_F16U16)]
    seqs = [synth.sequence(c, 4, seed=81 + i)[0] for i, c in enumerate(cfgs)]
    b = kf.Batch(cfgs)
    alone = [kf.KinectFusion(c) for c in cfgs]
    for k in range(4):
        frames = [seqs[i][k] if (k + i) % 3 else None for i in range(len(cfgs))]   # uneven arrivals
        _, poses = b.step(frames)
        for i, f in enumerate(frames):
            if f is None:
                continue
            _, p = alone[i].process_frame(f)
            np.testing.assert_array_equal(poses[i], p)
    for i in range(len(cfgs)):
        np.testing.assert_array_equal(b.session(i).tsdf()[0], alone[i].tsdf()[0])
        alone[i].close()
    b.close()
