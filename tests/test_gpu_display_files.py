"""Headless display kernels and kf_render against the oracle's restatement of the reference's
display math (project/src/display.cu:63-105); session checkpoints (TSDF .bin + pose + frame
index) resumed in a new session; a TUM-layout sequence read by RgbdDataset driving the
pipeline exactly like the same frames passed directly.

Display bound: every channel within 1 of the oracle (float rounding before the truncation to
8 bits), and at least 99% of pixels equal."""
import os
import tempfile

import numpy as np
import pytest

from test_files_and_datasets import write_png16

pytestmark = pytest.mark.gpu


def close_rgba(a, b):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= 1, d.max()
    assert np.mean(np.all(d == 0, axis=-1)) >= 0.99
    assert np.all(a[..., 3] == 255)


@pytest.fixture(scope="module")
def tracked(kf):
    from kfb200 import synth
    cfg = kf.config_small()
    imgs, _ = synth.sequence(cfg, 8, seed=51)
    s = kf.KinectFusion(cfg)
    for img in imgs[:6]:
        s.process_frame(img)
    return cfg, imgs, s


def test_display_kernels_vs_oracle(kf, orc, cuda, tracked):
    cfg, imgs, s = tracked
    _, nmap = s.raycast_maps(0)
    pose = s.pose()
    ik = np.linalg.inv(kf.level_intrinsics(cfg, 0).astype(np.float64)).astype(np.float32)
    nd = cuda.from_numpy(np.ascontiguousarray(nmap)).cuda()
    rgba = cuda.zeros((cfg.height, cfg.width, 4), dtype=cuda.uint8, device="cuda")
    kf.kernel.normalMapToWindowContent(nd, pose[:3, :3].T, rgba)
    close_rgba(rgba.cpu().numpy(), orc.display_normals(nmap, pose[:3, :3].T))
    kf.kernel.shadingToWindowContent(nd, pose, ik, rgba)
    close_rgba(rgba.cpu().numpy(), orc.display_shading(nmap, pose, ik))
    depth = cuda.from_numpy(s.depth(0)).cuda()
    kf.kernel.oneFloatChannelToWindowContent(depth, 100.0, rgba)
    g = rgba.cpu().numpy()
    expect = np.clip(np.floor(s.depth(0) * np.float32(100.0)), 0, 255).astype(np.uint8)
    np.testing.assert_array_equal(g[..., 0], expect)


def test_render_matches_raycast_and_display(kf, orc, cuda, tracked):
    cfg, imgs, s = tracked
    pose = s.pose()
    # the library's own K^-1: a ray direction one ulp apart moves a sample by ~1e-5 of a
    # voxel, enough to flip a 0.99 or 0 test near a surface
    ik = kf.level_inverse_intrinsics(cfg, 0)
    vt = cuda.zeros((cfg.height, cfg.width, 4), dtype=cuda.float32, device="cuda")
    nt = cuda.zeros_like(vt)
    kf.kernel.raycast(s.volume(), pose, ik, vt, nt, cfg.min_depth, cfg.max_depth, cfg.step_large, cfg.step_small)
    nmap = nt.cpu().numpy()
    assert np.mean(nmap[..., 3] == -1) > 0.2
    img = s.render(kf.KF_RENDER_NORMALS)
    close_rgba(img, orc.display_normals(nmap, pose[:3, :3].T))
    img = s.render(kf.KF_RENDER_SHADING)
    close_rgba(img, orc.display_shading(nmap, pose, ik))
    # a static view from the initial pose renders without disturbing tracking
    before = s.raycast_maps(0)[0].copy()
    s.render(kf.KF_RENDER_SHADING, pose=kf.start_pose(cfg.volume_width))
    np.testing.assert_array_equal(s.raycast_maps(0)[0], before)


def test_checkpoint_resume(kf, tracked):
    cfg, imgs, s0 = tracked
    from kfb200 import synth
    imgs, _ = synth.sequence(cfg, 9, seed=53)
    a = kf.KinectFusion(cfg)
    for img in imgs[:6]:
        a.process_frame(img)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "session.bin")
        a.saveCheckpoint(path)
        assert os.path.getsize(path) == cfg.volume_n ** 3 * 8
        b = kf.KinectFusion(cfg)
        b.loadCheckpoint(path)
        np.testing.assert_array_equal(b.tsdf()[0], a.tsdf()[0])
        np.testing.assert_array_equal(b.pose(), a.pose())
        for img in imgs[6:]:
            _, pa = a.process_frame(img)
            _, pb = b.process_frame(img)
            assert b.frame_stats()["icp_iters"] != [0, 0, 0]   # tracked, not a first frame
            ang, dist = kf.poseError(pa, pb)
            assert ang <= 1e-5 and dist <= 1e-5, (ang, dist)
        b.close()
    a.close()


def test_tum_sequence_drives_the_pipeline(kf, tracked):
    cfg, _, _ = tracked
    from kfb200 import synth
    imgs, poses = synth.sequence(cfg, 5, seed=57)
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "depth"))
        with open(os.path.join(d, "groundtruth.txt"), "w") as gt, open(os.path.join(d, "depth.txt"), "w") as dl:
            gt.write("#\n#\n#\n")
            dl.write("#\n#\n#\n")
            for k, (img, P) in enumerate(zip(imgs, poses)):
                t = 100.0 + 0.1 * k
                # rotation to a quaternion (x, y, z, w); the poses are proper rotations
                R = np.asarray(P, np.float64)[:3, :3]
                w = np.sqrt(max(0.0, 1.0 + R[0, 0] + R[1, 1] + R[2, 2])) / 2
                q = np.array([(R[2, 1] - R[1, 2]) / (4 * w), (R[0, 2] - R[2, 0]) / (4 * w),
                              (R[1, 0] - R[0, 1]) / (4 * w), w])
                gt.write("%.6f %.9f %.9f %.9f %.9f %.9f %.9f %.9f\n" % (t, *P[:3, 3], *q))
                rel = "depth/%d.png" % k
                write_png16(os.path.join(d, rel), img, (k % 5,))
                dl.write("%.6f %s\n" % (t + 0.001, rel))
        ds = kf.RgbdDataset(d)
        s1, s2 = kf.KinectFusion(cfg), kf.KinectFusion(cfg)
        for k in range(len(ds)):
            depth, gt_pose = ds.nextFrame(cfg.width, cfg.height)
            np.testing.assert_array_equal(depth, imgs[k])
            np.testing.assert_allclose(gt_pose, poses[k], atol=1e-5)
            _, p1 = s1.process_frame(depth)
            _, p2 = s2.process_frame(imgs[k])
            np.testing.assert_array_equal(p1, p2)
        s1.close()
        s2.close()


def test_visualization_volume(kf, orc, cuda):
    """The reference's second grid (project/src/kinect_fusion.cpp:19, :179-203): fused every frame
    at the frame's pose from the unfiltered depth, as the oracle fuses it (max over touched
    voxels but boundary flips within 1e-3 of its truncation); tracking is unchanged by it, bit for
    bit; kf_render raycasts it (the stage raycast of that volume plus the display kernel)."""
    import parity
    from kfb200 import synth
    cfg0 = kf.config_small()
    vn, vw = 128, 3.0
    cfg = kf.config_small(vis_volume_n=vn, vis_volume_width=vw, vis_mu=2.0 * vw / (vn - 1))
    imgs, _ = synth.sequence(cfg, 5, seed=55)
    xs, zs = orc.voxel_axes(vn, vw)
    plain = kf.KinectFusion(cfg0)
    s = kf.KinectFusion(cfg)
    for img in imgs:
        f0, w0 = s.vis_tsdf()
        _, pose = s.process_frame(img)
        np.testing.assert_array_equal(pose, plain.process_frame(img)[1])
        f1, w1 = s.vis_tsdf()
        fo, wo = f0.copy(), w0.copy()
        depth_m = orc.convert(img, cfg.depth_scale)
        orc.fuse(depth_m, kf.level_intrinsics(cfg, 0), fo, wo, vw, cfg.vis_mu, pose, prec=1)
        vcfg = kf.config_small(volume_n=vn, volume_width=vw, mu=cfg.vis_mu)
        t = parity.tsdf_frame_parity(vcfg, f0, w0, f1, w1, fo, wo, pose, depth_m, xs, zs)
        assert t["touched"] > 1000 and t["max_nonflip"] <= 1e-3, t
        assert t["boundary_flips"] <= 5e-3 * t["touched"], t
    np.testing.assert_array_equal(s.tsdf()[0], plain.tsdf()[0])   # the tracking volume is the same
    pose = s.pose()
    ik = kf.level_inverse_intrinsics(cfg, 0)
    vt = cuda.zeros((cfg.height, cfg.width, 4), dtype=cuda.float32, device="cuda")
    nt = cuda.zeros_like(vt)
    kf.kernel.raycast(s.vis_volume(), pose, ik, vt, nt, cfg.min_depth, cfg.max_depth, cfg.step_large, cfg.step_small)
    nmap = nt.cpu().numpy()
    assert np.mean(nmap[..., 3] == -1) > 0.2
    close_rgba(s.render(kf.KF_RENDER_SHADING), orc.display_shading(nmap, pose, ik))
    close_rgba(s.render(kf.KF_RENDER_NORMALS), orc.display_normals(nmap, pose[:3, :3].T))
    # saveTSDF / loadTSDF write and read the visualization grid, as the reference's do
    vf, vwt = s.vis_tsdf()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "vis.bin")
        s.saveTSDF(path)
        assert os.path.getsize(path) == vn ** 3 * 8
        other = kf.KinectFusion(cfg)
        other.loadTSDF(path)
        f2, w2 = other.vis_tsdf()
        np.testing.assert_array_equal(f2, vf)
        np.testing.assert_array_equal(w2, vwt)
        other.close()
    plain.close()
    s.close()
