"""The library against the reference's own pipeline, compiled from the reference's sources on
this machine (oracle/_ref/libkfref.so through oracle/refpipe.py): the reference's kernels, its
ICP::computePose with cuBLAS and Eigen, and its VoxelGrid run on the same GPU, on the same
seeded frames.  Both use the reference's constants (640 x 480, fx = fy = 525, bilateral 4 px /
0.25 m / 7 x 7, mu = 3 voxels, ICP 10/5/3 at 0.4 m / 40 degrees with its early stop; a 512^3
f32 volume over 3 m).  Synced per frame: the reference and the FP64 oracle start each frame from
the library's volume and pose.

Bounds:
  - converted depth, the filtered and down-sampled depth of every level and the vertex maps,
    bit for bit (the library computes the pyramid with the reference's Release float
    semantics);
  - ICP correspondence masks (first pass of every level, same poses) agree on >= 99.9 % of
    pixels;
  - fusing the frame at the same pose: within 1e-3 of the truncation distance on every touched
    voxel except boundary flips, which are at most 1e-4 of the touched voxels;
  - raycast: hits agree on >= 99.9 % of pixels.  Where both hit, the depth is within 1 mm,
    except on pixels where the reference's own depth is more than 1 mm from the FP64 oracle's
    (at most 1 % of those may fall outside).  Hardware texture filtering, which the reference's
    raycast samples through (project/src/raycast.cu:87, voxel_grid.cpp:35-42), keeps 8
    fractional bits of the interpolation weights, and that moves 0.99 / 0 decisions; the
    library's trilinear interpolation is exact float arithmetic and follows the FP64 oracle to
    <= 1 mm on all but 1e-4 of the pixels.
  - pose: within 1e-4 rad / 1e-4 m of the FP64 oracle, and no farther from the reference's pose
    than the reference is from the FP64 oracle, plus 1e-4."""
import pytest

import refpipe

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpipe.available(), reason="the reference harness is not built here")]

NFRAMES = 4


@pytest.fixture(scope="module")
def ref_run(kf, orc, cuda):
    from kfb200 import synth
    cfg = refpipe.matching_config(kf, depth_scale=1e-3, volume_n=512, volume_width=3.0,
                                  initial_pose=kf.start_pose(3.0), vis_volume_n=0, keep_on_miss=0)
    imgs, _ = synth.sequence(cfg, NFRAMES, seed=3, kind=synth.LOOP)
    return cfg, refpipe.compare_synced(kf, orc, cuda, cfg, imgs)


def test_pyramid_bit_exact_vs_reference(ref_run):
    cfg, rows = ref_run
    for r in rows:
        assert r["meters"], r["frame"]
        for l, (depth_eq, vertex_eq) in enumerate(r.get("pyramid", [])):
            assert depth_eq and vertex_eq, (r["frame"], l, depth_eq, vertex_eq)


def test_icp_masks_vs_reference(ref_run):
    cfg, rows = ref_run
    for r in rows[1:]:
        for l, agree in enumerate(r["icp_masks"]):
            assert agree >= 0.999, (r["frame"], l, agree)


def test_fusion_vs_reference(ref_run):
    cfg, rows = ref_run
    for r in rows:
        t = r["tsdf"]
        assert t["touched"] > 100000, (r["frame"], t)
        assert t["max_nonflip"] <= 1e-3, (r["frame"], t)
        assert t["boundary_flips"] <= 1e-4 * t["touched"], (r["frame"], t)


def test_raycast_vs_reference(ref_run):
    cfg, rows = ref_run
    for r in rows[1:]:
        for p in r["rays"]:
            assert p["hit_agreement"] >= 0.999, (r["frame"], p)
            assert p["both"] > 0.1 * (cfg.width >> p["level"]) * (cfg.height >> p["level"]), (r["frame"], p)
            # every >1 mm difference from the reference but a few sits where the reference is
            # itself >1 mm from the FP64 oracle
            assert p["unexplained"] <= max(2, 0.01 * p["lib_ref_over_1mm"]), (r["frame"], p)
            # and the library follows the FP64 oracle
            assert p["lib_fp64_over_1mm"] <= 1e-4 * p["lib_fp64_both"] + 1, (r["frame"], p)


def test_pose_vs_reference(kf, ref_run):
    cfg, rows = ref_run
    for r in rows[1:]:
        assert r["st"][0] == r["st"][1] == kf.KF_OK and r["st_ref"] == refpipe.OK, (r["frame"], r["st"], r["st_ref"])
        p = r["pose"]
        assert p["lib_fp64"][0] <= 1e-4 and p["lib_fp64"][1] <= 1e-4, (r["frame"], p)
        assert p["lib_ref"][0] <= p["ref_fp64"][0] + 1e-4, (r["frame"], p)
        assert p["lib_ref"][1] <= p["ref_fp64"][1] + 1e-4, (r["frame"], p)
