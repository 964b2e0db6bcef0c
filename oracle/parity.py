"""TEST INFRASTRUCTURE ONLY: how the CUDA library's maps and volume are compared with the oracle.

The reference's algorithm has hard decisions on float values: the raycast leaves large steps at
the first sample below 0.99 and refines at the first negative one
(project/src/raycast.cu:90-117), and fusion reads the depth pixel its projection truncates to
and updates only voxels with d - z >= -mu (project/src/tsdf.cu:40-58).  A sample or a
projection within a rounding error of such a threshold can decide differently in float and in
FP64: the reference's own float code and the FP64 oracle differ there too.  So the comparisons
below separate

  - rays whose march took the same decisions in both (equal decision traces: the samples at
    which large steps ended and the march ended, and how), whose hits may differ by rounding
    only, from rays where a sample near 0.99 or 0 decided otherwise (a "flip"); and
  - voxels whose projection lies within rounding of a pixel edge, the depth range or the
    -mu update limit (a boundary flip) from all others.

Bounds are then stated as maxima over the agreeing rays / non-flip voxels, with the flips
counted.  Only tests/ and bench.py's accuracy block use this module.
"""
import numpy as np

# how close to a threshold a projection must be for float and FP64 to disagree on it
PIXEL_EDGE_EPS = 1e-3     # pixels (float projection error at 640 px is ~1e-4 px)
DEPTH_EDGE_EPS = 1e-5     # metres


def same_decisions(a, b):
    """Elementwise: two decision traces (march_trace encoding) describe the same decisions.
    Rays that both ran to the far plane without a hit decided the same (a miss) whatever the
    number of samples: the last sample before the far plane is a rounding away from it."""
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    head = np.int64(~((1 << 40) - 1)) | np.int64(0xff)   # switch sample, switch mode, end
    exhausted = ((a & 3) == 0) & ((b & 3) == 0)
    return (a == b) | (exhausted & ((a & head) == (b & head)))


def raycast_parity(gv, ov, gtr, otr, cam):
    """Device maps (gv, traces gtr) against the oracle's (ov, otr) at one level; cam: the
    camera centre the raycast ran from.  Depth error is the difference of distances to the
    camera, in mm.  Returns a dict of counts and maxima."""
    gh, oh = gv[..., 3] == -1, ov[..., 3] == -1
    marched = (gtr != 0) | (otr != 0)
    same = same_decisions(gtr, otr)
    both = gh & oh
    agree = both & same
    cam = np.asarray(cam, np.float64)

    def mm(mask):
        if not mask.any():
            return np.zeros(0)
        a = np.linalg.norm(gv[mask][:, :3].astype(np.float64) - cam, axis=1)
        b = np.linalg.norm(ov[mask][:, :3].astype(np.float64) - cam, axis=1)
        return np.abs(a - b) * 1e3

    dz_agree, dz_all = mm(agree), mm(both)
    return {
        "rays": int(marched.sum()),
        "trace_flips": int((marched & ~same).sum()),
        "hit_agreement": float(np.mean(gh == oh)),
        "both_hit": int(both.sum()),
        "both_hit_same_trace": int(agree.sum()),
        "max_mm_same_trace": float(dz_agree.max()) if dz_agree.size else 0.0,
        "max_mm_all": float(dz_all.max()) if dz_all.size else 0.0,
        "over_1mm_flipped": int((dz_all > 1.0).sum()),
    }


def voxel_projection(cfg, pose, xs, zs, idx):
    """FP64 projection of voxels idx = (k, j, i) (z, y, x indices) into the frame of `pose`
    (camera->world 4x4): camera-frame z and pixel coordinates, as fuseKernel forms them."""
    k, j, i = idx
    p = np.stack([xs[i], xs[j], zs[k]], axis=1).astype(np.float64)
    R = np.asarray(pose, np.float64)[:3, :3]
    t = np.asarray(pose, np.float64)[:3, 3]
    pe = (p - t) @ R   # R^T (p - t), row-wise
    px = cfg.fx * pe[:, 0] / pe[:, 2] + cfg.cx
    py = cfg.fy * pe[:, 1] / pe[:, 2] + cfg.cy
    return pe[:, 2], px, py


def tsdf_frame_parity(cfg, f0, w0, fg, wg, fo, wo, pose, depth_m, xs, zs, tol=1e-3):
    """One frame's fusion: the device went from (f0, w0) to (fg, wg), the oracle fusing the same
    frame at the same pose from (f0, w0) to (fo, wo); arrays (n, n, n) indexed [z, y, x],
    distances in units of the truncation distance.  Voxels whose |fg - fo| exceeds tol are
    boundary flips when their FP64 projection is within rounding of a pixel edge, of the
    [min, max) depth range or of the d - z = -mu update limit.  Returns counts and maxima."""
    touched = (wg != w0) | (wo != w0)
    diff = np.abs(fg.astype(np.float64) - fo.astype(np.float64))
    d_t = diff[touched]
    bad = np.nonzero(touched & (diff > tol))
    flips = np.zeros(len(bad[0]), bool)
    if len(bad[0]):
        z, px, py = voxel_projection(cfg, pose, xs, zs, bad)
        fx, fy = px - np.floor(px), py - np.floor(py)
        edge = (np.minimum(fx, 1 - fx) < PIXEL_EDGE_EPS) | (np.minimum(fy, 1 - fy) < PIXEL_EDGE_EPS)
        edge |= (np.abs(z - cfg.min_depth) < DEPTH_EDGE_EPS) | (np.abs(z - cfg.max_depth) < DEPTH_EDGE_EPS)
        inside = (px >= 0) & (px < cfg.width) & (py >= 0) & (py < cfg.height)
        u = np.clip(px.astype(np.int64), 0, cfg.width - 1)
        v = np.clip(py.astype(np.int64), 0, cfg.height - 1)
        d = depth_m[v, u].astype(np.float64)
        edge |= inside & (np.abs(d - z + cfg.mu) < DEPTH_EDGE_EPS)
        flips = edge
    nonflip = np.ones(diff.shape, bool)
    nonflip[tuple(a[flips] for a in bad)] = False
    d_nf = diff[touched & nonflip]
    return {
        "touched": int(touched.sum()),
        "max_all": float(d_t.max()) if d_t.size else 0.0,
        "max_nonflip": float(d_nf.max()) if d_nf.size else 0.0,
        "over_tol": int(len(bad[0])),
        "boundary_flips": int(flips.sum()),
    }
