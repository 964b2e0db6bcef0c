"""TEST INFRASTRUCTURE ONLY: ctypes binding of the reference's own pipeline (oracle/_ref/libkfref.so).

The library is the reference's compute code (project/src: measurement.cu, raycast.cu, tsdf.cu,
icp.cu, icp.cpp, linear_least_squares.cpp, voxel_grid.cpp, ...) compiled from its sources by
oracle/Makefile, with ref_harness.cpp restating KinectFusion::startTracking's compute calls
(project/src/kinect_fusion.cpp:44-73) over it.  It runs the reference's kernels on the GPU.
It is built only where a reference checkout exists, and travels with the repository's other
built files; `available()` says whether it is here.  Only tests/ and bench.py's reference arm
load this module; the product never does.

The reference hard-codes a 640 x 480 frame with the principal point at (319.5, 239.5)
(project/src/sensor.h:14-16, tsdf.cu:40), three pyramid levels, the bilateral filter's
sigma_s = 4 px, sigma_r = 0.25 m and 7 x 7 window (measurement.cu:11-12, :38), the sensor range
0.4 - 6 m (tsdf.cuh:11-12) and the raycast steps 1.99 / 0.1 mu (raycast.cu:75-76); a library
session compared with it uses the same values (`matching_config`).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libkfref.so")
W, H, LEVELS = 640, 480, 3

_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_SIG = {
    "kfref_create": (_P, [_I, _F, _F, _F, _F, _P, _F, _F, _F, _F, _I, _F, _F]),
    "kfref_destroy": (None, [_P]),
    "kfref_set_pose": (_I, [_P, _P]),
    "kfref_get_pose": (_I, [_P, _P]),
    "kfref_upload": (_I, [_P, _P]),
    "kfref_convert": (_I, [_P]),
    "kfref_preprocess": (_I, [_P]),
    "kfref_raycast": (_I, [_P]),
    "kfref_compute_pose": (_I, [_P]),
    "kfref_fuse": (_I, [_P]),
    "kfref_visualize": (_I, [_P]),
    "kfref_process_frame": (_I, [_P, _P]),
    "kfref_time_frames": (_I, [_P, _P, _I, _I, _P, _P]),
    "kfref_stage_times": (_I, [_P, _P]),
    "kfref_frames": (_I, [_P]),
    "kfref_set_frames": (_I, [_P, _I]),
    "kfref_get_map": (_I, [_P, _I, _I, _P]),
    "kfref_clear_raycast_maps": (_I, [_P]),
    "kfref_get_tsdf": (_I, [_P, _I, _P]),
    "kfref_set_tsdf": (_I, [_P, _I, _P]),
    "kfref_icp_residuals": (_I, [_P, _I, _P, _P, _F, _F, _P, _P]),
    "kfref_pose_error": (_I, [_P, _P, _P]),
    "kfref_tum_open": (_P, [ctypes.c_char_p]),
    "kfref_tum_close": (None, [_P]),
    "kfref_tum_next": (_I, [_P, ctypes.c_char_p, _I, _P]),
    "kfref_tum_initial_pose_inverse": (_I, [_P, _P]),
    "kfref_sensor_intrinsics": (_I, [_F, _I, _P, _P]),
}
OK, NONFINITE, CUDA_ERROR, BAD_ARG = 0, 1, 2, 3


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("the reference harness is not built (oracle/_ref/libkfref.so): run make -C oracle "
                               "where a reference checkout exists")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIG.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _cm(pose):
    """4 x 4 matrix -> 16 column-major float32."""
    return np.ascontiguousarray(np.asarray(pose, np.float32).T).ravel()


def pose_error(pose1, pose2):
    """The reference's own poseError (project/src/general_helper.cpp:11-21) on two 4 x 4 poses:
    (rotation chord, translation distance).  Host only."""
    out = np.zeros(2, np.float32)
    st = lib().kfref_pose_error(_p(_cm(pose1)), _p(_cm(pose2)), _p(out))
    if st != OK:
        raise RuntimeError("kfref_pose_error: status %d" % st)
    return float(out[0]), float(out[1])


def tum_sequence(path):
    """The reference's own RgbdDataset (project/src/rgbd_dataset.cpp:6-96) on a TUM sequence
    directory: ([(depth image path, 4 x 4 ground-truth pose)], initial pose inverse).  Host
    only."""
    L = lib()
    d = L.kfref_tum_open(os.fsencode(path))
    if not d:
        raise RuntimeError("kfref_tum_open: no sequence at %s" % path)
    try:
        frames = []
        buf = ctypes.create_string_buffer(4096)
        pose = np.zeros(16, np.float32)
        while True:
            st = L.kfref_tum_next(d, buf, len(buf), _p(pose))
            if st == 0:
                break
            if st != 1:
                raise RuntimeError("kfref_tum_next: status %d" % st)
            frames.append((buf.value.decode(), pose.reshape(4, 4).T.copy()))
        inv = np.zeros(16, np.float32)
        if L.kfref_tum_initial_pose_inverse(d, _p(inv)) != OK:
            raise RuntimeError("kfref_tum_initial_pose_inverse failed")
        return frames, inv.reshape(4, 4).T.copy()
    finally:
        L.kfref_tum_close(d)


def sensor_intrinsics(fov, level):
    """The reference's own Sensor (project/src/sensor.h:10-52) at one level: (K, K^-1) as 3 x 3
    float32 arrays, its principal points fixed for 640 x 480.  Host only."""
    k = np.zeros(9, np.float32)
    ik = np.zeros(9, np.float32)
    st = lib().kfref_sensor_intrinsics(float(fov), int(level), _p(k), _p(ik))
    if st != OK:
        raise RuntimeError("kfref_sensor_intrinsics: status %d" % st)
    return k.reshape(3, 3).T.copy(), ik.reshape(3, 3).T.copy()


def mue_scale_for(cfg):
    """The reference's truncation is mue_scale voxels (VoxelGridStruct, voxel_grid.h:47-52)."""
    res = np.float32(cfg.volume_width) / np.float32(cfg.volume_n - 1)
    return float(np.float32(cfg.mu) / res)


def matching_config(kf, mue_scale=3.0, **overrides):
    """A library configuration with the reference's hard-coded values: kf_config_default
    (project/src/main.cpp:11-59) at 640 x 480, overridden by `overrides`; mu is the
    reference's mue_scale * resolution in float32 (voxel_grid.h:47-52; the fusion grid's
    mue_scale is 3, kinect_fusion.cpp:18)."""
    c = kf.default_config(**overrides)
    res = np.float32(c.volume_width) / np.float32(c.volume_n - 1)
    c.mu = float(np.float32(mue_scale) * res)
    return c


class RefPipeline:
    """The reference's pipeline on one GPU for a library configuration `cfg` whose frame,
    intrinsics and constants match the reference's (see `matching_config`)."""

    def __init__(self, cfg, vis=False, vis_n=512, vis_width=5.0, vis_mue_scale=2.0):
        assert (cfg.width, cfg.height, cfg.levels) == (W, H, LEVELS), "the reference's frame is 640 x 480, 3 levels"
        assert (cfg.cx, cfg.cy) == (319.5, 239.5) and cfg.fx == cfg.fy
        self.cfg = cfg
        self.n = cfg.volume_n
        iters = np.array(list(cfg.iters)[:3], np.int32)
        self.h = lib().kfref_create(cfg.volume_n, cfg.volume_width, mue_scale_for(cfg), cfg.fx, cfg.depth_scale,
                                    _p(iters), cfg.dist_thresh, cfg.angle_thresh, cfg.stop_angle, cfg.stop_dist,
                                    vis_n if vis else 0, vis_width, vis_mue_scale)
        if not self.h:
            raise RuntimeError("kfref_create failed")
        self.set_pose(np.asarray(cfg.initial_pose, np.float32).reshape(4, 4).T)

    def close(self):
        if self.h:
            lib().kfref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st, what):
        if st in (CUDA_ERROR, BAD_ARG):
            raise RuntimeError("%s: status %d" % (what, st))
        return st

    # ---- frame loop ----
    def process_frame(self, raw):
        """One iteration of the reference's frame loop (frame 0: convert + fuse).  Returns
        (status, pose): status 1 when ICP's solve was not finite (pose kept)."""
        raw = np.ascontiguousarray(raw, np.uint16)
        assert raw.shape == (H, W)
        st = self._ck(lib().kfref_process_frame(self.h, _p(raw)), "process_frame")
        return st, self.pose()

    def upload(self, raw):
        raw = np.ascontiguousarray(raw, np.uint16)
        assert raw.shape == (H, W)
        self._ck(lib().kfref_upload(self.h, _p(raw)), "upload")

    def preprocess(self):
        self._ck(lib().kfref_preprocess(self.h), "preprocess")

    def convert(self):
        self._ck(lib().kfref_convert(self.h), "convert")

    def raycast(self, clear=True):
        if clear:
            self._ck(lib().kfref_clear_raycast_maps(self.h), "clear")
        self._ck(lib().kfref_raycast(self.h), "raycast")

    def compute_pose(self):
        return self._ck(lib().kfref_compute_pose(self.h), "compute_pose")

    def fuse(self):
        self._ck(lib().kfref_fuse(self.h), "fuse")

    def time_frames(self, frames, nframes):
        """Wall-clock seconds of `nframes` frame-loop iterations over `frames` (cycled), each
        uploading its frame from host memory; returns (seconds, statuses)."""
        frames = np.ascontiguousarray(frames, np.uint16)
        assert frames.shape[1:] == (H, W)
        sec = np.zeros(1, np.float64)
        st = np.zeros(max(1, nframes), np.int32)
        self._ck(lib().kfref_time_frames(self.h, _p(frames), frames.shape[0], nframes, _p(sec), _p(st)), "time_frames")
        return float(sec[0]), st[:nframes]

    def stage_times(self):
        """The reference's own summed stage times (ms): preprocess, raycast, ICP residuals,
        ICP solve (host), fuse, visualization."""
        ms = np.zeros(6, np.float64)
        lib().kfref_stage_times(self.h, _p(ms))
        return ms

    @property
    def frames(self):
        return lib().kfref_frames(self.h)

    @frames.setter
    def frames(self, f):
        lib().kfref_set_frames(self.h, int(f))

    # ---- state ----
    def pose(self):
        out = np.zeros(16, np.float32)
        lib().kfref_get_pose(self.h, _p(out))
        return out.reshape(4, 4).T.copy()

    def set_pose(self, pose):
        lib().kfref_set_pose(self.h, _p(_cm(pose)))

    def _map(self, which, level, ch):
        w, h = W >> level, H >> level
        out = np.zeros((h, w, ch) if ch > 1 else (h, w), np.float32)
        self._ck(lib().kfref_get_map(self.h, which, level, _p(out)), "get_map")
        return out

    def depth_meters(self):
        return self._map(0, 0, 1)

    def depth(self, level=0):
        return self._map(1, level, 1)

    def vertex_map(self, level=0):
        return self._map(2, level, 4)

    def raycast_maps(self, level=0):
        return self._map(3, level, 4), self._map(4, level, 4)

    def normal_map(self):
        """kernel::createNormalMap of the level-0 vertex map."""
        return self._map(5, 0, 4)

    def tsdf(self, vis=False):
        n = self.n if not vis else 512
        buf = np.zeros((n, n, n, 2), np.float32)
        self._ck(lib().kfref_get_tsdf(self.h, int(vis), _p(buf)), "get_tsdf")
        return buf[..., 0].copy(), buf[..., 1].copy()

    def set_tsdf(self, f, w, vis=False):
        buf = np.stack([np.asarray(f, np.float32), np.asarray(w, np.float32)], axis=-1)
        buf = np.ascontiguousarray(buf)
        self._ck(lib().kfref_set_tsdf(self.h, int(vis), _p(buf)), "set_tsdf")

    def icp_residuals(self, level, prev_pose, cur_pose):
        """kernel::constructIcpResiduals at `level` against the current raycast maps: A (h, w, 6)
        and b (h, w); a row of zeros is a rejected pixel."""
        w, h = W >> level, H >> level
        A = np.zeros((h, w, 6), np.float32)
        b = np.zeros((h, w), np.float32)
        self._ck(lib().kfref_icp_residuals(self.h, level, _p(_cm(prev_pose)), _p(_cm(cur_pose)), self.cfg.dist_thresh,
                                           self.cfg.angle_thresh, _p(A), _p(b)), "icp_residuals")
        return A, b


# ---- the synced comparison the tests and the bench's accuracy block report ----

def _bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return bool(np.array_equal(a.view(np.uint32), b.view(np.uint32)))


def _depth_mm(a, b, cam):
    """|distance to the camera| difference (mm) where both maps hit (0 elsewhere), the
    both-hit mask and the hit agreement."""
    ha, hb = a[..., 3] == -1, b[..., 3] == -1
    both = ha & hb
    da = np.linalg.norm(a[..., :3].astype(np.float64) - cam, axis=-1)
    db = np.linalg.norm(b[..., :3].astype(np.float64) - cam, axis=-1)
    return np.where(both, np.abs(da - db) * 1e3, 0.0), both, float(np.mean(ha == hb))


def compare_synced(kf, orc, torch, cfg, imgs):
    """Run a library session, the reference's pipeline and the FP64 oracle over `imgs`, the
    latter two starting every frame from the library's volume and pose, and return one dict
    per frame:
      meters, pyramid   bit equality of the converted depth and, per level, of the filtered
                        depth and the vertex map;
      icp_masks         per level, agreement of the correspondence masks of the first ICP pass
                        (same poses, each side's own maps and residual kernel);
      rays              per level: hit agreement and >1 mm counts of library vs reference,
                        reference vs FP64 oracle and library vs FP64 oracle, and `unexplained`:
                        pixels >1 mm from the reference where the reference is within 1 mm
                        of the FP64 oracle;
      pose              poseError of library / reference / FP64 oracle pairs;
      tsdf              the frame's fusion by the reference at the library's pose against the
                        library's (parity.tsdf_frame_parity)."""
    import parity
    xs, zs = orc.voxel_axes(cfg.volume_n, cfg.volume_width)
    s = kf.KinectFusion(cfg)
    R = RefPipeline(cfg)
    O = orc.Pipeline(cfg, prec=1)
    rows = []
    try:
        for fi, img in enumerate(imgs):
            f0, w0 = s.tsdf()
            pose0 = s.pose()
            R.set_tsdf(f0, w0)
            R.set_pose(pose0)
            if fi:
                O.set_tsdf(f0, w0)
                O.set_pose(pose0)
            R.upload(img)
            if fi == 0:
                R.convert()
            else:
                R.preprocess()
                R.raycast(clear=True)   # rays that miss the volume leave zeros, as the library writes
            st_g, pose_g = s.process_frame(img)
            st_o, pose_o = O.process_frame(img)
            row = dict(frame=fi, st=(int(st_g), int(st_o)), meters=_bits_equal(s.depth(-1), R.depth_meters()))
            if fi:
                row["pyramid"] = [(_bits_equal(s.depth(l), R.depth(l)), _bits_equal(s.vertex_map(l), R.vertex_map(l)))
                                  for l in range(cfg.levels)]
                cam = pose0[:3, 3].astype(np.float64)
                row["rays"] = []
                for l in range(cfg.levels):
                    gv, _ = s.raycast_maps(l)
                    rv, _ = R.raycast_maps(l)
                    ov, _ = O.raycast_maps(l)
                    d_lr, both_lr, agree_lr = _depth_mm(gv, rv, cam)
                    d_ro, both_ro, agree_ro = _depth_mm(rv, ov, cam)
                    d_lo, both_lo, agree_lo = _depth_mm(gv, ov, cam)
                    lib_off = d_lr > 1.0
                    ref_off = d_ro > 1.0
                    row["rays"].append(dict(
                        level=l, hit_agreement=agree_lr, both=int(both_lr.sum()),
                        lib_ref_over_1mm=int(lib_off.sum()), lib_ref_median_mm=float(np.median(d_lr[both_lr])),
                        ref_fp64_over_1mm=int(ref_off.sum()), ref_fp64_median_mm=float(np.median(d_ro[both_ro])),
                        ref_fp64_hit_agreement=agree_ro,
                        unexplained=int((lib_off & ~ref_off).sum()),
                        lib_fp64_over_1mm=int((d_lo > 1.0).sum()), lib_fp64_median_mm=float(np.median(d_lo[both_lo])),
                        lib_fp64_both=int(both_lo.sum()), lib_fp64_hit_agreement=agree_lo))
                row["icp_masks"] = []
                for l in range(cfg.levels):
                    A, _ = R.icp_residuals(l, pose0, pose0)
                    rm = np.any(A[..., 3:6] != 0, axis=-1)
                    vm = torch.from_numpy(s.vertex_map(l)).cuda()
                    tv, tn = [torch.from_numpy(x).cuda() for x in s.raycast_maps(l)]
                    h, w = vm.shape[:2]
                    gA = torch.zeros((h * w, 6), dtype=torch.float32, device="cuda")
                    gb = torch.zeros(h * w, dtype=torch.float32, device="cuda")
                    kf.kernel.constructIcpResiduals(vm, tv, tn, pose0[:3, :3], pose0[:3, 3], pose0[:3, :3], pose0[:3, 3],
                                                    kf.level_intrinsics(cfg, l), cfg.dist_thresh, cfg.angle_thresh,
                                                    gA, gb)
                    gm = np.any(gA.cpu().numpy().reshape(h, w, 6)[..., 3:6] != 0, axis=-1)
                    row["icp_masks"].append(float(np.mean(gm == rm)))
                row["st_ref"] = int(R.compute_pose())
                pose_r = R.pose()
                pe = lambda a, b: tuple(float(x) for x in kf.poseError(a, b))   # noqa: E731
                row["pose"] = dict(lib_fp64=pe(pose_g, pose_o), ref_fp64=pe(pose_r, pose_o), lib_ref=pe(pose_g, pose_r))
            # the frame's fusion by the reference at the library's pose
            R.set_pose(pose_g)
            R.fuse()
            fr, wr = R.tsdf()
            f1, w1 = s.tsdf()
            row["tsdf"] = parity.tsdf_frame_parity(cfg, f0, w0, f1, w1, fr, wr, pose_g, s.depth(-1), xs, zs)
            rows.append(row)
            del f0, w0, f1, w1, fr, wr
    finally:
        s.close()
        R.close()
        O.close()
    return rows
