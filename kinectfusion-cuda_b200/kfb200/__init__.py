"""kfb200 -- Python host mirror of the reference's KinectFusion interface over libkfb200.so.

The names follow the reference (isikmustafa/kinectfusion-cuda, project/src):

    KinectFusion            project/src/kinect_fusion.h:38-48  (per-frame pipeline)
    kernel.*                project/src/measurement.cuh, raycast.cuh, tsdf.cuh, icp.cuh
    ICP.computePose         project/src/icp.h:35-36
    LinearLeastSquares      project/src/linear_least_squares.h:19
    poseError               project/src/general_helper.h:9

Host arrays are numpy; device arrays for the per-stage ``kernel`` calls are torch CUDA
tensors (torch is only the allocator here).  4x4 poses and 3x3 matrices are numpy arrays
indexed [row, col]; they are converted to the column-major layout of the C ABI at the
boundary.  Every call goes through the CUDA library; there is no CPU path.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import (KF_DEBUG_COUNTERS, KF_DEBUG_NO_GRAPH, KF_DEBUG_RAY_TRACE, KF_ERR_ARG, KF_ERR_CAPACITY,
                   KF_ERR_CUDA, KF_ERR_NONFINITE, KF_ERR_OOM_BUDGET, KF_ERR_SHAPE, KF_ERR_STATE, KF_ERR_TIMEOUT,
                   KF_MAX_LEVELS, KF_OK, KF_RENDER_NORMALS, KF_RENDER_SHADING, KF_TSDF_F16U16, KF_TSDF_F32F32,
                   KF_WEIGHT_SCALE, RAY_COUNT_NAMES, KfConfig, KfError, KfFrameStats, KfServerStats, KfVolume, check,
                   lib)

__all__ = [
    "KfConfig", "KfError", "default_config", "config_small", "config_full", "KinectFusion", "kernel", "ICP",
    "LinearLeastSquares", "poseError", "Batch", "Server", "RgbdDataset", "read_png16", "lib", "to_colmajor",
    "from_colmajor",
]


# ------------------------------------------------------------------------------------------
# conversions
# ------------------------------------------------------------------------------------------
def to_colmajor(m):
    """numpy [row, col] matrix -> ctypes float array in column-major (glm) order."""
    m = np.asarray(m, dtype=np.float32)
    flat = np.ascontiguousarray(m.T).reshape(-1)
    return (ctypes.c_float * flat.size)(*flat.tolist())


def from_colmajor(arr, dim):
    a = np.array(arr[: dim * dim], dtype=np.float32)
    return a.reshape(dim, dim).T.copy()


def _fptr(a):
    return ctypes.cast(a, ctypes.POINTER(ctypes.c_float))


def _np_ptr(a):
    # data_as keeps a reference to the array, so temporaries live through the call
    return a.ctypes.data_as(ctypes.c_void_p)


def _dev_ptr(t):
    """Device address of a torch CUDA tensor (the only accepted device buffer type)."""
    if not hasattr(t, "data_ptr") or not getattr(t, "is_cuda", False):
        raise TypeError("device buffers must be torch CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("device buffers must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        return None
    return ctypes.c_void_p(int(getattr(stream, "cuda_stream", stream)))


# ------------------------------------------------------------------------------------------
# configuration
# ------------------------------------------------------------------------------------------
def default_config(**overrides):
    """The reference's configuration (project/src/main.cpp:11-59, dataset mode), with
    keyword overrides for any field of kf_config."""
    c = KfConfig()
    lib.kf_config_default(ctypes.byref(c))
    for k, v in overrides.items():
        if k == "iters":
            for i in range(KF_MAX_LEVELS):
                c.iters[i] = int(v[i]) if i < len(v) else 0
        elif k == "initial_pose":
            flat = np.asarray(v, dtype=np.float32).T.reshape(-1)
            for i in range(16):
                c.initial_pose[i] = float(flat[i])
        else:
            if not hasattr(c, k):
                raise AttributeError("kf_config has no field %r" % k)
            setattr(c, k, v)
    return c


def start_pose(cube_width):
    """Camera at (0, 0, -cube_width) looking along +z: the synthetic scenes' start pose."""
    p = np.eye(4, dtype=np.float32)
    p[2, 3] = -cube_width
    return p


def config_small(**overrides):
    """Plain pipeline, small size: 320x240, fx = fy = 262.5, 128^3 float/float TSDF over a
    2 m cube, truncation 0.03 m, bilateral sigma_s 4.5 px / sigma_r 30 mm / 5x5, ICP 4/5/10
    coarse to fine, 0.1 m / 20 degrees, depth in millimetres; no visualization volume."""
    kw = dict(width=320, height=240, fx=262.5, fy=262.5, cx=159.5, cy=119.5, depth_scale=1e-3,
              iters=(10, 5, 4), dist_thresh=0.1, angle_thresh=float(np.deg2rad(20.0)),
              bilateral_sigma_s=4.5, bilateral_sigma_r=0.03, bilateral_radius=2,
              volume_n=128, volume_width=2.0, mu=0.03, initial_pose=start_pose(2.0), vis_volume_n=0)
    kw.update(overrides)
    return default_config(**kw)


def config_full(**overrides):
    """Plain pipeline at full size: 640x480, fx = fy = 525, 512^3 float/float TSDF over a
    3 m cube, truncation 0.02 m, ICP 4/5/10 coarse to fine; no visualization volume."""
    kw = dict(width=640, height=480, fx=525.0, fy=525.0, cx=319.5, cy=239.5, depth_scale=1e-3,
              iters=(10, 5, 4), dist_thresh=0.1, angle_thresh=float(np.deg2rad(20.0)),
              bilateral_sigma_s=4.5, bilateral_sigma_r=0.03, bilateral_radius=2,
              volume_n=512, volume_width=3.0, mu=0.02, initial_pose=start_pose(3.0), vis_volume_n=0)
    kw.update(overrides)
    return default_config(**kw)


def level_intrinsics(cfg, level):
    """K_l of the reference's Sensor (project/src/sensor.h:14-19) as a numpy 3x3."""
    s = np.float32(1.0) / np.float32(1 << level)
    k = np.zeros((3, 3), dtype=np.float32)
    k[0, 0] = np.float32(cfg.fx) * s
    k[1, 1] = np.float32(cfg.fy) * s
    k[0, 2] = (np.float32(cfg.cx) + np.float32(0.5)) * s - np.float32(0.5)
    k[1, 2] = (np.float32(cfg.cy) + np.float32(0.5)) * s - np.float32(0.5)
    k[2, 2] = 1.0
    return k


def level_inverse_intrinsics(cfg, level):
    """K_l^-1 exactly as the library forms it (adjugate over determinant in float32, the
    glm::inverse the reference applies to its 3x3), so a caller's stage raycast from this
    matrix takes the same rays as the session's own (kf_render)."""
    k = level_intrinsics(cfg, level)
    f = np.float32
    a, b, cc = k[0, 0], k[0, 1], k[0, 2]
    d, e, ff = k[1, 0], k[1, 1], k[1, 2]
    g, h, i = k[2, 0], k[2, 1], k[2, 2]
    det = f(f(a * f(f(e * i) - f(ff * h))) - f(b * f(f(d * i) - f(ff * g)))) + f(cc * f(f(d * h) - f(e * g)))
    od = f(f(1.0) / det)
    ik = np.zeros((3, 3), dtype=np.float32)
    ik[0, 0] = f(f(e * i) - f(ff * h)) * od
    ik[0, 1] = -f(f(b * i) - f(cc * h)) * od
    ik[0, 2] = f(f(b * ff) - f(cc * e)) * od
    ik[1, 0] = -f(f(d * i) - f(ff * g)) * od
    ik[1, 1] = f(f(a * i) - f(cc * g)) * od
    ik[1, 2] = -f(f(a * ff) - f(cc * d)) * od
    ik[2, 0] = f(f(d * h) - f(e * g)) * od
    ik[2, 1] = -f(f(a * h) - f(b * g)) * od
    ik[2, 2] = f(f(a * e) - f(b * d)) * od
    return ik


# ------------------------------------------------------------------------------------------
# the per-frame pipeline
# ------------------------------------------------------------------------------------------
class KinectFusion:
    """One reconstruction session (the reference's KinectFusion class).

    process_frame(depth) runs one frame: frame 0 fuses only, later frames preprocess,
    raycast at the previous pose, run ICP and fuse (project/src/kinect_fusion.cpp:44-94).
    """

    def __init__(self, config, _handle=None, _owner=None):
        self.config = config
        self._owner = _owner
        if _handle is not None:
            self._s = _handle
            self._owns = False
        else:
            h = ctypes.c_void_p()
            check(lib.kf_session_create(ctypes.byref(config), ctypes.byref(h)), "kf_session_create")
            self._s = h
            self._owns = True
        self.w, self.h = config.width, config.height

    def close(self):
        if getattr(self, "_owns", False) and self._s:
            lib.kf_session_destroy(self._s)
        self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        check(lib.kf_session_reset(self._s), "kf_session_reset")

    def process_frame(self, depth, stream=None):
        """depth: (h, w) uint16 numpy array (host) or torch CUDA tensor.  Returns
        (status, pose 4x4); a non-finite ICP solution returns KF_ERR_NONFINITE with the
        previous pose kept (the reference throws, project/src/icp.cpp:67-73)."""
        pose = (ctypes.c_float * 16)()
        if hasattr(depth, "is_cuda") and depth.is_cuda:
            st = lib.kf_process_frame(self._s, _dev_ptr(depth), 1, _stream(stream), pose)
        else:
            d = np.ascontiguousarray(depth, dtype=np.uint16)
            if d.shape != (self.h, self.w):
                raise ValueError("depth frame must be %dx%d" % (self.h, self.w))
            st = lib.kf_process_frame(self._s, _np_ptr(d), 0, _stream(stream), pose)
        if st not in (KF_OK, KF_ERR_NONFINITE):
            raise KfError(st, "kf_process_frame")
        return st, from_colmajor(pose, 4)

    def submit_frame(self, depth, stream=None):
        """Queue a frame without waiting (kf_process_frame_submit): an (h, w) uint16 numpy
        array that stays unchanged until its wait_frame returns, or a torch CUDA tensor."""
        if hasattr(depth, "is_cuda") and depth.is_cuda:
            st = lib.kf_process_frame_submit(self._s, _dev_ptr(depth), 1, _stream(stream))
        else:
            if depth.shape != (self.h, self.w) or depth.dtype != np.uint16 or not depth.flags.c_contiguous:
                raise ValueError("depth frame must be a contiguous %dx%d uint16 array" % (self.h, self.w))
            st = lib.kf_process_frame_submit(self._s, _np_ptr(depth), 0, _stream(stream))
        check(st, "kf_process_frame_submit")

    def wait_frame(self):
        """(status, pose 4x4) of the oldest submitted frame (kf_process_frame_wait)."""
        pose = (ctypes.c_float * 16)()
        st = lib.kf_process_frame_wait(self._s, pose, None)
        if st not in (KF_OK, KF_ERR_NONFINITE):
            raise KfError(st, "kf_process_frame_wait")
        return st, from_colmajor(pose, 4)

    def startTracking(self, frames):
        """Run every frame of an iterable (the reference reads them from a dataset,
        project/src/kinect_fusion.cpp:44-73); returns the list of poses."""
        return [self.process_frame(f)[1] for f in frames]

    # taps
    def pose(self):
        p = (ctypes.c_float * 16)()
        check(lib.kf_get_pose(self._s, p))
        return from_colmajor(p, 4)

    def set_pose(self, pose):
        check(lib.kf_set_pose(self._s, to_colmajor(pose)))

    def frame_stats(self):
        st = KfFrameStats()
        check(lib.kf_get_frame_stats(self._s, ctypes.byref(st)))
        return {"frame": st.frame, "status": st.status, "icp_iters": list(st.icp_iters)}

    def _lw(self, level):
        return self.w >> level, self.h >> level

    def depth(self, level=0):
        w, h = (self.w, self.h) if level < 0 else self._lw(level)
        out = np.empty((h, w), np.float32)
        check(lib.kf_get_depth(self._s, level, _np_ptr(out), 1))
        return out

    def vertex_map(self, level=0):
        w, h = self._lw(level)
        out = np.empty((h, w, 4), np.float32)
        check(lib.kf_get_vertex(self._s, level, _np_ptr(out), 1))
        return out

    def raycast_maps(self, level=0):
        w, h = self._lw(level)
        v = np.empty((h, w, 4), np.float32)
        n = np.empty((h, w, 4), np.float32)
        check(lib.kf_get_raycast(self._s, level, _np_ptr(v), _np_ptr(n), 1))
        return v, n

    def icp_mask(self, level=0):
        w, h = self._lw(level)
        m = np.empty((h, w), np.uint8)
        check(lib.kf_get_icp_mask(self._s, level, _np_ptr(m), 1))
        return m

    def tsdf(self):
        """(f, w) float32 arrays of shape (n, n, n) indexed [z, y, x]."""
        n = self.config.volume_n
        inter = np.empty((n, n, n, 2), np.float32)
        check(lib.kf_get_tsdf(self._s, _np_ptr(inter), inter.nbytes, 1, 1))
        return inter[..., 0].copy(), inter[..., 1].copy()

    def vis_tsdf(self):
        """The visualization volume's (f, w) float32 arrays (n, n, n) indexed [z, y, x]."""
        n = self.config.vis_volume_n
        inter = np.empty((n, n, n, 2), np.float32)
        check(lib.kf_get_vis_tsdf(self._s, _np_ptr(inter), inter.nbytes, 1, 1), "kf_get_vis_tsdf")
        return inter[..., 0].copy(), inter[..., 1].copy()

    def vis_volume(self):
        v = KfVolume()
        check(lib.kf_get_vis_volume(self._s, ctypes.byref(v)), "kf_get_vis_volume")
        return v

    def set_tsdf(self, f, w):
        n = self.config.volume_n
        inter = np.empty((n, n, n, 2), np.float32)
        inter[..., 0] = f
        inter[..., 1] = w
        check(lib.kf_set_tsdf(self._s, _np_ptr(inter), inter.nbytes, 1, 1))

    def saveTSDF(self, path):
        """KinectFusion::saveTSDF (project/src/kinect_fusion.cpp:327-330): the visualization grid
        when the session has one (as the reference), else the tracking volume, in the .bin layout
        of VoxelGrid::saveVoxelGrid (project/src/voxel_grid.cpp:43-62): n^3 float2 {f, w}, x
        fastest."""
        if self.config.vis_volume_n:
            check(lib.kf_save_vis_tsdf_file(self._s, os.fsencode(path)), "kf_save_vis_tsdf_file")
        else:
            check(lib.kf_save_tsdf_file(self._s, os.fsencode(path)), "kf_save_tsdf_file")

    def loadTSDF(self, path):
        """KinectFusion::loadTSDF (project/src/kinect_fusion.cpp:332-335), the same grid as saveTSDF
        (VoxelGrid::loadVoxelGrid, project/src/voxel_grid.cpp:64-80)."""
        if self.config.vis_volume_n:
            check(lib.kf_load_vis_tsdf_file(self._s, os.fsencode(path)), "kf_load_vis_tsdf_file")
        else:
            check(lib.kf_load_tsdf_file(self._s, os.fsencode(path)), "kf_load_tsdf_file")

    def saveCheckpoint(self, path):
        """TSDF (.bin at path) + pose and frame count (path + '.pose')."""
        check(lib.kf_session_checkpoint_save(self._s, os.fsencode(path)), "kf_session_checkpoint_save")

    def loadCheckpoint(self, path):
        """Resume a saved session: the next frame tracks against the loaded model."""
        check(lib.kf_session_checkpoint_load(self._s, os.fsencode(path)), "kf_session_checkpoint_load")

    def render(self, mode=KF_RENDER_NORMALS, pose=None, stream=None):
        """KinectFusion::visualizeCurrentModel, headless: (h, w, 4) uint8 RGBA image of the model
        raycast from `pose` (default: the current pose)."""
        c = self.config
        img = np.empty((c.height, c.width, 4), np.uint8)
        pp = to_colmajor(pose) if pose is not None else None
        check(lib.kf_render(self._s, int(mode), pp, _np_ptr(img), 1, _stream(stream)), "kf_render")
        return img

    def volume(self):
        v = KfVolume()
        check(lib.kf_get_volume(self._s, ctypes.byref(v)))
        return v

    def process_frame_async(self, depth_dev, stream=None):
        """Enqueue a frame already in device memory (torch CUDA uint16 tensor); no sync."""
        check(lib.kf_process_frame_async(self._s, _dev_ptr(depth_dev), _stream(stream)), "kf_process_frame_async")

    def set_profiling(self, on=True):
        check(lib.kf_session_set_profiling(self._s, int(bool(on))))

    def stage_times(self):
        """Device ms of preprocess, raycast, ICP and fusion in the last completed step."""
        ms = (ctypes.c_float * 4)()
        check(lib.kf_session_stage_times(self._s, ms))
        return list(ms)

    def set_debug(self, flags):
        """Debug modes (KF_DEBUG_RAY_TRACE: record march decision traces; KF_DEBUG_NO_GRAPH:
        plain launches per stage inside NVTX ranges instead of the captured graph)."""
        check(lib.kf_session_set_debug(self._s, int(flags)), "kf_session_set_debug")

    def debug_counts(self):
        """The raycast's work counts of the last step (KF_DEBUG_COUNTERS), as a dict."""
        c = np.zeros(len(RAY_COUNT_NAMES), np.uint64)
        check(lib.kf_session_debug_counts(self._s, _np_ptr(c), len(c)), "kf_session_debug_counts")
        return {k: int(v) for k, v in zip(RAY_COUNT_NAMES, c)}

    def ray_trace(self, level=0):
        """(h, w) int64 march decision traces of the last raycast at `level` (debug mode)."""
        w, h = self._lw(level)
        t = np.empty((h, w), np.int64)
        check(lib.kf_get_ray_trace(self._s, level, _np_ptr(t), 1), "kf_get_ray_trace")
        return t


# ------------------------------------------------------------------------------------------
# per-stage calls (the reference's kernel:: namespace), on torch CUDA tensors
# ------------------------------------------------------------------------------------------
class kernel:  # noqa: N801 -- mirrors the reference's C++ namespace
    """Each call returns the elapsed milliseconds, like the reference's wrappers
    (project/src/measurement.cuh:11), and raises KfError(KF_ERR_SHAPE) where the reference
    throws std::runtime_error."""

    @staticmethod
    def _ms(fn, *args):
        ms = ctypes.c_float(0.0)
        check(fn(*args, ctypes.byref(ms)), fn.__name__)
        return ms.value

    @staticmethod
    def convertToDepthMeters(raw, out, scale, unmirror=False, stream=None):
        h, w = raw.shape
        oh, ow = out.shape
        return kernel._ms(lib.kf_convert_to_depth_meters, _dev_ptr(raw), w, h, _dev_ptr(out), ow, oh, scale,
                          int(unmirror), _stream(stream))

    @staticmethod
    def applyBilateralFilter(inp, out, sigma_s=4.0, sigma_r=0.25, radius=3, stream=None):
        h, w = inp.shape
        oh, ow = out.shape
        return kernel._ms(lib.kf_apply_bilateral_filter, _dev_ptr(inp), w, h, _dev_ptr(out), ow, oh, sigma_s,
                          sigma_r, radius, _stream(stream))

    @staticmethod
    def downSample(inp, out, sigma_r=0.25, stream=None):
        h, w = inp.shape
        oh, ow = out.shape
        return kernel._ms(lib.kf_down_sample, _dev_ptr(inp), w, h, _dev_ptr(out), ow, oh, sigma_r, _stream(stream))

    @staticmethod
    def createVertexMap(depth, vertex, inv_cam_k, stream=None):
        h, w = depth.shape
        oh, ow = vertex.shape[:2]
        return kernel._ms(lib.kf_create_vertex_map, _dev_ptr(depth), w, h, _dev_ptr(vertex), ow, oh,
                          to_colmajor(inv_cam_k), _stream(stream))

    @staticmethod
    def createNormalMap(vertex, normal, stream=None):
        h, w = vertex.shape[:2]
        oh, ow = normal.shape[:2]
        return kernel._ms(lib.kf_create_normal_map, _dev_ptr(vertex), w, h, _dev_ptr(normal), ow, oh,
                          _stream(stream))

    @staticmethod
    def volume(f, w, width, mu, fmt=KF_TSDF_F32F32, max_weight=0.0):
        """A kf_volume over torch tensors f, w of shape (n, n, n)."""
        v = KfVolume()
        v.f = _dev_ptr(f).value
        v.w = _dev_ptr(w).value
        v.n = int(f.shape[0])
        v.width = float(width)
        v.mu = float(mu)
        v.format = int(fmt)
        v.max_weight = float(max_weight)
        return v

    @staticmethod
    def initializeGrid(vol, stream=None):
        return kernel._ms(lib.kf_initialize_grid, ctypes.byref(vol), _stream(stream))

    @staticmethod
    def fuse(depth_m, vol, pose, cam_k, min_depth=0.4, max_depth=6.0, stream=None):
        h, w = depth_m.shape
        return kernel._ms(lib.kf_fuse, _dev_ptr(depth_m), w, h, to_colmajor(cam_k), ctypes.byref(vol),
                          to_colmajor(pose), min_depth, max_depth, _stream(stream))

    @staticmethod
    def raycast(vol, pose, inv_cam_k, vertex, normal, min_depth=0.4, max_depth=6.0, step_large=1.99,
                step_small=0.1, stream=None):
        h, w = vertex.shape[:2]
        nh, nw = normal.shape[:2]
        return kernel._ms(lib.kf_raycast, ctypes.byref(vol), to_colmajor(pose), to_colmajor(inv_cam_k),
                          _dev_ptr(vertex), w, h, _dev_ptr(normal), nw, nh, min_depth, max_depth, step_large,
                          step_small, _stream(stream))

    @staticmethod
    def normalMapToWindowContent(normal, inverse_rotation, rgba, stream=None):
        """project/src/display.cu:143-154, into an (h, w, 4) uint8 device image."""
        h, w = normal.shape[:2]
        return kernel._ms(lib.kf_normal_map_to_rgba, _dev_ptr(normal), w, h, to_colmajor(inverse_rotation),
                          _dev_ptr(rgba), _stream(stream))

    @staticmethod
    def shadingToWindowContent(normal, pose, inv_cam_k, rgba, stream=None):
        """project/src/display.cu:156-167."""
        h, w = normal.shape[:2]
        return kernel._ms(lib.kf_shading_to_rgba, _dev_ptr(normal), w, h, to_colmajor(pose), to_colmajor(inv_cam_k),
                          _dev_ptr(rgba), _stream(stream))

    @staticmethod
    def oneFloatChannelToWindowContent(src, scale, rgba, stream=None):
        """project/src/display.cu:117-128."""
        h, w = src.shape[:2]
        return kernel._ms(lib.kf_float_channel_to_rgba, _dev_ptr(src), w, h, float(scale), _dev_ptr(rgba),
                          _stream(stream))

    @staticmethod
    def constructIcpResiduals(vertex, target_vertex, target_normal, prev_rot, prev_transl, cur_rot, cur_transl,
                              cam_k, distance_thresh, angle_thresh, mat_a, vec_b, stream=None):
        h, w = vertex.shape[:2]
        pt = (ctypes.c_float * 3)(*[float(x) for x in prev_transl])
        ct = (ctypes.c_float * 3)(*[float(x) for x in cur_transl])
        return kernel._ms(lib.kf_construct_icp_residuals, _dev_ptr(vertex), _dev_ptr(target_vertex),
                          _dev_ptr(target_normal), w, h, to_colmajor(prev_rot), pt, to_colmajor(cur_rot), ct,
                          to_colmajor(cam_k), distance_thresh, angle_thresh, _dev_ptr(mat_a), _dev_ptr(vec_b),
                          _stream(stream))


class LinearLeastSquares:
    """LinearLeastSquares::solve (project/src/linear_least_squares.cpp:23-44) on device A, b."""

    def solve(self, mat_a, vec_b, n_equations, stream=None):
        x = (ctypes.c_float * 6)()
        st = lib.kf_solve_linear_least_squares(_dev_ptr(mat_a), _dev_ptr(vec_b), int(n_equations), x,
                                               _stream(stream))
        if st not in (KF_OK, KF_ERR_NONFINITE):
            raise KfError(st, "kf_solve_linear_least_squares")
        return np.array(x[:], dtype=np.float32)


class ICP:
    """ICP::computePose (project/src/icp.cpp:25-58) over device pyramids."""

    def __init__(self, config):
        self.config = config

    def computePose(self, vertex_pyramid, target_vertex_pyramid, target_normal_pyramid, pose, stream=None):
        levels = len(vertex_pyramid)
        h, w = vertex_pyramid[0].shape[:2]
        arr = ctypes.c_void_p * levels
        v = arr(*[_dev_ptr(t) for t in vertex_pyramid])
        tv = arr(*[_dev_ptr(t) for t in target_vertex_pyramid])
        tn = arr(*[_dev_ptr(t) for t in target_normal_pyramid])
        out = (ctypes.c_float * 16)()
        iters = (ctypes.c_int * KF_MAX_LEVELS)()
        st = lib.kf_compute_pose(v, tv, tn, w, h, levels, ctypes.byref(self.config), to_colmajor(pose), out, iters,
                                 _stream(stream))
        if st not in (KF_OK, KF_ERR_NONFINITE):
            raise KfError(st, "kf_compute_pose")
        return st, from_colmajor(out, 4), list(iters)


def poseError(pose_1, pose_2):
    """poseError (project/src/general_helper.cpp:11-21): (rotation chord, translation distance)."""
    out = (ctypes.c_float * 2)()
    check(lib.kf_pose_error(to_colmajor(pose_1), to_colmajor(pose_2), out))
    return float(out[0]), float(out[1])


# ------------------------------------------------------------------------------------------
# datasets
# ------------------------------------------------------------------------------------------
class RgbdDataset:
    """RgbdDataset (project/src/rgbd_dataset.h:12-27): a TUM RGB-D sequence directory, read by
    the library (kf_tum_*).  Frames come back as (h, w) uint16 depth and a 4x4 ground-truth
    camera->world pose."""

    def __init__(self, path=None):
        self._d = None
        self.m_current_index = 0
        if path is not None:
            self.load(path)

    def load(self, path):
        self.close()
        h = ctypes.c_void_p()
        check(lib.kf_tum_open(os.fsencode(path), ctypes.byref(h)), "kf_tum_open")
        self._d = h
        self.m_current_index = 0

    def close(self):
        if self._d:
            lib.kf_tum_close(self._d)
        self._d = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        n = ctypes.c_int()
        check(lib.kf_tum_count(self._d, ctypes.byref(n)))
        return n.value

    def frame(self, index, width=640, height=480):
        depth = np.empty((height, width), np.uint16)
        pose = (ctypes.c_float * 16)()
        check(lib.kf_tum_frame(self._d, int(index), _np_ptr(depth), width, height, pose), "kf_tum_frame")
        return depth, from_colmajor(pose, 4)

    def getCurrentPose(self):
        pose = (ctypes.c_float * 16)()
        check(lib.kf_tum_frame(self._d, self.m_current_index, None, 0, 0, pose), "kf_tum_frame")
        return from_colmajor(pose, 4)

    def getInitialPoseInverse(self):
        out = (ctypes.c_float * 16)()
        check(lib.kf_tum_initial_pose_inverse(self._d, out), "kf_tum_initial_pose_inverse")
        return from_colmajor(out, 4)

    def nextFrame(self, width=640, height=480):
        """The next depth image and its pose (getNextDepthImagePath + DepthMap::update)."""
        out = self.frame(self.m_current_index, width, height)
        self.m_current_index += 1
        return out

    def isFinished(self):
        return self.m_current_index >= len(self)


def read_png16(path, width, height):
    """A 16-bit greyscale PNG (DepthMap::update(path)) as an (h, w) uint16 array."""
    depth = np.empty((height, width), np.uint16)
    check(lib.kf_png16_read(os.fsencode(path), _np_ptr(depth), width, height), "kf_png16_read")
    return depth


# ------------------------------------------------------------------------------------------
# batched and served forms
# ------------------------------------------------------------------------------------------
class Batch:
    """Many independent sessions stepped together: one persistent launch per stage over all
    of them, replayed from a captured CUDA graph."""

    def __init__(self, configs):
        self.configs = list(configs)
        arr = (KfConfig * len(self.configs))(*self.configs)
        h = ctypes.c_void_p()
        check(lib.kf_batch_create(arr, len(self.configs), ctypes.byref(h)), "kf_batch_create")
        self._b = h
        self._sessions = {}

    def close(self):
        if self._b:
            lib.kf_batch_destroy(self._b)
        self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.configs)

    def step(self, frames, stream=None):
        """frames: list (one per session) of (h, w) uint16 numpy arrays or None to skip.
        Returns (status, poses (n, 4, 4))."""
        n = len(self.configs)
        if len(frames) != n:
            raise ValueError("one entry per session: %d for %d sessions" % (len(frames), n))
        keep = []
        ptrs = (ctypes.c_void_p * n)()
        for i, f in enumerate(frames):
            if f is None:
                ptrs[i] = None
                continue
            a = np.ascontiguousarray(f, dtype=np.uint16)
            keep.append(a)
            ptrs[i] = a.ctypes.data
        poses = (ctypes.c_float * (16 * n))()
        st = lib.kf_batch_step(self._b, ptrs, 0, _stream(stream), poses)
        if st not in (KF_OK, KF_ERR_NONFINITE):
            raise KfError(st, "kf_batch_step")
        p = np.array(poses[:], dtype=np.float32).reshape(n, 4, 4).transpose(0, 2, 1).copy()
        return st, p

    def session(self, i):
        h = ctypes.c_void_p()
        check(lib.kf_batch_session(self._b, i, ctypes.byref(h)))
        return KinectFusion(self.configs[i], _handle=h, _owner=self)

    def input_buffer(self, i):
        p = ctypes.c_void_p()
        check(lib.kf_batch_input_buffer(self._b, i, ctypes.byref(p)))
        return p.value

    def step_async(self, active, stream=None):
        arr = (ctypes.c_int * len(self.configs))(*[int(bool(a)) for a in active])
        check(lib.kf_batch_step_async(self._b, arr, _stream(stream)), "kf_batch_step_async")

    def autotune_start(self, cache_path=None):
        """Start tuning the launch shapes on the next steps (kf_batch_autotune_start); with a
        cache file holding this session mix, the cached shape applies at once."""
        check(lib.kf_batch_autotune_start(self._b, os.fsencode(cache_path) if cache_path else None),
              "kf_batch_autotune_start")

    def autotune_status(self):
        """(steps the tuning still needs, report dict)."""
        left = ctypes.c_int(0)
        buf = ctypes.create_string_buffer(4096)
        check(lib.kf_batch_autotune_status(self._b, ctypes.byref(left), buf, 4096), "kf_batch_autotune_status")
        import json
        return left.value, json.loads(buf.value.decode() or "{}")

    def set_profiling(self, on=True):
        check(lib.kf_batch_set_profiling(self._b, int(bool(on))))

    def stage_times(self):
        ms = (ctypes.c_float * 4)()
        check(lib.kf_batch_stage_times(self._b, ms))
        return list(ms)

    def set_debug(self, flags):
        """Debug modes for every session of the batch (see KinectFusion.set_debug)."""
        check(lib.kf_batch_set_debug(self._b, int(flags)), "kf_batch_set_debug")

    def debug_counts(self):
        """The raycast's work counts of the last step (KF_DEBUG_COUNTERS), as a dict."""
        c = np.zeros(len(RAY_COUNT_NAMES), np.uint64)
        check(lib.kf_batch_debug_counts(self._b, _np_ptr(c), len(c)), "kf_batch_debug_counts")
        return {k: int(v) for k, v in zip(RAY_COUNT_NAMES, c)}


def selftest_bounded_wait(timeout_ms=50):
    """Runs a device wait nothing releases; returns (status, wall ms).  The expected status
    is KF_ERR_TIMEOUT: the wait gave up on its own and the context is still usable."""
    waited = ctypes.c_int(0)
    st = lib.kf_selftest_bounded_wait(int(timeout_ms), ctypes.byref(waited))
    return st, waited.value


class Server:
    """Continuous batching: sessions open and close at any time, frames are submitted as
    they arrive and every step serves all queued frames together."""

    def __init__(self, max_slots, hbm_budget_bytes):
        h = ctypes.c_void_p()
        check(lib.kf_server_create(int(max_slots), int(hbm_budget_bytes), ctypes.byref(h)), "kf_server_create")
        self._s = h
        self._cfg = {}

    def close(self):
        if self._s:
            lib.kf_server_destroy(self._s)
        self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def open(self, config):
        """Returns the session id, or raises KfError(KF_ERR_OOM_BUDGET / KF_ERR_CAPACITY)."""
        sid = ctypes.c_int()
        check(lib.kf_server_open(self._s, ctypes.byref(config), ctypes.byref(sid)), "kf_server_open")
        self._cfg[sid.value] = config
        return sid.value

    def try_open(self, config):
        sid = ctypes.c_int()
        st = lib.kf_server_open(self._s, ctypes.byref(config), ctypes.byref(sid))
        if st == KF_OK:
            self._cfg[sid.value] = config
            return sid.value
        if st in (KF_ERR_OOM_BUDGET, KF_ERR_CAPACITY):
            return None
        raise KfError(st, "kf_server_open")

    def close_session(self, sid):
        check(lib.kf_server_close(self._s, sid), "kf_server_close")
        self._cfg.pop(sid, None)

    def submit(self, sid, depth, t_ms=None):
        d = np.ascontiguousarray(depth, dtype=np.uint16)
        t = lib.kf_now_ms() if t_ms is None else float(t_ms)
        return lib.kf_server_submit(self._s, sid, _np_ptr(d), t)

    def step(self):
        n = ctypes.c_int()
        st = lib.kf_server_step(self._s, ctypes.byref(n))
        if st not in (KF_OK, KF_ERR_NONFINITE):
            raise KfError(st, "kf_server_step")
        return n.value

    def result(self, sid):
        p = (ctypes.c_float * 16)()
        fs = KfFrameStats()
        check(lib.kf_server_result(self._s, sid, p, ctypes.byref(fs)), "kf_server_result")
        return from_colmajor(p, 4), {"frame": fs.frame, "status": fs.status, "icp_iters": list(fs.icp_iters)}

    def session(self, sid):
        h = ctypes.c_void_p()
        check(lib.kf_server_get_session(self._s, sid, ctypes.byref(h)))
        return KinectFusion(self._cfg[sid], _handle=h, _owner=self)

    def stats(self):
        s = KfServerStats()
        check(lib.kf_server_stats_get(self._s, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in KfServerStats._fields_}

    def reserve(self, config, count):
        """Pre-allocate device arenas (and pinned staging) for `count` sessions like config."""
        check(lib.kf_server_reserve(self._s, ctypes.byref(config), int(count)), "kf_server_reserve")

    def reset_stats(self):
        check(lib.kf_server_stats_reset(self._s), "kf_server_stats_reset")

    @staticmethod
    def now_ms():
        return lib.kf_now_ms()
