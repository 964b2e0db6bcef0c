"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/liboracle.so).

The oracle restates the reference's per-frame path on the CPU (kf_oracle.cpp).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU legs load this module; the product never does.
prec = 0 runs the float instantiation (the reference's arithmetic), prec = 1 the FP64 one.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(LIB_PATH):
    build()
_lib = ctypes.CDLL(LIB_PATH)

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_LL = ctypes.c_longlong

_SIG = {
    "kfo_half_value": (_F, [ctypes.c_uint16]),
    "kfo_convert": (_I, [_P, _P, _I, _I, _F, _I, _I]),
    "kfo_bilateral": (_I, [_P, _P, _I, _I, _F, _F, _I, _I, _I]),
    "kfo_down_sample": (_I, [_P, _P, _I, _I, _F, _I, _I]),
    "kfo_vertex_map": (_I, [_P, _P, _I, _I, _P, _I, _I]),
    "kfo_normal_map": (_I, [_P, _P, _I, _I, _I, _I]),
    "kfo_compute_normal": (_I, [_P, _I, _I, _I, _I, _P]),
    "kfo_raycast": (_LL, [_P, _I, _F, _F, _P, _P, _P, _P, _I, _I, _F, _F, _F, _F, _I, _I, _I, _I, _P, _I]),
    "kfo_fuse": (_LL, [_P, _I, _I, _P, _P, _P, _I, _F, _F, _F, _P, _F, _F, _I, _I]),
    "kfo_voxel_axes": (_I, [_I, _F, _P, _P]),
    "kfo_icp_residuals": (_I, [_P, _P, _P, _I, _I, _P, _P, _P, _P, _P, _F, _F, _P, _P, _P, _I]),
    "kfo_solve_lls": (_I, [_P, _P, _I, _P, _I]),
    "kfo_fill_a_b": (_I, [_P, _P, _P, _P, _P]),
    "kfo_update_pose": (_I, [_P, _P, _I]),
    "kfo_euler_yxz": (_I, [_F, _F, _F, _P]),
    "kfo_pose_error": (_I, [_P, _P, _P]),
    "kfo_compute_correspondence": (_I, [_P, _P, _P, _P, _P]),
    "kfo_normals_too_different": (_I, [_P, _P, _P, _F]),
    "kfo_compute_pose": (_I, [_P, _P, _P, _P, _P, _P, _P, _I]),
    "kfo_pipeline_create": (_P, [_P, _I, _I]),
    "kfo_pipeline_destroy": (None, [_P]),
    "kfo_pipeline_frame": (_I, [_P, _P, _P]),
    "kfo_pipeline_reset": (_I, [_P]),
    "kfo_pipeline_get_pose": (_I, [_P, _P]),
    "kfo_pipeline_set_pose": (_I, [_P, _P]),
    "kfo_pipeline_get_iters": (_I, [_P, _P]),
    "kfo_pipeline_get_depth": (_I, [_P, _I, _P]),
    "kfo_pipeline_get_vertex": (_I, [_P, _I, _P]),
    "kfo_pipeline_get_raycast": (_I, [_P, _I, _P, _P]),
    "kfo_pipeline_get_mask": (_I, [_P, _I, _P]),
    "kfo_pipeline_get_trace": (_I, [_P, _I, _P]),
    "kfo_pipeline_get_tsdf": (_I, [_P, _P, _P]),
    "kfo_pipeline_set_tsdf": (_I, [_P, _P, _P]),
    "kfo_pipeline_last_samples": (_LL, [_P, _I]),
    "kfo_pipeline_last_fused": (_LL, [_P]),
    "kfo_display_normals": (None, [_P, _I, _I, _P, _P]),
    "kfo_display_shading": (None, [_P, _I, _I, _P, _P, _P]),
}
for _n, (_r, _a) in _SIG.items():
    _f = getattr(_lib, _n)
    _f.restype = _r
    _f.argtypes = _a


def _p(a):
    # data_as keeps a reference to the array, so temporaries live through the call
    return a.ctypes.data_as(ctypes.c_void_p)


def _cm(m):
    """[row, col] numpy matrix -> column-major float32 array."""
    return np.ascontiguousarray(np.asarray(m, np.float32).T).reshape(-1).copy()


def _uncm(a, dim):
    return np.asarray(a, np.float32).reshape(dim, dim).T.copy()


def half_value(u):
    return _lib.kfo_half_value(int(u))


def convert(raw, scale, unmirror=False, trunc8=False):
    h, w = raw.shape
    raw = np.ascontiguousarray(raw, np.uint16)
    out = np.zeros((h, w), np.float32)
    _lib.kfo_convert(_p(raw), _p(out), w, h, scale, int(unmirror), int(trunc8))
    return out


def bilateral(depth, sigma_s, sigma_r, radius, prec=0, trunc8=False):
    h, w = depth.shape
    d = np.ascontiguousarray(depth, np.float32)
    out = np.zeros_like(d)
    _lib.kfo_bilateral(_p(d), _p(out), w, h, sigma_s, sigma_r, radius, int(trunc8), prec)
    return out


def down_sample(depth, sigma_r, prec=0, trunc8=False):
    h, w = depth.shape
    d = np.ascontiguousarray(depth, np.float32)
    out = np.zeros((h // 2, w // 2), np.float32)
    _lib.kfo_down_sample(_p(d), _p(out), w // 2, h // 2, sigma_r, int(trunc8), prec)
    return out


def vertex_map(depth, inv_k, prec=0, trunc8=False):
    h, w = depth.shape
    d = np.ascontiguousarray(depth, np.float32)
    out = np.zeros((h, w, 4), np.float32)
    _lib.kfo_vertex_map(_p(d), _p(out), w, h, _p(_cm(inv_k)), int(trunc8), prec)
    return out


def normal_map(vmap, prec=0, trunc8=False):
    h, w = vmap.shape[:2]
    v = np.ascontiguousarray(vmap, np.float32)
    out = np.zeros((h, w, 4), np.float32)
    _lib.kfo_normal_map(_p(v), _p(out), w, h, int(trunc8), prec)
    return out


def compute_normal(vmap, i, j):
    h, w = vmap.shape[:2]
    v = np.ascontiguousarray(vmap, np.float32)
    out = np.zeros(4, np.float32)
    _lib.kfo_compute_normal(_p(v), w, h, i, j, _p(out))
    return out


def raycast(tsdf_f, width, mu, pose, inv_k, w, h, min_d=0.4, max_d=6.0, step_l=1.99, step_s=0.1,
            keep_on_miss=True, tex9bit=False, prec=0, vmap=None, nmap=None, trunc8=False, trace=False,
            exact_positions=False):
    """Returns (vertex (h,w,4), normal (h,w,4), samples), plus the (h, w) int64 march decision
    traces (see march_trace in kf_oracle.cpp) when trace is true.  exact_positions: sample
    positions base + k * inc with one rounding (the CUDA library's) instead of the reference's
    repeated additions."""
    n = tsdf_f.shape[0]
    f = np.ascontiguousarray(tsdf_f, np.float32)
    v = np.zeros((h, w, 4), np.float32) if vmap is None else np.ascontiguousarray(vmap, np.float32).copy()
    nn = np.zeros((h, w, 4), np.float32) if nmap is None else np.ascontiguousarray(nmap, np.float32).copy()
    tr = np.zeros((h, w), np.int64) if trace else None
    s = _lib.kfo_raycast(_p(f), n, width, mu, _p(_cm(pose)), _p(_cm(inv_k)), _p(v), _p(nn), w, h, min_d, max_d,
                         step_l, step_s, int(keep_on_miss), int(tex9bit), int(trunc8), prec,
                         _p(tr) if trace else None, int(exact_positions))
    return (v, nn, s, tr) if trace else (v, nn, s)


def fuse(depth_m, cam_k, tsdf_f, tsdf_w, width, mu, pose, max_w=0.0, min_d=0.4, max_d=6.0, prec=0, trunc8=False):
    """In-place update of float32 arrays tsdf_f / tsdf_w (n, n, n); returns voxels updated."""
    h, w = depth_m.shape
    n = tsdf_f.shape[0]
    d = np.ascontiguousarray(depth_m, np.float32)
    assert tsdf_f.flags.c_contiguous and tsdf_w.flags.c_contiguous
    return _lib.kfo_fuse(_p(d), w, h, _p(_cm(cam_k)), _p(tsdf_f), _p(tsdf_w), n, width, mu, max_w, _p(_cm(pose)),
                         min_d, max_d, int(trunc8), prec)


def voxel_axes(n, width):
    xs = np.zeros(n, np.float32)
    zs = np.zeros(n, np.float32)
    _lib.kfo_voxel_axes(n, width, _p(xs), _p(zs))
    return xs, zs


def icp_residuals(vmap, tv, tn, prev_R, prev_t, cur_R, cur_t, k, dist, angle, trunc8=False):
    """Returns (A (w*h, 6), b (w*h), mask (h, w), count)."""
    h, w = vmap.shape[:2]
    A = np.zeros((w * h, 6), np.float32)
    b = np.zeros(w * h, np.float32)
    m = np.zeros((h, w), np.uint8)
    pt = np.asarray(prev_t, np.float32).copy()
    ct = np.asarray(cur_t, np.float32).copy()
    c = _lib.kfo_icp_residuals(_p(np.ascontiguousarray(vmap, np.float32)), _p(np.ascontiguousarray(tv, np.float32)),
                               _p(np.ascontiguousarray(tn, np.float32)), w, h, _p(_cm(prev_R)), _p(pt),
                               _p(_cm(cur_R)), _p(ct), _p(_cm(k)), dist, angle, _p(A), _p(b), _p(m), int(trunc8))
    return A, b, m, c


def fill_a_b(s, n, d):
    a = np.zeros(6, np.float32)
    b = np.zeros(1, np.float32)
    ss, nn, dd = (np.asarray(x, np.float32).copy() for x in (s, n, d))
    _lib.kfo_fill_a_b(_p(ss), _p(nn), _p(dd), _p(a), _p(b))
    return a, float(b[0])


def solve_lls(A, b, prec=0):
    A = np.ascontiguousarray(A, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    x = np.zeros(6, np.float32)
    _lib.kfo_solve_lls(_p(A), _p(b), b.size, _p(x), prec)
    return x


def update_pose(pose, x, prec=0):
    p = _cm(pose)
    xx = np.asarray(x, np.float32).copy()
    st = _lib.kfo_update_pose(_p(p), _p(xx), prec)
    return st, _uncm(p, 4)


def euler_yxz(beta, gamma, alpha):
    out = np.zeros(9, np.float32)
    _lib.kfo_euler_yxz(beta, gamma, alpha, _p(out))
    return _uncm(out, 3)


def pose_error(p1, p2):
    out = np.zeros(2, np.float32)
    _lib.kfo_pose_error(_p(_cm(p1)), _p(_cm(p2)), _p(out))
    return float(out[0]), float(out[1])


def compute_correspondence(vtx, R, t, k):
    out = np.zeros(2, np.int32)
    v = np.asarray(vtx, np.float32).copy()
    tt = np.asarray(t, np.float32).copy()
    _lib.kfo_compute_correspondence(_p(v), _p(_cm(R)), _p(tt), _p(_cm(k)), _p(out))
    return int(out[0]), int(out[1])


def normals_too_different(n, tn, R, angle):
    a = np.asarray(n, np.float32).copy()
    b = np.asarray(tn, np.float32).copy()
    return bool(_lib.kfo_normals_too_different(_p(a), _p(b), _p(_cm(R)), angle))


def compute_pose(cfg, vmaps, tvs, tns, pose, prec=0):
    """ICP::computePose on host pyramids; returns (status, pose, iters)."""
    L = len(vmaps)
    keep = [np.ascontiguousarray(a, np.float32) for a in list(vmaps) + list(tvs) + list(tns)]
    arr = ctypes.c_void_p * L
    pv = arr(*[k.ctypes.data for k in keep[:L]])
    pt = arr(*[k.ctypes.data for k in keep[L:2 * L]])
    pn = arr(*[k.ctypes.data for k in keep[2 * L:]])
    out = np.zeros(16, np.float32)
    iters = np.zeros(3, np.int32)
    st = _lib.kfo_compute_pose(pv, pt, pn, ctypes.byref(cfg), _p(_cm(pose)), _p(out), _p(iters), prec)
    return st, _uncm(out, 4), iters.tolist()


class Pipeline:
    """The reference's per-frame loop on the CPU (KinectFusion::startTracking)."""

    def __init__(self, cfg, prec=0, tex9bit=False):
        self.cfg = cfg
        self._h = _lib.kfo_pipeline_create(ctypes.byref(cfg), prec, int(tex9bit))

    def close(self):
        if self._h:
            _lib.kfo_pipeline_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def process_frame(self, raw):
        r = np.ascontiguousarray(raw, np.uint16)
        out = np.zeros(16, np.float32)
        st = _lib.kfo_pipeline_frame(self._h, _p(r), _p(out))
        return st, _uncm(out, 4)

    def pose(self):
        out = np.zeros(16, np.float32)
        _lib.kfo_pipeline_get_pose(self._h, _p(out))
        return _uncm(out, 4)

    def set_pose(self, pose):
        _lib.kfo_pipeline_set_pose(self._h, _p(_cm(pose)))

    def iters(self):
        out = np.zeros(3, np.int32)
        _lib.kfo_pipeline_get_iters(self._h, _p(out))
        return out.tolist()

    def _wh(self, level):
        return self.cfg.width >> max(level, 0), self.cfg.height >> max(level, 0)

    def depth(self, level=0):
        w, h = self._wh(level)
        out = np.zeros((h, w), np.float32)
        _lib.kfo_pipeline_get_depth(self._h, level, _p(out))
        return out

    def vertex_map(self, level=0):
        w, h = self._wh(level)
        out = np.zeros((h, w, 4), np.float32)
        _lib.kfo_pipeline_get_vertex(self._h, level, _p(out))
        return out

    def raycast_maps(self, level=0):
        w, h = self._wh(level)
        v = np.zeros((h, w, 4), np.float32)
        n = np.zeros((h, w, 4), np.float32)
        _lib.kfo_pipeline_get_raycast(self._h, level, _p(v), _p(n))
        return v, n

    def ray_trace(self, level=0):
        """(h, w) int64 march decision traces of the last frame's raycast at `level`."""
        w, h = self._wh(level)
        t = np.zeros((h, w), np.int64)
        _lib.kfo_pipeline_get_trace(self._h, level, _p(t))
        return t

    def icp_mask(self, level=0):
        w, h = self._wh(level)
        m = np.zeros((h, w), np.uint8)
        _lib.kfo_pipeline_get_mask(self._h, level, _p(m))
        return m

    def tsdf(self):
        n = self.cfg.volume_n
        f = np.zeros((n, n, n), np.float32)
        w = np.zeros((n, n, n), np.float32)
        _lib.kfo_pipeline_get_tsdf(self._h, _p(f), _p(w))
        return f, w

    def set_tsdf(self, f, w):
        _lib.kfo_pipeline_set_tsdf(self._h, _p(np.ascontiguousarray(f, np.float32)),
                                   _p(np.ascontiguousarray(w, np.float32)))

    def last_samples(self, level=0):
        return _lib.kfo_pipeline_last_samples(self._h, level)

    def last_fused(self):
        return _lib.kfo_pipeline_last_fused(self._h)


def display_normals(nmap, inv_rot):
    """normalMapToWindowContentKernel (project/src/display.cu:63-81) -> (h, w, 4) uint8."""
    n = np.ascontiguousarray(nmap, np.float32)
    h, w = n.shape[:2]
    out = np.zeros((h, w, 4), np.uint8)
    _lib.kfo_display_normals(_p(n), w, h, _p(_cm(inv_rot)), _p(out))
    return out


def display_shading(nmap, pose, inv_k):
    """shadingToWindowContentKernel (project/src/display.cu:83-105) -> (h, w, 4) uint8."""
    n = np.ascontiguousarray(nmap, np.float32)
    h, w = n.shape[:2]
    out = np.zeros((h, w, 4), np.uint8)
    _lib.kfo_display_shading(_p(n), w, h, _p(_cm(pose)), _p(_cm(inv_k)), _p(out))
    return out
