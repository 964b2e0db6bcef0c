"""Seeded synthetic depth sequences (libkfsynth.so), the stand-in for the TUM RGB-D files the
reference reads (project/src/rgbd_dataset.cpp).  Host-only; see csrc/synth.cpp for the scene,
noise model and trajectories."""
import ctypes
import os

import numpy as np

from ._lib import LIB_DIR

_PATH = os.path.join(LIB_DIR, "libkfsynth.so")
if not os.path.exists(_PATH):
    raise ImportError("libkfsynth.so is not built (%s); run `python kinectfusion-cuda_b200/build.py`" % _PATH)
_lib = ctypes.CDLL(_PATH)


class Scene(ctypes.Structure):
    _fields_ = [
        ("cube_width", ctypes.c_float), ("plane_y", ctypes.c_float),
        ("sphere_c", ctypes.c_float * 3), ("sphere_r", ctypes.c_float),
        ("box_lo", ctypes.c_float * 3), ("box_hi", ctypes.c_float * 3),
    ]


_lib.kfs_scene_make.argtypes = [ctypes.c_float, ctypes.POINTER(Scene)]
_lib.kfs_scene_make.restype = ctypes.c_int
_lib.kfs_trajectory.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_float, ctypes.c_void_p]
_lib.kfs_trajectory.restype = ctypes.c_int
_lib.kfs_render.argtypes = [ctypes.POINTER(Scene), ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                            ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint64, ctypes.c_int,
                            ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
_lib.kfs_render.restype = ctypes.c_int

WOBBLE = 0   # smooth wobble around the start pose (<= 2 cm, <= 1 degree per frame)
LOOP = 1     # closed loop around the objects
# frames of one closed loop: the full-size sequence (about 1.6 cm and 0.4 degrees per frame).
# A shorter LOOP request is the start of this loop, not a faster loop: a loop squeezed into a
# few frames moves the camera up to 0.8 m per frame, which no tracker follows.
LOOP_FRAMES = 300


def scene(cube_width):
    s = Scene()
    if _lib.kfs_scene_make(float(cube_width), ctypes.byref(s)) != 0:
        raise ValueError("cube width too small for the scene")
    return s


def trajectory(kind, frames, seed, cube_width):
    """Camera->world poses, (frames, 4, 4) float32, indexed [row, col].  A LOOP of fewer
    than LOOP_FRAMES frames is the start of the LOOP_FRAMES-frame loop."""
    total = max(int(frames), LOOP_FRAMES) if kind == LOOP else int(frames)
    buf = np.zeros((total, 16), np.float32)
    if _lib.kfs_trajectory(int(kind), total, int(seed), float(cube_width), buf.ctypes.data) != 0:
        raise ValueError("bad trajectory request")
    return buf.reshape(total, 4, 4).transpose(0, 2, 1)[: int(frames)].copy()


def render(sc, pose, width, height, fx, fy, cx, cy, seed, frame, noise=True, true_depth=False):
    """One uint16 millimetre frame (and the noise-free metres map when true_depth)."""
    out = np.zeros((height, width), np.uint16)
    flat = np.ascontiguousarray(np.asarray(pose, np.float32).T).reshape(-1)
    td = np.zeros((height, width), np.float32) if true_depth else None
    r = _lib.kfs_render(ctypes.byref(sc), flat.ctypes.data, width, height, fx, fy, cx, cy, int(seed), int(frame),
                        1 if noise else 0, out.ctypes.data, td.ctypes.data if td is not None else None)
    if r != 0:
        raise ValueError("render failed")
    return (out, td) if true_depth else out


def sequence(cfg, frames, seed, kind=WOBBLE, noise=True):
    """Frames and ground-truth poses for a session configuration (kfb200.KfConfig)."""
    sc = scene(cfg.volume_width)
    poses = trajectory(kind, frames, seed, cfg.volume_width)
    imgs = [render(sc, poses[f], cfg.width, cfg.height, cfg.fx, cfg.fy, cfg.cx, cfg.cy, seed, f, noise)
            for f in range(frames)]
    return imgs, poses
