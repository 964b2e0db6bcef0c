"""Accumulated drift over 300 free-running full-size frames: the library (f32+f32 and
f16+u16 volumes), the reference's own pipeline built from its sources (when oracle/_ref holds
it) and the FP64 oracle, all on the same seeded 300-frame loop (640x480, 512^3 over 3 m), each
tracking on its own from the identity start -- no re-synchronisation.

A measurement script, not a test module (pytest does not collect it):

    python tests/drift_300.py gpu OUT_GPU.npz        # library and reference poses (a B200)
    python tests/drift_300.py oracle OUT_ORACLE.npz  # FP64 oracle poses (CPU, a few minutes)
    python tests/drift_300.py report OUT_GPU.npz OUT_ORACLE.npz

The report gives each pipeline's end-of-sequence pose error against the synthetic ground truth
and against the FP64 oracle (poseError: rotation chord in radians, translation in metres), and
the share of frames whose ICP iteration counts equal the oracle's."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (os.path.join(ROOT, "kinectfusion-cuda_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import kfb200 as kf  # noqa: E402
from kfb200 import synth  # noqa: E402

FRAMES = 300
SEED = 63


def frames():
    cfg = kf.config_full()
    imgs, truth = synth.sequence(cfg, FRAMES, seed=SEED, kind=synth.LOOP)
    return cfg, imgs, np.stack(truth)


def run_gpu(path):
    import refpipe
    cfg, imgs, truth = frames()
    out = {"truth": truth}
    for name, fmt in (("lib_f32", kf.KF_TSDF_F32F32), ("lib_f16u16", kf.KF_TSDF_F16U16)):
        s = kf.KinectFusion(kf.config_full(tsdf_format=fmt))
        poses, iters = [], []
        for img in imgs:
            _, p = s.process_frame(img)
            poses.append(p)
            iters.append(list(s.frame_stats()["icp_iters"]))
        out[name] = np.stack(poses)
        out[name + "_iters"] = np.array(iters)
        s.close()
    if refpipe.available():
        R = refpipe.RefPipeline(cfg)
        out["ref"] = np.stack([R.process_frame(img)[1] for img in imgs])
        R.close()
    np.savez_compressed(path, **out)


def run_oracle(path):
    import oracle
    cfg, imgs, truth = frames()
    P = oracle.Pipeline(cfg, prec=1)
    poses, iters = [], []
    for img in imgs:
        _, p = P.process_frame(img)
        poses.append(p)
        iters.append(list(P.iters()))
    np.savez_compressed(path, truth=truth, poses=np.stack(poses), iters=np.array(iters))


def report(gpu_path, oracle_path):
    g, o = np.load(gpu_path), np.load(oracle_path)
    truth = g["truth"]
    assert np.array_equal(truth, o["truth"]), "different frame sequences"

    def err(a, b):
        r, t = kf.poseError(a, b)
        return {"rad": float(r), "m": float(t)}

    res = {"frames": FRAMES, "workload": "640x480, 512^3 over 3 m, mu 0.02 m, seeded 300-frame loop (seed %d)" % SEED,
           "oracle_fp64_vs_truth": err(o["poses"][-1], truth[-1])}
    for name in ("lib_f32", "lib_f16u16", "ref"):
        if name not in g:
            continue
        res[name] = {"vs_truth": err(g[name][-1], truth[-1]), "vs_oracle_fp64": err(g[name][-1], o["poses"][-1])}
        if name + "_iters" in g:
            res[name]["frames_icp_iterations_equal"] = float(np.mean(np.all(g[name + "_iters"] == o["iters"], axis=1)))
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    mode = sys.argv[1] if len(sys.argv) > 1 else ""
    if mode == "gpu" and len(sys.argv) == 3:
        run_gpu(sys.argv[2])
    elif mode == "oracle" and len(sys.argv) == 3:
        run_oracle(sys.argv[2])
    elif mode == "report" and len(sys.argv) == 4:
        report(sys.argv[2], sys.argv[3])
    else:
        sys.exit(__doc__)
