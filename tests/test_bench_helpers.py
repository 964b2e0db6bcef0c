"""bench.py's bookkeeping on the CPU: the per-frame launch count against the committed launch
list, the algorithmic-bytes formulas and the per-stage roofline arithmetic."""
import json
import os
import re
import sys
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_kernels_per_frame_matches_the_launch_list():
    """gpu_launches = KERNELS_PER_FRAME x steps: the committed ncu launch list of the bench's own
    workload shows exactly that many kernels launched once per frame."""
    with open(os.path.join(ROOT, "profiles", "launches_plain_640x480_512cube_f32.md")) as f:
        text = f.read()
    rows = re.findall(r"^\| ([^|]+?) \| (\d+) \| [\d.]+ \|", text, re.M)
    frames = max(int(n) for _, n in rows)
    per_frame = [k for k, n in rows if int(n) == frames and "set-up" not in k]
    assert len(per_frame) == bench.KERNELS_PER_FRAME, per_frame


def test_ncu_issue_and_issue_rooflines():
    """The instruction-issue view of the stages: ncu warp instructions per frame over the stage
    time, against SMs x 4 schedulers x clock."""
    issue = bench.ncu_issue()
    for k in ("preprocess", "raycast", "icp", "fuse"):
        assert issue[k]["warp_instructions"] > 0 and issue[k]["thread_instructions"] > issue[k]["warp_instructions"]
    r = bench.issue_rooflines(issue, np.array([0.02, 0.15, 0.05, 0.06]), 148, 1965.0)
    peak = 148 * 4 * 1965e6
    assert set(r) == {"preprocess", "raycast", "icp", "fuse"}
    assert r["raycast"]["peak_per_s"] == round(peak, 1)
    assert abs(r["raycast"]["frac"] - issue["raycast"]["warp_instructions"] / 0.15e-3 / peak) < 1e-4
    # a stage without a count or without a time is left out
    assert "icp" not in bench.issue_rooflines({"raycast": issue["raycast"]}, [0.02, 0.15, 0.05, 0.06], 148, 1965.0)
    assert "raycast" not in bench.issue_rooflines(issue, [0.02, 0.0, 0.05, 0.06], 148, 1965.0)


def test_ncu_traffic_has_every_stage():
    t = bench.ncu_traffic()
    for k in ("preprocess", "raycast", "icp", "fuse"):
        assert isinstance(t[k], int) and t[k] > 0


def cfg(fmt=0):
    return SimpleNamespace(volume_n=512, tsdf_format=fmt, width=640, height=480, levels=3)


def test_algorithmic_bytes():
    ab = bench.algorithmic_bytes(cfg(), fused_voxels=1000, samples=10, hits=2)
    px = 640 * 480
    assert ab["fuse_dense"] == 512 ** 3 * 16 + px * 4          # f32 value + f32 weight, read + write
    assert ab["fuse_updated"] == 1000 * 16 + px * 4
    maps = (px + px // 4 + px // 16) * 32                      # vertex + normal float4 per pixel
    assert ab["raycast_gather"] == 10 * 8 * 4 + 2 * 6 * 8 * 4 + maps
    ab16 = bench.algorithmic_bytes(cfg(1), fused_voxels=1000, samples=10, hits=2)
    assert ab16["fuse_dense"] == 512 ** 3 * 8 + px * 4          # f16 value + u16 weight
    assert ab16["raycast_gather"] == 10 * 8 * 2 + 2 * 6 * 8 * 2 + maps


def test_stage_rooflines_arithmetic():
    c = cfg()
    ab = bench.algorithmic_bytes(c, fused_voxels=2_000_000, samples=30_000_000, hits=300_000)
    stage_ms = [0.02, 0.16, 0.05, 0.064]
    out = bench.stage_rooflines(c, ab, stage_ms, peak=6400.0, icp_iters=[2, 1, 2],
                                traffic={"raycast": 123}, fps=3500.0)
    for k, ms in zip(["preprocess", "raycast", "icp", "fuse"], stage_ms):
        row = out[k]
        assert row["ms"] == ms
        assert row["achieved_gbs"] == pytest.approx(row["algorithmic_bytes"] / (ms / 1e3) / 1e9, abs=0.05)
        assert row["frac"] == pytest.approx(row["achieved_gbs"] / 6400.0, abs=1e-4)
    assert out["raycast"]["algorithmic_bytes"] == ab["raycast_gather"]
    assert out["raycast"]["dram_bytes_ncu"] == 123 and out["icp"]["dram_bytes_ncu"] is None
    px = [640 * 480, 320 * 240, 160 * 120]
    assert out["icp"]["algorithmic_bytes"] == (px[0] * 2 + px[1] * 1 + px[2] * 2) * 48
    assert out["fuse"]["voxels_per_s_dense"] == pytest.approx(512 ** 3 / 0.064e-3, rel=1e-6)
    assert out["frame"]["voxels_per_s"] == pytest.approx(512 ** 3 * 3500.0, rel=1e-6)


def test_drift_report(tmp_path, capsys):
    """tests/drift_300.py's report on small stand-in pose sequences: errors against the truth
    and the FP64 oracle's poses, and the share of frames with equal ICP iteration counts."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import drift_300
    eye = np.eye(4, dtype=np.float32)
    truth = np.stack([eye] * 3)
    moved = truth.copy()
    moved[:, 0, 3] = 0.01   # 1 cm off in x
    iters = np.array([[1, 1, 2]] * 3)
    np.savez(tmp_path / "g.npz", truth=truth, lib_f32=truth, lib_f32_iters=iters, lib_f16u16=moved,
             lib_f16u16_iters=iters[::-1] * np.array([[1, 1, 1], [1, 2, 1], [1, 1, 1]]))
    np.savez(tmp_path / "o.npz", truth=truth, poses=truth, iters=iters)
    drift_300.report(str(tmp_path / "g.npz"), str(tmp_path / "o.npz"))
    r = json.loads(capsys.readouterr().out)
    assert r["lib_f32"]["vs_oracle_fp64"]["m"] == 0.0 and r["lib_f32"]["frames_icp_iterations_equal"] == 1.0
    assert abs(r["lib_f16u16"]["vs_truth"]["m"] - 0.01) < 1e-6
    assert abs(r["lib_f16u16"]["frames_icp_iterations_equal"] - 2 / 3) < 1e-9
    assert "ref" not in r
