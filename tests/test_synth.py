"""The synthetic depth sequences that stand in for the reference's TUM input.  CPU only."""
import numpy as np

import pytest


@pytest.fixture(scope="module")
def synth():
    from kfb200 import synth
    return synth


def test_deterministic(kf, synth):
    cfg = kf.config_small()
    a, pa = synth.sequence(cfg, 3, seed=11)
    b, pb = synth.sequence(cfg, 3, seed=11)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(pa, pb)
    c, _ = synth.sequence(cfg, 1, seed=12)
    assert not np.array_equal(a[0], c[0])


def test_noise_model(kf, synth):
    cfg = kf.config_small()
    sc = synth.scene(cfg.volume_width)
    pose = synth.trajectory(synth.WOBBLE, 1, 5, cfg.volume_width)[0]
    noisy, true = synth.render(sc, pose, cfg.width, cfg.height, cfg.fx, cfg.fy, cfg.cx, cfg.cy, 5, 0, True, True)
    clean = synth.render(sc, pose, cfg.width, cfg.height, cfg.fx, cfg.fy, cfg.cx, cfg.cy, 5, 0, False)
    seen = (true > 0) & (true <= 3.9)
    # ~3% dropouts among visible pixels
    drop = np.mean(noisy[seen] == 0)
    assert 0.02 < drop < 0.04
    # residuals scaled by 0.0012 z^2 are ~N(0, 1) (plus the 1 mm rounding)
    keep = seen & (noisy > 0)
    z = true[keep]
    r = (noisy[keep].astype(np.float64) / 1000.0 - z) / (0.0012 * z * z)
    assert abs(np.mean(r)) < 0.1 and 0.9 < np.std(r) < 1.3
    # exact frame: rounding only
    assert np.max(np.abs(clean[seen].astype(np.float64) / 1000.0 - true[seen])) <= 0.0005 + 1e-6
    # nothing beyond 4 m
    assert noisy.max() <= 4000


def test_scene_inside_cube(kf, synth):
    for width in (2.0, 3.0):
        s = synth.scene(width)
        h = width / 2
        assert -h < s.sphere_c[2] - s.sphere_r and s.sphere_c[2] + s.sphere_r < h
        assert -h < s.box_lo[2] and s.box_hi[2] < h and s.plane_y < h


@pytest.mark.parametrize("kind,frames", [(0, 60), (1, 300)])
def test_trajectory_motion_bounds(synth, kind, frames):
    poses = synth.trajectory(kind, frames, 9, 3.0 if kind else 2.0)
    for a, b in zip(poses[:-1], poses[1:]):
        dt = np.linalg.norm(b[:3, 3] - a[:3, 3])
        rel = a[:3, :3].T @ b[:3, :3]
        ang = np.degrees(np.arccos(np.clip((np.trace(rel) - 1) / 2, -1, 1)))
        assert dt <= 0.02 and ang <= 1.0
    # the loop closes
    if kind == 1:
        np.testing.assert_allclose(poses[0], poses[-1], atol=0.03)


def test_short_loop_is_the_start_of_the_full_loop(synth):
    """A LOOP of a few frames follows the full-size sequence's camera (per-frame motion <= 2 cm,
    <= 1 degree), not a loop squeezed into those frames."""
    full = synth.trajectory(synth.LOOP, synth.LOOP_FRAMES, 63, 3.0)
    for frames in (2, 6, 46):
        short = synth.trajectory(synth.LOOP, frames, 63, 3.0)
        assert short.shape == (frames, 4, 4)
        np.testing.assert_array_equal(short, full[:frames])
    longer = synth.trajectory(synth.LOOP, 400, 63, 3.0)
    assert longer.shape == (400, 4, 4)
    assert max(np.linalg.norm(b[:3, 3] - a[:3, 3]) for a, b in zip(longer[:-1], longer[1:])) <= 0.02
