"""Batched and served forms: every session's result is the same whether it runs alone or in
a mix of uneven sessions (bit-identical: each session's pixels, tiles and reduction order
do not depend on the other sessions), admission follows the HBM budget, and the launch shapes
the tuner tries change no result."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mix_configs(kf):
    return [
        kf.config_small(),
        kf.config_small(volume_n=96, tsdf_format=kf.KF_TSDF_F16U16),
        kf.config_full(volume_n=256, tsdf_format=kf.KF_TSDF_F16U16, volume_width=3.0),
        kf.config_small(levels=2, iters=(6, 4, 0)),
    ]


@pytest.fixture(scope="module")
def mix(kf):
    from kfb200 import synth
    cfgs = mix_configs(kf)
    seqs = [synth.sequence(c, 5, seed=100 + i, kind=synth.WOBBLE if c.width == 320 else synth.LOOP)[0]
            for i, c in enumerate(cfgs)]
    alone = []
    for c, seq in zip(cfgs, seqs):
        s = kf.KinectFusion(c)
        poses = [s.process_frame(img)[1] for img in seq]
        alone.append((poses, s.tsdf(), s.raycast_maps(0)))
        s.close()
    return cfgs, seqs, alone


def test_batch_equals_alone(kf, mix):
    cfgs, seqs, alone = mix
    b = kf.Batch(cfgs)
    for f in range(5):
        st, poses = b.step([seq[f] for seq in seqs])
        assert st == kf.KF_OK
        for i in range(len(cfgs)):
            np.testing.assert_array_equal(poses[i], alone[i][0][f])
    for i in range(len(cfgs)):
        s = b.session(i)
        f, w = s.tsdf()
        np.testing.assert_array_equal(f, alone[i][1][0])
        np.testing.assert_array_equal(w, alone[i][1][1])
        v, n = s.raycast_maps(0)
        np.testing.assert_array_equal(v, alone[i][2][0])
    b.close()


def test_long_lane_budget_batch_equals_alone(kf):
    """Two 640x480 sessions make 2 x 12,600 ray tiles, past the 25,000 at which a step's lanes
    march 64 iterations before handing a ray to a warp (40 alone): the hand-off point moves,
    the samples and results do not."""
    from kfb200 import synth
    cfgs = [kf.config_full(volume_n=256), kf.config_full(volume_n=256, tsdf_format=kf.KF_TSDF_F16U16)]
    seqs = [synth.sequence(c, 5, seed=150 + i, kind=synth.LOOP)[0] for i, c in enumerate(cfgs)]
    alone = []
    for c, seq in zip(cfgs, seqs):
        s = kf.KinectFusion(c)
        poses = [s.process_frame(img)[1] for img in seq]
        alone.append((poses, s.raycast_maps(0)))
        s.close()
    b = kf.Batch(cfgs)
    for f in range(5):
        st, poses = b.step([seq[f] for seq in seqs])
        assert st == kf.KF_OK
        for i in range(2):
            np.testing.assert_array_equal(poses[i], alone[i][0][f])
    for i in range(2):
        v, n = b.session(i).raycast_maps(0)
        np.testing.assert_array_equal(v, alone[i][1][0])
        np.testing.assert_array_equal(n, alone[i][1][1])
    b.close()


def test_batch_skipped_session_is_untouched(kf, mix):
    cfgs, seqs, alone = mix
    b = kf.Batch(cfgs[:2])
    b.step([seqs[0][0], seqs[1][0]])
    b.step([seqs[0][1], None])          # session 1 sits this step out
    b.step([seqs[0][2], seqs[1][1]])
    _, poses = b.step([seqs[0][3], seqs[1][2]])
    np.testing.assert_array_equal(poses[0], alone[0][0][3])
    np.testing.assert_array_equal(poses[1], alone[1][0][2])
    b.close()


def test_autotune_on_live_steps_changes_no_result_and_is_cached(kf, tmp_path):
    """The tuner tries a different launch shape on each live step (grids, raycast form, lane
    budget, ray tile, fusion split): every step's poses equal the untuned sessions' bit for bit.
    The chosen shape goes to the cache file, and a new batch of the same mix takes it from there
    without spending a step."""
    from kfb200 import synth
    cfgs = [kf.config_small(), kf.config_small(volume_n=96, tsdf_format=kf.KF_TSDF_F16U16)]
    nframes = 80
    seqs = [synth.sequence(c, nframes, seed=120 + i)[0] for i, c in enumerate(cfgs)]
    alone = []
    for c, seq in zip(cfgs, seqs):
        s = kf.KinectFusion(c)
        alone.append([s.process_frame(img)[1] for img in seq])
        s.close()
    cache = str(tmp_path / "shapes.json")
    b = kf.Batch(cfgs)
    b.step([seq[0] for seq in seqs])
    b.autotune_start(cache)
    left0, rep = b.autotune_status()
    assert left0 > 0 and rep["source"] == "tuning"
    f = 1
    while True:
        _, poses = b.step([seq[f] for seq in seqs])
        for i in range(len(cfgs)):
            np.testing.assert_array_equal(poses[i], alone[i][f])
        f += 1
        left, rep = b.autotune_status()
        if left == 0:
            break
        assert f < nframes
    assert f - 1 == left0
    assert rep["source"] == "tuned" and set(rep["shape"]) >= {"grid_ray", "ray_budget", "ray_tw", "fuse_split"}
    for g in range(f, f + 3):   # the chosen shape keeps the results too
        _, poses = b.step([seq[g] for seq in seqs])
        for i in range(len(cfgs)):
            np.testing.assert_array_equal(poses[i], alone[i][g])
    b.close()
    b2 = kf.Batch(cfgs)
    b2.autotune_start(cache)
    left, rep2 = b2.autotune_status()
    assert left == 0 and rep2["source"] == "cache" and rep2["shape"] == rep["shape"]
    b2.close()


def test_server_alone_vs_mix(kf, mix):
    cfgs, seqs, alone = mix
    srv = kf.Server(max_slots=8, hbm_budget_bytes=8 << 30)
    ids = [srv.open(c) for c in cfgs]
    # frames arrive unevenly: each step serves whatever is queued
    pending = [0] * len(cfgs)
    got = [[] for _ in cfgs]
    order = [[0, 1, 2, 3], [0, 2], [1, 2, 3], [0, 1, 3], [0, 1, 2, 3], [2, 3, 0], [1, 3, 0, 2], [1, 0, 2, 3]]
    for step_sessions in order:
        submitted = [i for i in step_sessions if pending[i] < 5]
        for i in submitted:
            assert srv.submit(ids[i], seqs[i][pending[i]]) == kf.KF_OK
        assert srv.step() == len(submitted)
        for i in submitted:
            pose, stats = srv.result(ids[i])
            assert stats["frame"] == pending[i]
            got[i].append(pose)
            pending[i] += 1
    for i in range(len(cfgs)):
        for f, pose in enumerate(got[i]):
            np.testing.assert_array_equal(pose, alone[i][0][f])
    st = srv.stats()
    assert st["frames_done"] == sum(len(g) for g in got) and st["p99_ms"] > 0
    srv.close()


def test_server_one_queued_frame_per_session(kf, mix):
    cfgs, seqs, alone = mix
    srv = kf.Server(max_slots=2, hbm_budget_bytes=4 << 30)
    sid = srv.open(cfgs[0])
    assert srv.submit(sid, seqs[0][0]) == kf.KF_OK
    assert srv.submit(sid, seqs[0][1]) == kf.KF_ERR_STATE
    assert srv.step() == 1
    srv.close()


def test_server_admission_by_budget(kf, mix):
    cfgs, seqs, alone = mix
    import ctypes
    need = ctypes.c_size_t()
    kf.lib.kf_session_footprint(ctypes.byref(cfgs[0]), ctypes.byref(need))
    budget = int(need.value * 2.5)
    srv = kf.Server(max_slots=4, hbm_budget_bytes=budget)
    a = srv.open(cfgs[0])
    b = srv.open(cfgs[0])
    with pytest.raises(kf.KfError) as e:
        srv.open(cfgs[0])
    assert e.value.status == kf.KF_ERR_OOM_BUDGET
    srv.close_session(a)
    c = srv.open(cfgs[0])                 # closing freed the budget
    assert srv.stats()["sessions_refused"] == 1
    srv2 = kf.Server(max_slots=1, hbm_budget_bytes=8 << 30)
    srv2.open(cfgs[0])
    assert srv2.try_open(cfgs[0]) is None   # capacity
    srv.close()
    srv2.close()


def test_server_submit_while_stepping(kf, mix):
    """Frames submitted from another thread while a step runs join the next step."""
    cfgs, seqs, alone = mix
    srv = kf.Server(max_slots=4, hbm_budget_bytes=8 << 30)
    ids = [srv.open(c) for c in cfgs[:2]]
    done = [0, 0]
    stop = threading.Event()

    def producer(i):
        for f in range(5):
            while srv.submit(ids[i], seqs[i][f]) != kf.KF_OK:
                if stop.is_set():
                    return
            done[i] = f + 1

    threads = [threading.Thread(target=producer, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    served = 0
    for _ in range(2000):
        served += srv.step()
        if served >= 10:
            break
    stop.set()
    for t in threads:
        t.join()
    assert served == 10
    for i in range(2):
        pose, _ = srv.result(ids[i])
        np.testing.assert_array_equal(pose, alone[i][0][4])
    srv.close()
