"""Host-side file formats: the TUM RGB-D sequence reader and its 16-bit PNG decoder
(kf_tum_*, kf_png16_read; the reference's RgbdDataset, project/src/rgbd_dataset.cpp:6-96),
checked against PNG files and a sequence directory written here by an independent encoder
(zlib from the Python standard library).  CPU only."""
import os
import struct
import tempfile
import zlib

import numpy as np
import pytest


def write_png16(path, img, filters=(0,)):
    """16-bit greyscale PNG; row filters cycle through `filters` (0 none, 1 sub, 2 up, 3 avg, 4 paeth)."""
    h, w = img.shape
    be = img.astype(">u2").tobytes()
    stride = w * 2
    rows = [be[y * stride:(y + 1) * stride] for y in range(h)]
    raw = bytearray()
    prev = bytes(stride)
    for y, row in enumerate(rows):
        f = filters[y % len(filters)]
        out = bytearray(stride)
        for x in range(stride):
            a = row[x - 2] if x >= 2 else 0
            b = prev[x]
            c = prev[x - 2] if x >= 2 else 0
            if f == 0:
                pr = 0
            elif f == 1:
                pr = a
            elif f == 2:
                pr = b
            elif f == 3:
                pr = (a + b) // 2
            else:
                p = a + b - c
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                pr = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            out[x] = (row[x] - pr) & 0xFF
        raw.append(f)
        raw += out
        prev = row

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    ihdr = struct.pack(">IIBBBBB", w, h, 16, 0, 0, 0, 0)
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", ihdr) + chunk(b"IDAT", zlib.compress(bytes(raw), 6))
                + chunk(b"IEND", b""))


def quat_pose(t, q):
    """glm::mat4_cast(quat(w, x, y, z)) with translation t, as a numpy 4x4."""
    x, y, z, w = q
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                  [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                  [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
    P = np.eye(4)
    P[:3, :3] = R
    P[:3, 3] = t
    return P


@pytest.mark.parametrize("filters", [(0,), (1,), (2,), (3,), (4,), (0, 1, 2, 3, 4)])
def test_png16_decoder_filters(kf, filters):
    rng = np.random.default_rng(3)
    img = rng.integers(0, 65536, size=(37, 53), dtype=np.uint16)
    img[5] = 0
    img[:, 7] = 65535
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "x.png")
        write_png16(p, img, filters)
        np.testing.assert_array_equal(kf.read_png16(p, 53, 37), img)
        with pytest.raises(kf.KfError):
            kf.read_png16(p, 52, 37)     # size mismatch: KF_ERR_SHAPE


def test_tum_sequence(kf):
    rng = np.random.default_rng(4)
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "depth"))
        gt_t = np.arange(0.0, 2.0, 0.01) + 1305031102.0          # ground truth at 100 Hz
        trans = rng.normal(size=(gt_t.size, 3))
        quats = rng.normal(size=(gt_t.size, 4))
        quats /= np.linalg.norm(quats, axis=1, keepdims=True)
        with open(os.path.join(d, "groundtruth.txt"), "w") as f:
            f.write("# ground truth trajectory\n# file: 'x.bag'\n# timestamp tx ty tz qx qy qz qw\n")
            for t, tr, q in zip(gt_t, trans, quats):
                f.write("%.4f %.4f %.4f %.4f %.4f %.4f %.4f %.4f\n" % (t, *tr, *q))
        depth_t = gt_t[3::7][:12] + 0.0031                          # 12 depth frames between poses
        imgs = []
        with open(os.path.join(d, "depth.txt"), "w") as f:
            f.write("# depth maps\n# file: 'x.bag'\n# timestamp filename\n")
            for k, t in enumerate(depth_t):
                img = rng.integers(0, 30000, size=(48, 64), dtype=np.uint16)
                imgs.append(img)
                rel = "depth/%.6f.png" % t
                write_png16(os.path.join(d, rel), img, (k % 5,))
                f.write("%.6f %s\n" % (t, rel))
        ds = kf.RgbdDataset(d)
        assert len(ds) == 12
        for k in range(12):
            depth, pose = ds.nextFrame(64, 48)
            np.testing.assert_array_equal(depth, imgs[k])
            i = int(np.argmin(np.abs(gt_t - depth_t[k])))          # the nearest ground-truth pose
            # poses round-trip through the 4-decimal text file
            tq = np.round(trans[i], 4), np.round(quats[i], 4)
            np.testing.assert_allclose(pose, quat_pose(*tq), atol=2e-6)
        assert ds.isFinished()
        inv = ds.getInitialPoseInverse()
        first = ds.frame(0, 64, 48)[1]
        np.testing.assert_allclose(inv @ first, np.eye(4), atol=1e-5)
        ds.close()


def test_tum_missing_directory(kf):
    with pytest.raises(kf.KfError):
        kf.RgbdDataset("/nonexistent/sequence")
