"""Film output without a device (Film::writeEXR / writePNG, src/film/Film.cpp:
154-272): the EXR holds R, G, B and the albedo.* / normals.* layers as 32-bit
floats with ZIP compression, read back bit for bit by OpenCV (beauty) and by
an independent parser of the OpenEXR scanline layout (every channel); the PNG
holds the reference's exposure + sRGB bytes, read back by Pillow."""
import os
import struct
import zlib

import numpy as np
import pytest

from anacapa_b200 import api


def parse_exr(path):
    """Minimal OpenEXR reader: single-part scanline, FLOAT channels, NONE or
    ZIP compression. Returns {channel name: (H, W) float32}."""
    b = open(path, "rb").read()
    assert struct.unpack_from("<I", b, 0)[0] == 20000630
    pos, attrs = 8, {}
    while b[pos] != 0:
        e = b.index(b"\0", pos)
        name = b[pos:e].decode()
        e2 = b.index(b"\0", e + 1)
        typ = b[e + 1:e2].decode()
        size = struct.unpack_from("<I", b, e2 + 1)[0]
        attrs[name] = (typ, b[e2 + 5:e2 + 5 + size])
        pos = e2 + 5 + size
    pos += 1
    chans, raw = [], attrs["channels"][1]
    q = 0
    while raw[q] != 0:
        e = raw.index(b"\0", q)
        chans.append(raw[q:e].decode())
        assert struct.unpack_from("<i", raw, e + 1)[0] == 2  # FLOAT
        q = e + 1 + 16
    comp = attrs["compression"][1][0]
    x0, y0, x1, y1 = struct.unpack("<4i", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    lines = {0: 1, 3: 16}[comp]
    nb = (h + lines - 1) // lines
    offs = struct.unpack_from(f"<{nb}Q", b, pos)
    out = {c: np.zeros((h, w), np.float32) for c in chans}
    for off in offs:
        y, n = struct.unpack_from("<iI", b, off)
        data = b[off + 8:off + 8 + n]
        rows = min(lines, h - y)
        want = rows * len(chans) * w * 4
        if n < want:
            t = np.frombuffer(zlib.decompress(data), np.uint8).astype(np.int64)
            t = (np.cumsum(t - 128) + 128) & 0xFF  # undo the predictor
            t[0] = np.frombuffer(zlib.decompress(data), np.uint8)[0]
            t = t.astype(np.uint8)
            half = (len(t) + 1) // 2
            data = np.empty(len(t), np.uint8)
            data[0::2] = t[:half]
            data[1::2] = t[half:]
            data = data.tobytes()
        v = np.frombuffer(data, np.float32).reshape(rows, len(chans), w)
        for k, c in enumerate(chans):
            out[c][y:y + rows] = v[:, k]
    return out


@pytest.fixture(scope="module")
def images():
    rng = np.random.default_rng(2)
    h, w = 37, 53  # not a multiple of the 16-line ZIP block
    rgb = rng.gamma(1.0, 0.6, (h, w, 3)).astype(np.float32)
    rgb[:5, :7] = 0.0  # runs of identical bytes
    al = rng.uniform(0, 1, (h, w, 3)).astype(np.float32)
    nr = rng.normal(size=(h, w, 3)).astype(np.float32)
    return rgb, al, nr


def test_exr_layers_round_trip(lib_built, tmp_path, images):
    rgb, al, nr = images
    p = tmp_path / "f.exr"
    api.image_write_exr(p, rgb, al, nr)
    ch = parse_exr(p)
    assert sorted(ch) == ["B", "G", "R", "albedo.B", "albedo.G", "albedo.R", "normals.B", "normals.G",
                          "normals.R"]
    for pre, img in (("", rgb), ("albedo.", al), ("normals.", nr)):
        got = np.stack([ch[pre + "R"], ch[pre + "G"], ch[pre + "B"]], -1)
        assert np.array_equal(got, img)


def test_exr_beauty_reads_in_opencv(lib_built, tmp_path, images):
    os.environ["OPENCV_IO_ENABLE_OPENEXR"] = "1"
    cv2 = pytest.importorskip("cv2")
    rgb, _, _ = images
    p = tmp_path / "beauty.exr"
    api.image_write_exr(p, rgb)
    assert set(parse_exr(p)) == {"R", "G", "B"}
    got = cv2.imread(str(p), cv2.IMREAD_UNCHANGED)
    if got is None:
        pytest.skip("this OpenCV build reads no EXR")
    assert np.array_equal(got[..., ::-1], rgb)


@pytest.mark.parametrize("exposure", [0.0, 1.5])
def test_png_bytes(lib_built, tmp_path, images, exposure):
    Image = pytest.importorskip("PIL.Image")
    rgb, _, _ = images
    p = tmp_path / "f.png"
    api.image_write_png(p, rgb, exposure)
    assert not (tmp_path / "f.png.writing.png").exists()
    got = np.asarray(Image.open(p).convert("RGB"))
    x = np.clip(rgb * np.float32(2.0 ** exposure), 0, 1).astype(np.float32)
    srgb = np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x.astype(np.float64), 1 / 2.4) - 0.055)
    want = (srgb.astype(np.float32) * np.float32(255) + np.float32(0.5)).astype(np.uint8)
    diff = np.abs(got.astype(int) - want.astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() > 0.999


def test_writer_errors(lib_built, tmp_path, images):
    rgb, _, _ = images
    with pytest.raises(api.AnaError):
        api.image_write_exr(tmp_path / "missing_dir" / "f.exr", rgb)
