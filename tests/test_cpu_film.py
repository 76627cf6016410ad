"""Film output (Film::to_rgb_image, src/film.rs:136-302; Film::save_exr,
:304-346): the oracle's tone-mapping restatement against an independent numpy
restatement, the PNG writer, and the oracle's EXR writer read back by
OpenCV's OpenEXR reader."""
import os
import struct
import zlib

import numpy as np
import pytest

import agentray
import oracle as O


def _numpy_rgb8(hdr, tm, white_point, gamma, scale):
    c = hdr.astype(np.float32) * np.float32(scale)
    lum = (np.float32(0.2126) * c[..., 0] + np.float32(0.7152) * c[..., 1]) + np.float32(0.0722) * c[..., 2]
    one = np.float32(1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        if tm == 1:
            s = np.where(lum > np.float32(1e-6), (lum / (one + lum)) / lum, one / (one + lum))
        elif tm == 2:
            lw2 = np.float32(white_point) * np.float32(white_point)
            mapped = (lum * (one + lum / lw2)) / (one + lum)
            s = np.where(lum > np.float32(1e-6), mapped / lum, one)
        else:
            s = np.ones_like(lum)
    m = np.clip(c * s[..., None].astype(np.float32), 0, 1).astype(np.float32)
    e = np.power(m, np.float32(one / np.float32(gamma)), dtype=np.float32)
    v = np.minimum(e * np.float32(255.0) + np.float32(0.5), np.float32(255.0))
    return np.where(v > 0, v, 0).astype(np.uint8)


def test_oracle_film_matches_numpy_restatement():
    rng = np.random.default_rng(3)
    hdr = (rng.lognormal(-1.0, 1.5, (37, 29, 3))).astype(np.float32)
    hdr[0, 0] = 0.0
    hdr[0, 1] = [1e-8, 0, 0]
    for tm, wp in ((0, 1.0), (1, 1.0), (2, 4.0)):
        a = O.film_to_rgb8(hdr, tm, wp, 2.2, 0.7)
        b = _numpy_rgb8(hdr, tm, wp, 2.2, 0.7)
        d = np.abs(a.astype(int) - b.astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 1e-3, (tm, d.max(), (d > 0).mean())


def test_png_round_trip(tmp_path):
    img = (np.arange(6 * 7 * 3) * 7 % 256).astype(np.uint8).reshape(6, 7, 3)
    p = str(tmp_path / "x.png")
    agentray.write_png(p, img)
    d = open(p, "rb").read()
    assert d[:8] == b"\x89PNG\r\n\x1a\n"
    i, chunks = 8, {}
    while i < len(d):
        n = struct.unpack(">I", d[i:i + 4])[0]
        tag = d[i + 4:i + 8]
        chunks[tag] = d[i + 8:i + 8 + n]
        assert struct.unpack(">I", d[i + 8 + n:i + 12 + n])[0] == zlib.crc32(tag + chunks[tag]) & 0xFFFFFFFF
        i += 12 + n
    assert struct.unpack(">IIBBBBB", chunks[b"IHDR"]) == (7, 6, 8, 2, 0, 0, 0)
    raw = zlib.decompress(chunks[b"IDAT"])
    rows = [raw[r * 22 + 1:(r + 1) * 22] for r in range(6)]
    assert all(raw[r * 22] == 0 for r in range(6))
    np.testing.assert_array_equal(np.frombuffer(b"".join(rows), np.uint8).reshape(6, 7, 3), img)


def _cv2_read_exr(path):
    os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
    cv2 = pytest.importorskip("cv2")
    img = cv2.imread(str(path), cv2.IMREAD_UNCHANGED)
    assert img is not None, "OpenCV could not read the EXR file"
    return img[:, :, ::-1]  # BGR -> RGB


def _exr_attrs(data):
    pos, attrs = 8, {}
    while data[pos] != 0:
        e = data.index(b"\0", pos)
        name = data[pos:e].decode()
        e2 = data.index(b"\0", e + 1)
        typ = data[e + 1:e2].decode()
        n = struct.unpack("<i", data[e2 + 1:e2 + 5])[0]
        attrs[name] = (typ, data[e2 + 5:e2 + 5 + n])
        pos = e2 + 5 + n
    return attrs, pos + 1


@pytest.mark.parametrize("h,w", [(37, 29), (16, 5), (1, 1), (33, 64)])
def test_oracle_exr_read_back_by_opencv(tmp_path, h, w):
    # Film::save_exr restated: OpenCV's OpenEXR reader (an independent
    # implementation) gets back exactly the f16-rounded values.
    rng = np.random.default_rng(h * 100 + w)
    hdr = rng.lognormal(-1.0, 2.0, (h, w, 3)).astype(np.float32)
    hdr.reshape(-1)[:3] = [0.0, 7e4, 3e-6]  # zero, f16 overflow (inf), an f16 subnormal
    p = tmp_path / "o.exr"
    O.film_save_exr(hdr, str(p), scale=0.5)
    want = (hdr * np.float32(0.5)).astype(np.float16).astype(np.float32)
    got = _cv2_read_exr(p)
    np.testing.assert_array_equal(got, want)
    data = p.read_bytes()
    assert struct.unpack("<II", data[:8]) == (20000630, 2)
    attrs, end = _exr_attrs(data)
    assert attrs["compression"] == ("compression", b"\x03")
    assert attrs["name"] == ("string", b"beauty")
    assert struct.unpack("<4i", attrs["dataWindow"][1]) == (0, 0, w - 1, h - 1)
    assert len(data) > end + 8 * ((h + 15) // 16)


def test_f16_nan_rule():
    x = np.array([np.nan, -np.nan, 1.0, 65520.0, 65519.0, 5.96e-8, -0.0], np.float32)
    x[1] = np.frombuffer(np.uint32(0xFFC12345).tobytes(), np.float32)[0]
    b = O.f32_to_f16_bits(x)
    assert b[0] == 0x7E00 and b[1] == (0x8000 | 0x7E00 | (0x412345 >> 13))
    assert b[2] == 0x3C00 and b[3] == 0x7C00 and b[4] == 0x7BFF and b[5] == 0x0001 and b[6] == 0x8000
