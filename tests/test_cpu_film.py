"""Film output (Film::to_rgb_image, src/film.rs:136-302): the oracle's
restatement against an independent numpy restatement, and the PNG writer."""
import struct
import zlib

import numpy as np

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
