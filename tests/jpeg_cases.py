"""JPEG test inputs: files made by the oracle's encoder (oracle/at_jpeg.c)
across the formats a baseline decoder meets, and damaged or truncated
variants with the reference decoder's error codes (common/pjpeg.h:84-96)."""
import numpy as np

import oracle.oracle as O

OK, FILE, DQT, SOF, DHT, SOS, MISSING_DHT, DRI, RESET, EOF, UNSUPPORTED = range(11)


def _gray(h, w, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    img = 128 + 50 * np.sin(x / 7.0 + seed) * np.cos(y / 11.0) + rng.normal(0, 12, (h, w))
    img[h // 4: h // 2, w // 3: 2 * w // 3] = 20  # a flat dark patch with sharp edges
    return np.clip(img, 0, 255).astype(np.uint8)


def _rgb(h, w, seed):
    g = _gray(h, w, seed).astype(int)
    return np.clip(np.stack([g, np.roll(g, 5, 1) // 2 + 60, 255 - g], -1), 0, 255).astype(np.uint8)


def encode_matrix(small=True):
    """(name, bytes, decode flags) over gray / YCbCr, luma sampling, quality,
    restart intervals, standard or optimal tables, extra segments, the
    MJPEG case and tiny or odd sizes."""
    out = []
    h, w = (53, 75) if small else (301, 419)
    g = _gray(h, w, 1)
    for q in (50, 90, 100):
        for samp in ((1, 1), (2, 2)):
            for rst in (0, 1, 3):
                for fl in (0, O.JPEG_OPTIMIZE):
                    out.append((f"gray q{q} {samp} rst{rst} f{fl}", O.jpeg_encode(g, q, samp, rst, fl), 0))
    c = _rgb(h - 6, w + 7, 2)
    for samp in ((1, 1), (2, 1), (1, 2), (2, 2)):
        for rst in (0, 2):
            for fl in (0, O.JPEG_OPTIMIZE):
                out.append((f"rgb {samp} rst{rst} f{fl}", O.jpeg_encode(c, 85, samp, rst, fl), 0))
    for hh, ww in ((1, 1), (8, 8), (9, 17), (16, 16), (17, 33)):
        out.append((f"gray {ww}x{hh}", O.jpeg_encode(_gray(hh, ww, 3), 80), 0))
        out.append((f"rgb {ww}x{hh} 420", O.jpeg_encode(_rgb(hh, ww, 4), 80, (2, 2)), 0))
    out.append(("markers one-dqt", O.jpeg_encode(c, 75, (2, 2), 0, O.JPEG_MARKERS | O.JPEG_ONE_DQT), 0))
    out.append(("mjpeg tables", O.jpeg_encode(c, 75, (2, 1), 0, O.JPEG_NO_DHT), O.JPEG_MJPEG))
    out.append(("mjpeg flag with tables", O.jpeg_encode(c, 75, (2, 1), 4, O.JPEG_OPTIMIZE), O.JPEG_MJPEG))
    return out


def _find(buf, code):
    i = buf.find(bytes([0xFF, code]))
    assert i >= 0
    return i


def _patch(buf, at, vals):
    b = bytearray(buf)
    b[at:at + len(vals)] = bytes(vals)
    return bytes(b)


def bad_files():
    """(name, bytes, flags, expected code or None) for files the reference
    decoder refuses or reads past: only cases it handles without undefined
    behaviour, so the oracle and the GPU must give its exact output."""
    g = _gray(40, 56, 5)
    base = O.jpeg_encode(g, 90)
    rst = O.jpeg_encode(g, 90, (1, 1), 2)
    col = O.jpeg_encode(_rgb(40, 56, 6), 90, (2, 2), 3)
    out = []
    sof = _find(base, 0xC0)
    out.append(("progressive", _patch(base, sof + 1, [0xC2]), 0, UNSUPPORTED))
    out.append(("arithmetic", _patch(base, sof + 1, [0xC9]), 0, UNSUPPORTED))
    out.append(("precision 12", _patch(base, sof + 4, [12]), 0, SOF))
    out.append(("four components", _patch(base, sof + 9, [4]), 0, SOF))
    out.append(("no components", _patch(base, sof + 9, [0]), 0, SOF))
    dqt = _find(base, 0xDB)
    out.append(("dqt length", _patch(base, dqt + 2, [0, 0x44]), 0, DQT))
    out.append(("dqt 16-bit", _patch(base, dqt + 4, [0x10]), 0, DQT))
    dht = _find(base, 0xC4)
    out.append(("dht class 2", _patch(base, dht + 4, [0x20]), 0, DHT))
    out.append(("dht overfull", _patch(base, dht + 5, [3]), 0, DHT))
    sos = _find(base, 0xDA)
    out.append(("sos unknown component", _patch(base, sos + 5, [9]), 0, SOS))
    out.append(("sos spectral", _patch(base, sos + 7, [1]), 0, SOS))
    out.append(("sos missing table", _patch(base, sos + 6, [0x11]), 0, MISSING_DHT))
    out.append(("no tables", O.jpeg_encode(g, 90, (1, 1), 0, O.JPEG_NO_DHT), 0, MISSING_DHT))
    dri = _find(rst, 0xDD)
    out.append(("dri length", _patch(rst, dri + 2, [0, 5]), 0, DRI))
    r0 = _find(rst[_find(rst, 0xDA):], 0xD0) + _find(rst, 0xDA)
    out.append(("restart out of order", _patch(rst, r0 + 1, [0xD3]), 0, RESET))
    out.append(("restart missing", rst[:r0] + rst[r0 + 2:], 0, RESET))
    c0 = _find(col[_find(col, 0xDA):], 0xD0) + _find(col, 0xDA)
    out.append(("color restart out of order", _patch(col, c0 + 1, [0xD5]), 0, RESET))
    out.append(("zero width", _patch(base, sof + 7, [0, 0]), 0, OK))
    out.append(("empty", b"", 0, OK))
    out.append(("garbage", bytes(np.random.default_rng(7).integers(0, 256, 300, dtype=np.uint8)), 0, None))
    for name, b in (("gray", base), ("restart", rst), ("color", col)):
        for frac in (0.97, 0.6, 0.3):
            out.append((f"{name} truncated {frac}", b[:int(len(b) * frac)], 0, None))
        out.append((f"{name} without EOI", b[:-2], 0, OK))
    return out
