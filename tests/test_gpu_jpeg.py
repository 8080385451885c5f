"""GPU JPEG decode (csrc/at_jpeg.cu) through its C ABI against the CPU
oracle (oracle/at_jpeg.c, pinned to the reference's common/pjpeg.c by
tests/test_jpeg_oracle.py) and, where it is built, the reference's own
decoder (oracle/_ref). Pixels and error codes must be equal byte for byte.
A gray frame is component 0 cropped to the image (pjpeg_to_u8_baseline);
where the reference would read outside its planes there (no scan of
component 0, or a plane smaller than the image) the GPU decoder refuses
the image with an error code instead."""
import numpy as np
import pytest

import apriltags_fast_b200 as AT
from apriltags_fast_b200 import synth
from oracle import oracle as O
from tests import helpers as H
from tests.jpeg_cases import bad_files, encode_matrix

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dec():
    d = AT.JpegDecoder()
    yield d
    d.close()


def expected_gray(buf, flags):
    """(error or 'refused', frame) as the oracle decodes the file."""
    e, w, h, p = O.jpeg_decode(buf, flags)
    if e:
        return e, None
    if not p or p[0].shape[0] < h or p[0].shape[1] < w:
        return "refused", None
    return 0, O.gray_of(w, h, p)


def check_batch(dec, cases, device=False, pad=0):
    by_flags = {}
    for name, buf, flags, *_ in cases:
        by_flags.setdefault(flags, []).append((name, buf))
    for flags, items in by_flags.items():
        bufs = [b for _, b in items]
        if device:
            frames, errs = dec.decode_device(bufs, flags, pad)
            frames = [f.cpu().numpy() if f is not None else None for f in frames]
        else:
            frames, errs = dec.decode(bufs, flags)
        for (name, buf), f, e in zip(items, frames, errs):
            xe, xf = expected_gray(buf, flags)
            if xe == "refused":
                assert e != 0, name
                continue
            assert e == xe, (name, e, xe)
            if xe == 0:
                assert f.shape == xf.shape and (f == xf).all(), name


def frames_1080p():
    out = []
    cfg = synth.Config(1920, 1080)
    for seed, q in ((0, 75), (1, 90), (2, 95)):
        img = synth.make_frame(cfg, seed)
        img = img[0] if isinstance(img, tuple) else img
        out.append((f"1080p q{q}", O.jpeg_encode(img, q), 0))
        rgb = np.stack([img, np.roll(img, 3, 1), 255 - img], -1)
        out.append((f"1080p 4:2:0 q{q}", O.jpeg_encode(rgb, q, (2, 2), 0, O.JPEG_OPTIMIZE), 0))
    out.append(("1080p restart 8", O.jpeg_encode(img, 85, (1, 1), 8), 0))
    return out


def test_matrix_to_host_frames(dec):
    check_batch(dec, encode_matrix(small=False))


def test_bad_and_truncated_files(dec):
    check_batch(dec, bad_files())


def test_device_frames_with_padded_rows(dec):
    check_batch(dec, encode_matrix(small=True), device=True, pad=13)


def test_1080p_frames_one_batch(dec):
    cases = frames_1080p()
    check_batch(dec, cases, device=True)
    st = dec.last_stats()
    assert st["substreams"] > 1000 and st["entropy_bytes"] > 500_000


@pytest.mark.parametrize("bits", [64, 256, 2048, 65536])
def test_substream_size_does_not_change_pixels(bits):
    d = AT.JpegDecoder(sub_bits=bits)
    try:
        check_batch(d, frames_1080p()[:2] + encode_matrix(small=True)[::7])
    finally:
        d.close()


def test_pjpeg_dropin_planes_and_rgb():
    """pjpeg_create_from_buffer gives the reference's planes (every
    component, padding columns zero) and pjpeg_to_u8x3_baseline its RGB."""
    ref = O.ref_lib() is not None
    for name, buf, flags in encode_matrix(small=True)[::3] + [frames_1080p()[1]]:
        a = AT.pjpeg_decode(buf, flags)
        b = O.jpeg_decode(buf, flags)
        assert a[:3] == b[:3] and len(a[3]) == len(b[3]), name
        for x, y in zip(a[3], b[3]):
            assert x.shape == y.shape and (x == y).all(), name
        if ref:
            r = O.ref_jpeg_rgb(buf, flags)
            g = AT.pjpeg_rgb(buf, flags)
            assert (r is None) == (g is None), name
            if r is not None:
                assert (r == g).all(), name


def test_detect_on_a_decoded_jpeg(dec):
    """Camera frame as JPEG -> GPU decode into device memory -> detector on
    that device frame: the detections of the reference's pixels."""
    cfg = synth.Config(1920, 1080)
    img = synth.make_frame(cfg, 4)
    img = img[0] if isinstance(img, tuple) else img
    buf = O.jpeg_encode(img, 92)
    frames, errs = dec.decode_device([buf])
    assert errs == [0]
    e, w, h, p = O.jpeg_decode(buf)
    host = O.gray_of(w, h, p)
    det = AT.Detector()
    assert det.add_family("tag36h11", 2)
    got = [d.key() for d in det.detect(frames[0])]
    want = O.detect(host, [H.oracle_family("tag36h11")], [2], O.default_params(), order=O.ORDER_REF).dets
    assert got == want and len(got) >= 3


def _flip_entropy(buf, rng, nflips):
    """Random bytes of the entropy-coded data changed, none of them an FF,
    next to an FF, or made into one (the markers stay where they were)."""
    b = bytearray(buf)
    sos = buf.find(b"\xff\xda")
    lo = sos + 2 + (buf[sos + 2] << 8 | buf[sos + 3])
    hi = len(buf) - 2
    done = 0
    while done < nflips:
        i = int(rng.integers(lo + 1, hi - 1))
        if 0xFF in (b[i - 1], b[i], b[i + 1]):
            continue
        v = int(rng.integers(0, 255))  # never 0xFF
        if v == b[i]:
            continue
        b[i] = v
        done += 1
    return bytes(b)


def test_damaged_entropy_data_equals_the_oracle(dec):
    """Damaged scans decode as the oracle decodes them (codes that match
    nothing, runs past the last coefficient, decodes that stop moving),
    gray, 4:2:0 with restart markers, and 4:4:4, with no fault."""
    rng = np.random.default_rng(42)
    cfg = synth.Config(640, 480)
    img = synth.make_frame(cfg, 9)[0]
    rgb = np.stack([img, np.roll(img, 5, 0), 255 - img], -1)
    bases = [O.jpeg_encode(img, 90), O.jpeg_encode(rgb, 80, (2, 2), 6), O.jpeg_encode(rgb, 95, (1, 1))]
    cases = []
    for k, base in enumerate(bases):
        for n in (1, 3, 8, 40):
            for rep in range(3):
                cases.append((f"base{k} flips{n} #{rep}", _flip_entropy(base, rng, n), 0))
    check_batch(dec, cases)
    check_batch(dec, cases[::5], device=True, pad=3)
