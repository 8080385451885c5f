"""The JPEG input path on the CPU: the oracle's restatement of the
reference's decoder (oracle/at_jpeg.c, after common/pjpeg.c) against the
reference itself built from its sources (oracle/_ref), the test encoder,
and the host side of the GPU decoder (header walk, sizes, error codes)."""
import glob
import os

import numpy as np
import pytest

import apriltags_fast_b200 as AT
import oracle.oracle as O

from tests.jpeg_cases import MISSING_DHT, RESET, SOF, SOS, bad_files, encode_matrix


def same(a, b):
    return a[0] == b[0] and a[1:3] == b[1:3] and len(a[3]) == len(b[3]) and all(
        x.shape == y.shape and (x == y).all() for x, y in zip(a[3], b[3]))


def need_ref():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")


def test_encoder_round_trip_is_close():
    """The test encoder writes what it was given (PSNR of a smooth image)."""
    y, x = np.mgrid[0:120, 0:160]
    img = (128 + 60 * np.sin(x / 9.0) * np.cos(y / 13.0)).astype(np.uint8)
    for samp in ((1, 1), (2, 2)):
        e, w, h, p = O.jpeg_decode(O.jpeg_encode(img, 95, samp))
        assert e == 0 and (w, h) == (160, 120)
        g = O.gray_of(w, h, p).astype(float)
        assert 10 * np.log10(255 ** 2 / np.mean((g - img) ** 2)) > 38


def test_oracle_equals_reference_on_the_encoder_matrix():
    need_ref()
    for name, buf, flags in encode_matrix(small=True):
        assert same(O.jpeg_decode(buf, flags), O.ref_jpeg_decode(buf, flags)), name


def test_oracle_equals_reference_on_bad_and_truncated_files():
    need_ref()
    for name, buf, flags, _ in bad_files():
        a, r = O.jpeg_decode(buf, flags), O.ref_jpeg_decode(buf, flags)
        assert same(a, r), (name, a[0], r[0])


def test_bad_files_give_the_expected_codes():
    for name, buf, flags, code in bad_files():
        if code is not None:
            assert O.jpeg_decode(buf, flags)[0] == code, name


def test_reference_photos():
    """The reference's own test photos (APRILTAG_REFERENCE=<checkout>)."""
    need_ref()
    ref = os.environ.get("APRILTAG_REFERENCE")
    files = sorted(glob.glob(os.path.join(ref, "test", "data", "*.jpg"))) if ref else []
    if not files:
        pytest.skip("APRILTAG_REFERENCE not set")
    for f in files:
        buf = open(f, "rb").read()
        assert same(O.jpeg_decode(buf), O.ref_jpeg_decode(buf)), f
        assert AT.jpeg_info(buf)[:3] == (0, 799, 533)


def test_host_header_walk_matches_the_oracle():
    """at_jpeg_info reads the headers up to the first scan (host only): the
    oracle's frame size for files that decode, and the oracle's error for
    files whose headers fail before the first scan."""
    for name, buf, flags in encode_matrix(small=True):
        e, w, h, _ = O.jpeg_decode(buf, flags)
        assert AT.jpeg_info(buf, flags)[:3] == (e, w, h), name
    for name, buf, flags, _ in bad_files():
        e, w, h, p = O.jpeg_decode(buf, flags)
        ie, iw, ih, _ = AT.jpeg_info(buf, flags)
        if ie:
            assert e == ie or (e == 0 and all(x.size == 0 for x in p)), name  # a header error, or no scan
        elif e == 0:
            assert (iw, ih) == (w, h), name
        else:
            assert e in (RESET, MISSING_DHT, SOS, SOF), (name, e)  # found in or after the first scan


def test_oracle_equals_reference_on_1080p_frames():
    """Frames of the benchmark's size: gray and 4:2:0 with restart markers."""
    need_ref()
    from apriltags_fast_b200 import synth

    cfg = synth.Config(1920, 1080, ntags=(24, 24), side=(30, 220), tilt_deg=60.0, noise=4.0, distractors=200)
    img = synth.make_frame(cfg, 3)[0]
    rgb = np.stack([img, np.roll(img, 4, 1), 255 - img], -1)
    for buf in (O.jpeg_encode(img, 90), O.jpeg_encode(rgb, 85, (2, 2), 30, O.JPEG_OPTIMIZE)):
        assert same(O.jpeg_decode(buf), O.ref_jpeg_decode(buf))


def test_decoder_fails_loudly_without_a_gpu():
    """No CPU fallback: without a CUDA device the decoder cannot be made and
    the pjpeg.h drop-in reports PJPEG_ERR_FILE instead of decoding."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError):
        AT.JpegDecoder()
    g = (np.arange(64 * 48) % 251).astype(np.uint8).reshape(48, 64)
    assert AT.pjpeg_decode(O.jpeg_encode(g, 90))[0] == 1
