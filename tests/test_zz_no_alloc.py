"""The allocation-free threshold entry point (at_threshold_noalloc).

Some callers of this library cannot allocate device memory (their frame
loop may not absorb the device-wide synchronisation of cudaMalloc, or a pool
or framework owns all of the GPU's memory and only hands them buffers).
at_threshold_noalloc serves them: they pass device input and output, and
its scratch is a fixed array of the library. This test calls it through the
C ABI on three different images in a row, and checks each output against the
threshold image of the detector's own at_detect (the tolerance is zero: bytes
must be equal). The third image has sides that are not multiples of 4 and a
flat band along its right and bottom edges, so the rows and columns past the
last whole tile (which reuse the last tile and are never flat) are covered.
It runs alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import apriltags_fast_b200 as AT
from apriltags_fast_b200 import synth
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _reference_threshold(img, decimate=2.0):
    det = AT.Detector(["tag36h11"], 1, quad_decimate=decimate)
    det.detect(img)
    return det.diag("quad_image").copy(), det.diag("threshold").copy()


def _odd_frame():
    """643 x 485 (decimate 1: the quad image is the frame), a tag frame
    with a flat band (one gray level) along the right and bottom edges."""
    img = synth.make_frame(synth.CONFIGS["640x480"], 11)[0]
    out = np.full((485, 643), 140, np.uint8)
    out[:480, :640] = img
    out[:, 620:] = 140
    out[460:, :] = 140
    return out


def test_threshold_noalloc_two_calls():
    import torch

    L = AT.lib()
    fn = L.at_threshold_noalloc
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    images = [(H.golden_images()[0], 2.0), (synth.make_frame(synth.CONFIGS["1080p"], 3)[0], 2.0),
              (_odd_frame(), 1.0)]
    for img, dec in images:  # calls in a row through the shared scratch
        qim, thr = _reference_threshold(img, dec)
        qh, qw = qim.shape
        if dec == 1.0:
            assert qw % 4 == 3 and qh % 4 == 1 and (thr == 127).any()
        d_in = torch.from_numpy(qim).cuda()
        d_out = torch.full_like(d_in, 7)
        rc = fn(d_in.data_ptr(), qw, qh, 5, d_out.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == 0
        assert np.array_equal(d_out.cpu().numpy(), thr)


def test_threshold_noalloc_refuses_sizes():
    L = AT.lib()
    fn = L.at_threshold_noalloc
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    assert fn(None, 8192, 8192, 5, None, None) == 1  # above the fixed scratch
    assert fn(None, 3, 100, 5, None, None) == 1      # below one tile
