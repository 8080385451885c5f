"""The allocation-free threshold entry point (at_threshold_noalloc).

Some callers of this library cannot allocate device memory (their frame
loop may not absorb the device-wide synchronisation of cudaMalloc, or a pool
or framework owns all of the GPU's memory and only hands them buffers).
at_threshold_noalloc serves them: they pass device input and output, and
its scratch is a fixed array of the library. This test calls it through the
C ABI twice in a row, on two different images, and checks each output
against the threshold image of the detector's own at_detect (the tolerance
is zero: bytes must be equal). It runs alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import apriltags_fast_b200 as AT
from apriltags_fast_b200 import synth
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _reference_threshold(img):
    det = AT.Detector(["tag36h11"], 1)
    det.detect(img)
    return det.diag("quad_image").copy(), det.diag("threshold").copy()


def test_threshold_noalloc_two_calls():
    import torch

    L = AT.lib()
    fn = L.at_threshold_noalloc
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    images = [H.golden_images()[0], synth.make_frame(synth.CONFIGS["1080p"], 3)[0]]
    for img in images:  # two calls in a row through the shared scratch
        qim, thr = _reference_threshold(img)
        qh, qw = qim.shape
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
