"""CPU tests of the library's host-side parts against the reference compiled
into oracle/_ref: PNM reading and writing (fast/image.c:195-266 of the
reference), the upstream apriltag_to_image (apriltag.c:271-297) for every
built-in family. These functions run on the host only; no GPU is needed."""
import ctypes as C
import os

import numpy as np
import pytest

import apriltags_fast_b200 as AT
from oracle import oracle as O
from tests import helpers as H


class ImageU8(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("stride", C.c_int32), ("buf", C.POINTER(C.c_uint8))]


def _bind(L):
    L.at_read_pnm_into.argtypes = [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                   C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_int64)]
    L.at_read_pnm_into.restype = C.c_bool
    L.at_write_pgm.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_int64]
    L.at_write_pgm.restype = C.c_bool
    L.apriltag_to_image.argtypes = [C.c_void_p, C.c_uint32]
    L.apriltag_to_image.restype = C.POINTER(ImageU8)
    L.image_u8_destroy.argtypes = [C.POINTER(ImageU8)]
    return L


@pytest.fixture(scope="module")
def libs():
    R = O.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref not built")
    return _bind(C.CDLL(AT.LIB_PATH)), _bind(R)


def read_with(L, path, pixels=None, cap=0):
    w, h = C.c_int64(0), C.c_int64(0)
    px = C.POINTER(C.c_uint8)() if pixels is None else pixels
    c = C.c_int64(cap)
    ok = L.at_read_pnm_into(str(path).encode(), C.byref(w), C.byref(h), C.byref(px), C.byref(c))
    if not ok:
        return None
    return np.ctypeslib.as_array(px, shape=(h.value, w.value)).copy()


def _cases(tmp_path):
    rng = np.random.default_rng(7)
    gray = rng.integers(0, 256, size=(37, 53), dtype=np.uint8)
    rgb = rng.integers(0, 256, size=(21, 30, 3), dtype=np.uint8)
    files = {
        "plain_pgm": b"P5\n53 37\n255\n" + gray.tobytes(),
        "comments_pgm": b"P5 # a comment\n# another\n53\t37 #x\n255\n" + gray.tobytes(),
        "ppm": b"P6\n30 21\n255\n" + rgb.tobytes(),
        "truncated": b"P5\n53 37\n255\n" + gray.tobytes()[:-1],
        "maxval_65535": b"P5\n53 37\n65535\n" + gray.tobytes() * 2,
        "ascii_p2": b"P2\n2 2\n255\n1 2 3 4\n",
        "empty": b"",
        "zero_width": b"P5\n0 37\n255\n",
    }
    paths = {}
    for k, v in files.items():
        p = tmp_path / f"{k}.pnm"
        p.write_bytes(v)
        paths[k] = p
    return paths


def test_pnm_reader_matches_reference(libs, tmp_path):
    mine, ref = libs
    for name, path in _cases(tmp_path).items():
        a, b = read_with(mine, path), read_with(ref, path)
        assert (a is None) == (b is None), name
        if a is not None:
            assert a.shape == b.shape and np.array_equal(a, b), name
    for img in H.golden_images():
        p = tmp_path / "g.pgm"
        p.write_bytes(b"P5\n%d %d\n255\n" % (img.shape[1], img.shape[0]) + img.tobytes())
        assert np.array_equal(read_with(mine, p), img)


def test_pnm_reader_reuses_a_large_enough_buffer(libs, tmp_path):
    mine, _ = libs
    p = _cases(tmp_path)["plain_pgm"]
    buf = (C.c_uint8 * (53 * 37))()
    px = C.cast(buf, C.POINTER(C.c_uint8))
    w, h, cap = C.c_int64(0), C.c_int64(0), C.c_int64(53 * 37)
    assert mine.at_read_pnm_into(str(p).encode(), C.byref(w), C.byref(h), C.byref(px), C.byref(cap))
    assert C.addressof(px.contents) == C.addressof(buf) and cap.value == 53 * 37


def test_pgm_write_then_read(libs, tmp_path):
    mine, ref = libs
    img = np.random.default_rng(3).integers(0, 256, size=(19, 41), dtype=np.uint8)
    p = tmp_path / "w.pgm"
    assert mine.at_write_pgm(str(p).encode(), img.ctypes.data, 41, 19)
    assert np.array_equal(read_with(ref, p), img)
    assert not mine.at_write_pgm(str(tmp_path / "no" / "such" / "dir.pgm").encode(), img.ctypes.data, 41, 19)


@pytest.mark.parametrize("name", AT.FAMILY_NAMES)
def test_apriltag_to_image_matches_reference(libs, name):
    mine, ref = libs
    for L in (mine, ref):
        getattr(L, name + "_create").restype = C.c_void_p
        getattr(L, name + "_destroy").argtypes = [C.c_void_p]
    fm, fr = getattr(mine, name + "_create")(), getattr(ref, name + "_create")()
    try:
        ncodes = C.cast(fm, C.POINTER(C.c_uint32))[0]
        for idx in sorted({0, 1, ncodes // 2, ncodes - 1}):
            a, b = mine.apriltag_to_image(fm, idx), ref.apriltag_to_image(fr, idx)
            A, B = a.contents, b.contents
            assert (A.width, A.height) == (B.width, B.height)
            pa = np.ctypeslib.as_array(A.buf, shape=(A.height, A.stride))[:, :A.width]
            pb = np.ctypeslib.as_array(B.buf, shape=(B.height, B.stride))[:, :B.width]
            assert np.array_equal(pa, pb), (name, idx)
            mine.image_u8_destroy(a)
            ref.image_u8_destroy(b)
        assert not mine.apriltag_to_image(fm, ncodes)
    finally:
        getattr(mine, name + "_destroy")(fm)
        getattr(ref, name + "_destroy")(fr)
