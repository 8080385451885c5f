"""ctypes binding of the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY.

Used by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg to check the GPU library. Nothing in the product imports this module.

Also binds the reference library compiled from its own sources into
``oracle/_ref/`` (when it was built here), for stage-by-stage comparisons.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORDER_REF = 0
ORDER_CANON = 1


class Family(C.Structure):
    """The reference's ``at_family`` layout (fast/apriltag_fast.h:24-36)."""

    _fields_ = [
        ("name", C.c_char * 32),
        ("codes", C.POINTER(C.c_uint64)),
        ("ncodes", C.c_int64),
        ("nbits", C.c_int32),
        ("h", C.c_int32),
        ("width_at_border", C.c_int32),
        ("total_width", C.c_int32),
        ("reversed_border", C.c_bool),
        ("bit_x", C.c_int32 * 64),
        ("bit_y", C.c_int32 * 64),
    ]


class Detection(C.Structure):
    """The reference's ``at_detection`` layout (fast/apriltag_fast.h:52-64)."""

    _fields_ = [
        ("family", C.c_int32),
        ("id", C.c_int32),
        ("hamming", C.c_int32),
        ("decision_margin", C.c_float),
        ("H", C.c_double * 9),
        ("c", C.c_double * 2),
        ("p", (C.c_double * 2) * 4),
    ]


class Params(C.Structure):
    _fields_ = [
        ("quad_decimate", C.c_float),
        ("quad_sigma", C.c_float),
        ("refine_edges", C.c_int32),
        ("decode_sharpening", C.c_double),
        ("min_cluster_pixels", C.c_int32),
        ("max_nmaxima", C.c_int32),
        ("cos_critical_rad", C.c_float),
        ("max_line_fit_mse", C.c_float),
        ("min_white_black_diff", C.c_int32),
        ("deglitch", C.c_int32),
    ]


class Quad(C.Structure):
    _fields_ = [("p", (C.c_float * 2) * 4), ("reversed_border", C.c_int32), ("cluster", C.c_int32)]


class Result(C.Structure):
    _fields_ = [
        ("qw", C.c_int64),
        ("qh", C.c_int64),
        ("qim", C.POINTER(C.c_uint8)),
        ("thresh", C.POINTER(C.c_uint8)),
        ("nruns", C.c_int64),
        ("run_start", C.POINTER(C.c_uint16)),
        ("run_end", C.POINTER(C.c_uint16)),
        ("run_v", C.POINTER(C.c_uint8)),
        ("row_off", C.POINTER(C.c_uint32)),
        ("nnodes", C.c_int64),
        ("label", C.POINTER(C.c_uint32)),
        ("ref_root", C.POINTER(C.c_uint32)),
        ("comp_pixels", C.POINTER(C.c_uint32)),
        ("npoints", C.c_int64),
        ("nclusters", C.c_int64),
        ("cstart", C.POINTER(C.c_uint32)),
        ("cid", C.POINTER(C.c_uint64)),
        ("pts", C.POINTER(C.c_uint64)),
        ("nquads", C.c_int64),
        ("quads", C.POINTER(Quad)),
        ("ndet", C.c_int64),
        ("dets", C.POINTER(Detection)),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run `make -C oracle`)")
        L = C.CDLL(path)
        L.ao_default_params.argtypes = [C.POINTER(Params)]
        L.ao_detect.argtypes = [C.POINTER(Params), C.POINTER(Family), C.POINTER(C.c_int32), C.c_int32,
                                C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int32, C.POINTER(Result)]
        L.ao_detect.restype = C.c_int
        L.ao_result_free.argtypes = [C.POINTER(Result)]
        L.ao_keysort.argtypes = [C.c_void_p, C.c_int64]
        for f in ("ao_cosf", "ao_sinf"):
            getattr(L, f).argtypes = [C.c_float]
            getattr(L, f).restype = C.c_float
        L.ao_atan2f.argtypes = [C.c_float, C.c_float]
        L.ao_atan2f.restype = C.c_float
        _lib = L
    return _lib


def default_params(**kw) -> Params:
    p = Params()
    lib().ao_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def det_tuple(d) -> tuple:
    """A detection as a hashable tuple of its exact values."""
    return (int(d.family), int(d.id), int(d.hamming), float(d.decision_margin), tuple(d.H), tuple(d.c),
            tuple(tuple(r) for r in d.p))


@dataclass
class FrameResult:
    qw: int
    qh: int
    qim: np.ndarray
    thresh: np.ndarray
    run_start: np.ndarray
    run_end: np.ndarray
    run_v: np.ndarray
    row_off: np.ndarray
    label: np.ndarray
    ref_root: np.ndarray
    comp_pixels: np.ndarray
    cstart: np.ndarray
    cid: np.ndarray
    pts: np.ndarray
    quads: list
    dets: list


def _arr(ptr, n, dt):
    if n <= 0 or not ptr:
        return np.zeros(0, dt)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)


def detect(img: np.ndarray, families, bits, params: Params | None = None, order=ORDER_CANON) -> FrameResult:
    """Run the oracle on a u8 image (h, w). families: sequence of Family."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape
    if params is None:
        params = default_params()
    nf = len(families)
    fams = (Family * max(nf, 1))(*families)
    b = (C.c_int32 * max(nf, 1))(*bits)
    r = Result()
    rc = lib().ao_detect(C.byref(params), fams, b, nf, img.ctypes.data, w, h, w, order, C.byref(r))
    if rc != 0:
        lib().ao_result_free(C.byref(r))
        raise ValueError("oracle refused the families")
    try:
        qw, qh = r.qw, r.qh
        nn = r.nnodes
        out = FrameResult(
            qw=qw, qh=qh,
            qim=_arr(r.qim, qw * qh, np.uint8).reshape(qh, qw) if r.qim else np.zeros((0, 0), np.uint8),
            thresh=_arr(r.thresh, qw * qh, np.uint8).reshape(qh, qw) if r.thresh else np.zeros((0, 0), np.uint8),
            run_start=_arr(r.run_start, r.nruns, np.uint16),
            run_end=_arr(r.run_end, r.nruns, np.uint16),
            run_v=_arr(r.run_v, r.nruns, np.uint8),
            row_off=_arr(r.row_off, qh + 1, np.uint32) if r.row_off else np.zeros(0, np.uint32),
            label=_arr(r.label, nn, np.uint32),
            ref_root=_arr(r.ref_root, nn, np.uint32),
            comp_pixels=_arr(r.comp_pixels, nn, np.uint32),
            cstart=_arr(r.cstart, r.nclusters + 1, np.uint32) if r.cstart else np.zeros(1, np.uint32),
            cid=_arr(r.cid, r.nclusters, np.uint64),
            pts=_arr(r.pts, r.npoints, np.uint64),
            quads=[(tuple(tuple(p) for p in r.quads[i].p), int(r.quads[i].reversed_border), int(r.quads[i].cluster))
                   for i in range(r.nquads)],
            dets=[det_tuple(r.dets[i]) for i in range(r.ndet)],
        )
    finally:
        lib().ao_result_free(C.byref(r))
    return out


def keysort(keys: np.ndarray) -> np.ndarray:
    k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    lib().ao_keysort(k.ctypes.data, len(k))
    return k


# ---------------------------------------------------------------------------
# Hex lines in the format of the reference demo's --hex-detections
# (example/fast_demo.c:185-189): C's %a of each value.

_libc = C.CDLL(None)


def hexf(x: float) -> str:
    buf = C.create_string_buffer(64)
    _libc.snprintf(buf, 64, b"%a", C.c_double(x))
    return buf.value.decode()


def hex_line(path: str, d: tuple) -> str:
    fam, did, ham, margin, H, c, p = d
    parts = [path, str(did), str(ham), hexf(margin), hexf(c[0]), hexf(c[1])]
    for q in p:
        parts += [hexf(q[0]), hexf(q[1])]
    parts += [hexf(v) for v in H]
    return " ".join(parts)


# ---------------------------------------------------------------------------
# The reference library compiled into oracle/_ref (test infrastructure).

_ref = None


def ref_lib():
    """The unmodified reference built by `make -C oracle ref`, or None."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libapriltag_ref.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.at_family_by_name.argtypes = [C.c_char_p]
        L.at_family_by_name.restype = C.POINTER(Family)
        _ref = L
    return _ref


class _QTP(C.Structure):
    _fields_ = [("min_cluster_pixels", C.c_int32), ("max_nmaxima", C.c_int32), ("critical_rad", C.c_float),
                ("cos_critical_rad", C.c_float), ("max_line_fit_mse", C.c_float),
                ("min_white_black_diff", C.c_int32), ("deglitch", C.c_bool)]


class _RefDetector(C.Structure):
    """The reference's at_detector layout (fast/apriltag_fast.h:73-96)."""

    _fields_ = [("nthreads", C.c_int32), ("quad_decimate", C.c_float), ("quad_sigma", C.c_float),
                ("refine_edges", C.c_bool), ("decode_sharpening", C.c_double), ("debug", C.c_bool),
                ("qtp", _QTP), ("detections", C.POINTER(Detection)), ("ndetections", C.c_int64),
                ("nquads", C.c_int64), ("timing", C.c_double * 9), ("internal", C.c_void_p)]


def ref_detect(img: np.ndarray, family_names, bits, params: Params | None = None, nthreads: int = 1):
    """Run the reference itself (oracle/_ref) on an image: (detections, nquads).
    Detections in the reference's output order."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref not built (make -C oracle ref)")
    R.at_detector_create.restype = C.POINTER(_RefDetector)
    R.at_detector_destroy.argtypes = [C.POINTER(_RefDetector)]
    R.at_add_family.argtypes = [C.POINTER(_RefDetector), C.POINTER(Family), C.c_int]
    R.at_add_family.restype = C.c_bool
    R.at_detect.argtypes = [C.POINTER(_RefDetector), C.c_void_p, C.c_int64, C.c_int64, C.c_int64]
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape
    p = params or default_params()
    td = R.at_detector_create()
    try:
        for n, b in zip(family_names, bits):
            if not R.at_add_family(td, R.at_family_by_name(n.encode()), b):
                raise ValueError("reference refused the family")
        d = td.contents
        d.nthreads = nthreads
        d.quad_decimate = p.quad_decimate
        d.quad_sigma = p.quad_sigma
        d.refine_edges = bool(p.refine_edges)
        d.decode_sharpening = p.decode_sharpening
        d.qtp.min_cluster_pixels = p.min_cluster_pixels
        d.qtp.max_nmaxima = p.max_nmaxima
        d.qtp.cos_critical_rad = p.cos_critical_rad
        d.qtp.max_line_fit_mse = p.max_line_fit_mse
        d.qtp.min_white_black_diff = p.min_white_black_diff
        d.qtp.deglitch = bool(p.deglitch)
        R.at_detect(td, img.ctypes.data, w, h, w)
        d = td.contents
        return [det_tuple(d.detections[i]) for i in range(d.ndetections)], int(d.nquads)
    finally:
        R.at_detector_destroy(td)


# --------------------------------------------------------------------------
# JPEG input path (oracle/at_jpeg.c; the reference's common/pjpeg.c)

JPEG_MJPEG = 2
JPEG_OPTIMIZE, JPEG_NO_DHT, JPEG_MARKERS, JPEG_ONE_DQT = 1, 2, 4, 8


class _OJPlane(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("stride", C.c_uint32),
                ("data", C.POINTER(C.c_uint8)), ("id", C.c_uint8), ("hv", C.c_uint8), ("scalex", C.c_uint8),
                ("scaley", C.c_uint8), ("tq", C.c_uint8), ("tda", C.c_uint8)]


class _OJImage(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("ncomponents", C.c_int),
                ("comp", _OJPlane * 3)]


class _PJPEG(C.Structure):
    """The reference's pjpeg_t (common/pjpeg.h:64-72); its component type
    has the oracle's plane layout (common/pjpeg.h:38-62)."""

    _fields_ = [("error", C.c_int), ("width", C.c_uint32), ("height", C.c_uint32), ("ncomponents", C.c_int),
                ("components", C.POINTER(_OJPlane))]


def _planes(comps, n):
    out = []
    for i in range(n):
        c = comps[i]
        a = np.ctypeslib.as_array(c.data, shape=(c.height * c.stride,)).reshape(c.height, c.stride) \
            if c.height * c.stride else np.zeros((c.height, c.stride), np.uint8)
        out.append(a.copy())
    return out


def jpeg_encode(img: np.ndarray, quality: int = 90, sampling=(1, 1), restart: int = 0, flags: int = 0) -> bytes:
    """Test inputs: the package's synthetic-input encoder (synth.encode_jpeg)."""
    from apriltags_fast_b200 import synth

    return synth.encode_jpeg(img, quality, sampling, restart, flags)


def jpeg_decode(buf: bytes, flags: int = 0):
    """The oracle's decode: (error, width, height, [component planes])."""
    L = lib()
    L.oj_decode.argtypes = [C.c_char_p, C.c_int64, C.c_uint32, C.POINTER(_OJImage)]
    L.oj_decode.restype = C.c_int
    L.oj_free.argtypes = [C.POINTER(_OJImage)]
    im = _OJImage()
    e = L.oj_decode(buf, len(buf), flags, C.byref(im))
    if e:
        return e, 0, 0, []
    try:
        return 0, im.width, im.height, _planes(im.comp, im.ncomponents)
    finally:
        L.oj_free(C.byref(im))


def ref_jpeg_decode(buf: bytes, flags: int = 0):
    """The reference's own pjpeg (oracle/_ref), same return as jpeg_decode."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref not built (make -C oracle ref)")
    R.pjpeg_create_from_buffer.argtypes = [C.c_char_p, C.c_int, C.c_uint32, C.POINTER(C.c_int)]
    R.pjpeg_create_from_buffer.restype = C.POINTER(_PJPEG)
    R.pjpeg_destroy.argtypes = [C.POINTER(_PJPEG)]
    err = C.c_int(0)
    pj = R.pjpeg_create_from_buffer(buf, len(buf), flags, C.byref(err))
    if not pj:
        return err.value, 0, 0, []
    try:
        p = pj.contents
        return err.value, p.width, p.height, _planes(p.components, p.ncomponents)
    finally:
        R.pjpeg_destroy(pj)


def gray_of(width: int, height: int, planes) -> np.ndarray:
    """Component 0 cropped to the image (pjpeg_to_u8_baseline)."""
    return np.ascontiguousarray(planes[0][:height, :width])


def ref_jpeg_rgb(buf: bytes, flags: int = 0):
    """The reference's pjpeg_to_u8x3_baseline (oracle/_ref): (h, w, 3) or None."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref not built (make -C oracle ref)")

    class U8x3(C.Structure):
        _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("stride", C.c_int32),
                    ("buf", C.POINTER(C.c_uint8))]

    R.pjpeg_create_from_buffer.argtypes = [C.c_char_p, C.c_int, C.c_uint32, C.POINTER(C.c_int)]
    R.pjpeg_create_from_buffer.restype = C.POINTER(_PJPEG)
    R.pjpeg_destroy.argtypes = [C.POINTER(_PJPEG)]
    R.pjpeg_to_u8x3_baseline.argtypes = [C.POINTER(_PJPEG)]
    R.pjpeg_to_u8x3_baseline.restype = C.POINTER(U8x3)
    R.image_u8x3_destroy.argtypes = [C.POINTER(U8x3)]
    err = C.c_int(0)
    pj = R.pjpeg_create_from_buffer(buf, len(buf), flags, C.byref(err))
    if not pj:
        return None
    try:
        if pj.contents.ncomponents != 3:
            return None
        im = R.pjpeg_to_u8x3_baseline(pj)
        try:
            m = im.contents
            a = np.ctypeslib.as_array(m.buf, shape=(m.height * m.stride,)).reshape(m.height, m.stride)
            return a[:, :3 * m.width].reshape(m.height, m.width, 3).copy()
        finally:
            R.image_u8x3_destroy(im)
    finally:
        R.pjpeg_destroy(pj)
