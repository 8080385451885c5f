"""apriltags-b200: Python mirror of the AprilTag detector's C API.

The detector itself is libapriltag_b200.so (sm_100a CUDA kernels behind the
C ABI of include/apriltag_fast.h); this module binds it with ctypes and
mirrors the reference's native API (fast/apriltag_fast.h:99-141):

    det = Detector()                  # at_detector_create
    det.add_family("tag36h11", 2)     # at_add_family(td, at_tag36h11(), 2)
    dets = det.detect(image)          # at_detect; list of Detection
    det.nquads                        # td->nquads

There is no CPU path: loading fails loudly if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("APRILTAG_B200_LIB") or os.path.join(_HERE, "libapriltag_b200.so")


class Family(C.Structure):
    """at_family (fast/apriltag_fast.h:24-36)."""

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


class QuadThreshParams(C.Structure):
    _fields_ = [
        ("min_cluster_pixels", C.c_int32),
        ("max_nmaxima", C.c_int32),
        ("critical_rad", C.c_float),
        ("cos_critical_rad", C.c_float),
        ("max_line_fit_mse", C.c_float),
        ("min_white_black_diff", C.c_int32),
        ("deglitch", C.c_bool),
    ]


class CDetection(C.Structure):
    """at_detection (fast/apriltag_fast.h:52-64), 168 bytes."""

    _fields_ = [
        ("family", C.c_int32),
        ("id", C.c_int32),
        ("hamming", C.c_int32),
        ("decision_margin", C.c_float),
        ("H", C.c_double * 9),
        ("c", C.c_double * 2),
        ("p", (C.c_double * 2) * 4),
    ]


class Timing(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("decimate", "blur", "threshold", "unionfind", "clusters", "fit_quads", "decode", "reconcile",
                 "total")]


class CDetector(C.Structure):
    """at_detector (fast/apriltag_fast.h:73-96), 160 bytes."""

    _fields_ = [
        ("nthreads", C.c_int32),
        ("quad_decimate", C.c_float),
        ("quad_sigma", C.c_float),
        ("refine_edges", C.c_bool),
        ("decode_sharpening", C.c_double),
        ("debug", C.c_bool),
        ("qtp", QuadThreshParams),
        ("detections", C.POINTER(CDetection)),
        ("ndetections", C.c_int64),
        ("nquads", C.c_int64),
        ("timing", Timing),
        ("internal", C.c_void_p),
    ]


class Frame(C.Structure):
    _fields_ = [("pixels", C.c_void_p), ("width", C.c_int64), ("height", C.c_int64), ("stride", C.c_int64),
                ("family_mask", C.c_uint32)]


class FrameResult(C.Structure):
    _fields_ = [("first", C.c_int64), ("count", C.c_int64), ("nquads", C.c_int64)]


DIAG = {"quad_image": 0, "threshold": 1, "labels": 2, "points": 3, "clusters": 4, "quads": 5, "sizes": 6,
        "order_roots": 7}
QUAD_DTYPE = np.dtype([("p", np.float32, (4, 2)), ("reversed_border", np.int32), ("frame", np.int32)])
# at_detection as a numpy record (168 bytes)
DETECTION_DTYPE = np.dtype([("family", np.int32), ("id", np.int32), ("hamming", np.int32),
                            ("decision_margin", np.float32), ("H", np.float64, (9,)), ("c", np.float64, (2,)),
                            ("p", np.float64, (4, 2))])
assert DETECTION_DTYPE.itemsize == 168

FAMILY_NAMES = ("tag16h5", "tag25h9", "tag36h10", "tag36h11", "tagCircle21h7", "tagCircle49h12",
                "tagCustom48h12", "tagStandard41h12", "tagStandard52h13")

_lib = None


class ServerConfig(C.Structure):
    _fields_ = [("workers", C.c_int32), ("max_batch", C.c_int32), ("memory_budget", C.c_int64),
                ("device_mask", C.c_uint32)]


class ServerResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("user", C.c_uint64), ("status", C.c_int32), ("batch_frames", C.c_int32),
                ("worker", C.c_int32), ("pad", C.c_int32), ("ndetections", C.c_int64), ("nquads", C.c_int64),
                ("detections", C.POINTER(CDetection)), ("t_submit", C.c_double), ("t_start", C.c_double),
                ("t_done", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("admitted", C.c_int64), ("rejected", C.c_int64), ("completed", C.c_int64), ("batches", C.c_int64),
                ("in_flight", C.c_int64), ("pending", C.c_int64), ("cancelled", C.c_int64),
                ("peak_arena_bytes", C.c_int64), ("bytes_per_pixel", C.c_double)]


SERVER_CANCELLED = -1  # at_server_result.status of a cancelled request


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m apriltags_fast_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.at_detector_create.restype = C.POINTER(CDetector)
        L.at_detector_destroy.argtypes = [C.POINTER(CDetector)]
        L.at_add_family.argtypes = [C.POINTER(CDetector), C.POINTER(Family), C.c_int]
        L.at_add_family.restype = C.c_bool
        L.at_clear_families.argtypes = [C.POINTER(CDetector)]
        L.at_family_name.argtypes = [C.POINTER(CDetector), C.POINTER(CDetection)]
        L.at_family_name.restype = C.c_char_p
        L.at_detect.argtypes = [C.POINTER(CDetector), C.c_void_p, C.c_int64, C.c_int64, C.c_int64]
        L.at_detect_batch.argtypes = [C.POINTER(CDetector), C.POINTER(Frame), C.c_int64, C.POINTER(FrameResult)]
        L.at_shutdown.argtypes = [C.POINTER(CDetector)]
        L.at_detector_last_error.argtypes = [C.POINTER(CDetector), C.POINTER(C.c_char_p)]
        L.at_detector_last_error.restype = C.c_int
        L.at_detector_diag.argtypes = [C.POINTER(CDetector), C.c_int, C.c_void_p, C.c_int64]
        L.at_detector_diag.restype = C.c_int64
        L.at_detector_set_batch_split.argtypes = [C.POINTER(CDetector), C.c_int]
        L.at_detector_set_batch_split.restype = C.c_int
        L.at_server_create.argtypes = [C.POINTER(CDetector), C.POINTER(ServerConfig)]
        L.at_server_create.restype = C.c_void_p
        L.at_server_submit.argtypes = [C.c_void_p, C.POINTER(Frame), C.c_uint64]
        L.at_server_submit.restype = C.c_uint64
        L.at_server_cancel.argtypes = [C.c_void_p, C.c_uint64]
        L.at_server_cancel.restype = C.c_int
        L.at_server_poll.argtypes = [C.c_void_p, C.POINTER(ServerResult), C.c_int64, C.c_int32]
        L.at_server_poll.restype = C.c_int64
        L.at_server_free_result.argtypes = [C.POINTER(ServerResult)]
        L.at_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.at_server_destroy.argtypes = [C.c_void_p]
        L.at_server_worker_device.argtypes = [C.c_void_p, C.c_int32]
        L.at_server_worker_device.restype = C.c_int
        L.at_family_by_name.argtypes = [C.c_char_p]
        L.at_family_by_name.restype = C.POINTER(Family)
        for n in FAMILY_NAMES:
            getattr(L, "at_" + n).restype = C.POINTER(Family)
        _lib = L
    return _lib


def family(name: str) -> Family:
    """A built-in family (at_family_by_name); KeyError if unknown."""
    p = lib().at_family_by_name(name.encode())
    if not p:
        raise KeyError(f"no built-in family {name!r} (was the library built with the family tables?)")
    return p.contents


def family_codes(name: str) -> np.ndarray:
    f = family(name)
    return np.ctypeslib.as_array(f.codes, shape=(f.ncodes,)).copy()


@dataclass
class Detection:
    family: int
    id: int
    hamming: int
    decision_margin: float
    H: tuple
    c: tuple
    p: tuple

    def key(self) -> tuple:
        return (self.family, self.id, self.hamming, self.decision_margin, self.H, self.c, self.p)


def _detection(d: CDetection) -> Detection:
    return Detection(int(d.family), int(d.id), int(d.hamming), float(d.decision_margin), tuple(d.H), tuple(d.c),
                     tuple(tuple(r) for r in d.p))


class Detector:
    """Mirror of at_detector: the same parameters, the same defaults."""

    def __init__(self, families=(), bits_corrected: int = 2, **params):
        self._L = lib()
        self._td = self._L.at_detector_create()
        self._fams = []
        for f in families:
            self.add_family(f, bits_corrected)
        for k, v in params.items():
            self.set(k, v)

    def set(self, name, value):
        td = self._td.contents
        if hasattr(td.qtp, name) and name not in ("detections",):
            setattr(td.qtp, name, value)
        elif name in ("nthreads", "quad_decimate", "quad_sigma", "refine_edges", "decode_sharpening", "debug"):
            setattr(td, name, value)
        else:
            raise AttributeError(name)

    @property
    def params(self) -> CDetector:
        return self._td.contents

    def add_family(self, fam, bits_corrected: int = 2) -> bool:
        f = family(fam) if isinstance(fam, str) else fam
        ok = bool(self._L.at_add_family(self._td, C.byref(f), bits_corrected))
        if ok:
            self._fams.append(f)
        return ok

    def clear_families(self):
        self._L.at_clear_families(self._td)
        self._fams = []

    def detect(self, img, stride: int | None = None) -> list[Detection]:
        """Detect on a u8 image: a 2-D numpy array (host) or a uint8 CUDA
        torch tensor (device memory, read in place)."""
        ptr, w, h, s = _image_arg(img, stride)
        self._L.at_detect(self._td, ptr, w, h, s)
        self._check()
        td = self._td.contents
        return [_detection(td.detections[i]) for i in range(td.ndetections)]

    def detect_batch(self, images, family_masks=None, as_arrays: bool = False):
        """at_detect_batch over images of any sizes. Returns per frame a list
        of Detection, or with as_arrays a numpy record array (DETECTION_DTYPE,
        a copy of the library's at_detection array) per frame."""
        n = len(images)
        frames = (Frame * max(n, 1))()
        keep = []
        for i, img in enumerate(images):
            ptr, w, h, s = _image_arg(img, None)
            keep.append(img)
            frames[i] = Frame(ptr, w, h, s, 0 if family_masks is None else family_masks[i])
        res = (FrameResult * max(n, 1))()
        self._L.at_detect_batch(self._td, frames, n, res)
        self._check()
        td = self._td.contents
        self.last_batch_nquads = [int(res[i].nquads) for i in range(n)]
        if as_arrays:
            total = int(td.ndetections)
            if total:
                buf = C.cast(td.detections, C.POINTER(C.c_uint8 * (168 * total))).contents
                allv = np.frombuffer(buf, DETECTION_DTYPE, total).copy()
            else:
                allv = np.zeros(0, DETECTION_DTYPE)
            return [allv[res[i].first:res[i].first + res[i].count] for i in range(n)]
        return [[_detection(td.detections[res[i].first + k]) for k in range(res[i].count)] for i in range(n)]

    def _check(self):
        msg = C.c_char_p()
        code = self._L.at_detector_last_error(self._td, C.byref(msg))
        if code:
            raise RuntimeError(f"apriltag_b200 error {code}: {msg.value.decode() if msg.value else ''}")

    @property
    def nquads(self) -> int:
        return int(self._td.contents.nquads)

    @property
    def timing(self) -> dict:
        t = self._td.contents.timing
        return {n: getattr(t, n) for n, _ in Timing._fields_}

    def set_batch_split(self, pipelines: int) -> None:
        """Spread large batches over this many pipelines (1-4, default 3),
        each with its own streams, arenas and host thread; the results do
        not depend on it."""
        if self._L.at_detector_set_batch_split(self._td, int(pipelines)) != 0:
            raise ValueError("pipelines must be 1 to 4")

    def diag(self, what: str) -> np.ndarray:
        """An intermediate array of the last detection (frame 0), for
        stage-by-stage checks: quad_image, threshold, labels, points,
        clusters, quads, sizes or order_roots (rows of (smallest node,
        root) for the components beside quads whose ids repeat, in the
        reference's packed node numbering)."""
        code = DIAG[what]
        sizes = np.zeros(6, np.int64)
        self._L.at_detector_diag(self._td, DIAG["sizes"], sizes.ctypes.data, 48)
        if what == "sizes":
            return sizes
        nbytes = self._L.at_detector_diag(self._td, code, None, 0)
        buf = np.zeros(max(int(nbytes), 0), np.uint8)
        if nbytes > 0:
            self._L.at_detector_diag(self._td, code, buf.ctypes.data, nbytes)
        qw, qh = int(sizes[0]), int(sizes[1])
        if what in ("quad_image", "threshold"):
            return buf.reshape(qh, qw)
        if what == "labels":
            return buf.view(np.uint32).reshape(qh, qw)
        if what == "points":
            return buf.view(np.uint64)
        if what == "clusters":
            return buf.view(np.uint32)
        if what == "order_roots":
            return buf.view(np.uint32).reshape(-1, 2)
        return buf.view(QUAD_DTYPE)

    def family_name(self, d: Detection) -> str:
        return self._fams[d.family].name.decode()

    def shutdown(self):
        self._L.at_shutdown(self._td)

    def close(self):
        if getattr(self, "_td", None):
            self._L.at_detector_destroy(self._td)
            self._td = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Mirror of at_server: continuous batching over `workers` detectors made
    from `detector` (its parameters and families). submit() returns a ticket
    (0: rejected); the image must stay alive and unchanged until its result
    has been polled. poll() returns finished results as dicts with the
    detections as a numpy record array (DETECTION_DTYPE). `devices`: the
    GPUs to deal the workers out over (one detector replica per worker;
    None: the current GPU)."""

    def __init__(self, detector: "Detector", workers: int = 2, max_batch: int = 16, memory_budget: int = 24 << 30,
                 devices=None):
        self._L = lib()
        mask = 0
        for d in devices or ():
            mask |= 1 << int(d)
        cfg = ServerConfig(workers, max_batch, memory_budget, mask)
        self._s = self._L.at_server_create(detector._td, C.byref(cfg))
        if not self._s:
            raise RuntimeError("at_server_create failed")
        self._keep = {}

    def submit(self, img, user: int = 0, family_mask: int = 0) -> int:
        ptr, w, h, s = _image_arg(img, None)
        f = Frame(ptr, w, h, s, family_mask)
        t = int(self._L.at_server_submit(self._s, C.byref(f), user))
        if t:
            self._keep[t] = img
        return t

    def worker_device(self, worker: int) -> int:
        """The GPU of worker `worker` (a result's "worker"), or -1."""
        return int(self._L.at_server_worker_device(self._s, int(worker)))

    def cancel(self, ticket: int) -> bool:
        """Cancel a request still in the queue (its result comes back with
        status SERVER_CANCELLED); False when it already runs or is done."""
        return bool(self._L.at_server_cancel(self._s, int(ticket)))

    def poll(self, max_results: int = 256, wait_ms: int = 0) -> list:
        buf = (ServerResult * max_results)()
        n = int(self._L.at_server_poll(self._s, buf, max_results, wait_ms))
        out = []
        for i in range(n):
            r = buf[i]
            nd = int(r.ndetections)
            if nd:
                raw = C.cast(r.detections, C.POINTER(C.c_uint8 * (168 * nd))).contents
                dets = np.frombuffer(raw, DETECTION_DTYPE, nd).copy()
            else:
                dets = np.zeros(0, DETECTION_DTYPE)
            out.append({"ticket": int(r.ticket), "user": int(r.user), "status": int(r.status),
                        "detections": dets, "nquads": int(r.nquads), "batch_frames": int(r.batch_frames),
                        "worker": int(r.worker), "t_submit": r.t_submit, "t_start": r.t_start, "t_done": r.t_done})
            self._L.at_server_free_result(C.byref(buf[i]))
            self._keep.pop(int(r.ticket), None)
        return out

    def stats(self) -> dict:
        st = ServerStats()
        self._L.at_server_get_stats(self._s, C.byref(st))
        return {n: getattr(st, n) for n, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_s", None):
            self._L.at_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _image_arg(img, stride):
    if hasattr(img, "data_ptr") and getattr(img, "is_cuda", False):
        assert img.dtype.__str__() == "torch.uint8" and img.dim() == 2
        h, w = img.shape
        return C.c_void_p(img.data_ptr()), w, h, int(img.stride(0))
    a = np.asarray(img)
    if a.dtype != np.uint8 or a.ndim != 2:
        raise TypeError("image must be a 2-D uint8 array")
    if not a.flags["C_CONTIGUOUS"] and a.strides[1] != 1:
        a = np.ascontiguousarray(a)
    h, w = a.shape
    return C.c_void_p(a.ctypes.data), w, h, int(stride or a.strides[0])


# --------------------------------------------------------------------------
# JPEG input (csrc/at_jpeg.cu): baseline JPEG decoded on the GPU, pixels and
# error codes as the reference's common/pjpeg.c gives them.

PJPEG_MJPEG = 2
JPEG_ERRORS = ("OKAY", "FILE", "DQT", "SOF", "DHT", "SOS", "MISSING_DHT", "DRI", "RESET", "EOF", "UNSUPPORTED")


class _PJComponent(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("stride", C.c_uint32),
                ("data", C.POINTER(C.c_uint8)), ("id", C.c_uint8), ("hv", C.c_uint8), ("scalex", C.c_uint8),
                ("scaley", C.c_uint8), ("tq", C.c_uint8), ("tda", C.c_uint8)]


class _PJ(C.Structure):
    _fields_ = [("error", C.c_int), ("width", C.c_uint32), ("height", C.c_uint32), ("ncomponents", C.c_int),
                ("components", C.POINTER(_PJComponent))]


class _ImageU8x3(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("stride", C.c_int32), ("buf", C.POINTER(C.c_uint8))]


_jpeg_bound = False


def _jpeg_lib():
    global _jpeg_bound
    L = lib()
    if not _jpeg_bound:
        L.at_jpeg_create.restype = C.c_void_p
        L.at_jpeg_destroy.argtypes = [C.c_void_p]
        L.at_jpeg_info.argtypes = [C.c_char_p, C.c_int64, C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_int32)]
        L.at_jpeg_info.restype = C.c_int
        L.at_jpeg_decode_gray.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_int64),
                                          C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.c_int32,
                                          C.POINTER(C.c_int32)]
        L.at_jpeg_decode_gray.restype = C.c_int
        L.at_jpeg_last_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.at_jpeg_set_sub_bits.argtypes = [C.c_void_p, C.c_int32]
        L.at_jpeg_set_threads.argtypes = [C.c_void_p, C.c_int32]
        L.at_jpeg_set_run_in.argtypes = [C.c_void_p, C.c_int32]
        L.pjpeg_create_from_buffer.argtypes = [C.c_char_p, C.c_int, C.c_uint32, C.POINTER(C.c_int)]
        L.pjpeg_create_from_buffer.restype = C.POINTER(_PJ)
        L.pjpeg_destroy.argtypes = [C.POINTER(_PJ)]
        L.pjpeg_to_u8x3_baseline.argtypes = [C.POINTER(_PJ)]
        L.pjpeg_to_u8x3_baseline.restype = C.POINTER(_ImageU8x3)
        L.image_u8x3_destroy.argtypes = [C.POINTER(_ImageU8x3)]
        _jpeg_bound = True
    return L


def jpeg_info(buf: bytes, flags: int = 0):
    """(error, width, height, components) of the gray frame a decode gives."""
    L = _jpeg_lib()
    w, h, n = C.c_int32(), C.c_int32(), C.c_int32()
    e = L.at_jpeg_info(buf, len(buf), flags, C.byref(w), C.byref(h), C.byref(n))
    return e, w.value, h.value, n.value


class JpegDecoder:
    """Decodes batches of baseline JPEGs on the GPU into gray frames
    (component 0 cropped to the image, as pjpeg_to_u8_baseline gives it)."""

    def __init__(self, sub_bits: int | None = None, threads: int = 0, run_in: int | None = None):
        self._L = _jpeg_lib()
        self._d = self._L.at_jpeg_create()
        if not self._d:
            raise RuntimeError("at_jpeg_create failed (no CUDA device?)")
        if sub_bits is not None and self._L.at_jpeg_set_sub_bits(self._d, sub_bits):
            raise ValueError("sub_bits must be a multiple of 32 in [64, 65536]")
        if self._L.at_jpeg_set_threads(self._d, threads):
            raise ValueError("threads must be in [0, 256]")
        if run_in is not None and self._L.at_jpeg_set_run_in(self._d, run_in):
            raise ValueError("run_in must be in [0, 2**20]")

    def _call(self, bufs, dsts, strides, on_device, flags):
        n = len(bufs)
        cb = (C.c_char_p * n)(*bufs)
        cl = (C.c_int64 * n)(*[len(b) for b in bufs])
        cd = (C.c_void_p * n)(*dsts)
        cs = (C.c_int64 * n)(*strides)
        errs = (C.c_int32 * n)()
        r = self._L.at_jpeg_decode_gray(self._d, n, cb, cl, flags, cd, cs, int(on_device), errs)
        if r < 0:
            raise RuntimeError("at_jpeg_decode_gray: CUDA error")
        return list(errs)

    def decode(self, bufs, flags: int = 0):
        """Host numpy frames (None where an image failed) and error codes."""
        infos = [jpeg_info(b, flags) for b in bufs]
        outs = [np.zeros((max(h, 1), max(w, 1)), np.uint8) if e == 0 else np.zeros((1, 1), np.uint8)
                for e, w, h, _ in infos]
        errs = self._call(bufs, [o.ctypes.data for o in outs], [o.strides[0] for o in outs], False, flags)
        res = [o[:h, :w] if e == 0 else None for o, e, (_, w, h, _) in zip(outs, errs, infos)]
        return res, errs

    def decode_device(self, bufs, flags: int = 0, pad: int = 0):
        """torch.uint8 CUDA frames (rows padded by `pad` bytes) and error codes."""
        import torch
        infos = [jpeg_info(b, flags) for b in bufs]
        outs = [torch.zeros((max(h, 1), max(w, 1) + pad), dtype=torch.uint8, device="cuda") for _, w, h, _ in infos]
        errs = self._call(bufs, [o.data_ptr() for o in outs], [o.stride(0) for o in outs], True, flags)
        return [o[:h, :w] if e == 0 else None for o, e, (_, w, h, _) in zip(outs, errs, infos)], errs

    def last_stats(self) -> dict:
        a = (C.c_double * 10)()
        self._L.at_jpeg_last_stats(self._d, a)
        return dict(parse_ms=a[0], copy_in_ms=a[1], sync_ms=a[2], write_ms=a[3], copy_out_ms=a[4],
                    substreams=int(a[5]), extra_passes=int(a[6]), entropy_bytes=int(a[7]),
                    cta_rounds=int(a[8]))

    def close(self):
        if self._d:
            self._L.at_jpeg_destroy(self._d)
            self._d = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pjpeg_decode(buf: bytes, flags: int = 0):
    """Through the pjpeg.h drop-in: (error, width, height, [planes])."""
    L = _jpeg_lib()
    err = C.c_int(0)
    pj = L.pjpeg_create_from_buffer(buf, len(buf), flags, C.byref(err))
    if not pj:
        return err.value, 0, 0, []
    try:
        p = pj.contents
        planes = []
        for i in range(p.ncomponents):
            c = p.components[i]
            n = c.height * c.stride
            planes.append(np.ctypeslib.as_array(c.data, shape=(n,)).reshape(c.height, c.stride).copy()
                          if n else np.zeros((c.height, c.stride), np.uint8))
        return err.value, p.width, p.height, planes
    finally:
        L.pjpeg_destroy(pj)


def pjpeg_rgb(buf: bytes, flags: int = 0):
    """pjpeg_to_u8x3_baseline of the drop-in: (h, w, 3) array or None."""
    L = _jpeg_lib()
    err = C.c_int(0)
    pj = L.pjpeg_create_from_buffer(buf, len(buf), flags, C.byref(err))
    if not pj:
        return None
    try:
        im = L.pjpeg_to_u8x3_baseline(pj)
        if not im:
            return None
        try:
            m = im.contents
            a = np.ctypeslib.as_array(m.buf, shape=(m.height * m.stride,)).reshape(m.height, m.stride)
            return a[:, :3 * m.width].reshape(m.height, m.width, 3).copy()
        finally:
            L.image_u8x3_destroy(im)
    finally:
        L.pjpeg_destroy(pj)
