"""Tag pose on the GPU (at_estimate_poses, and the upstream estimate_tag_pose
family of include/apriltag_pose.h) against the reference's own
apriltag_pose.c compiled into oracle/_ref. The 3x3 algebra is grouped
differently and the SVD is the library's own, so the tolerance is 1e-9
relative (measured differences are about 1e-12); which of the two poses is
chosen, and whether a second pose exists, must agree."""
import ctypes as C

import numpy as np
import pytest

import apriltags_fast_b200 as AT
from apriltags_fast_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-9
CAM = (0.16, 1000.0, 1000.0, 960.0, 540.0)  # tag side (m), fx, fy, cx, cy (px)


class Matd(C.Structure):
    _fields_ = [("nrows", C.c_uint), ("ncols", C.c_uint), ("data", C.POINTER(C.c_double))]


class ApDet(C.Structure):
    _fields_ = [("family", C.c_void_p), ("id", C.c_int), ("hamming", C.c_int), ("decision_margin", C.c_float),
                ("H", C.POINTER(Matd)), ("c", C.c_double * 2), ("p", (C.c_double * 2) * 4)]


class Info(C.Structure):
    _fields_ = [("det", C.POINTER(ApDet)), ("tagsize", C.c_double), ("fx", C.c_double), ("fy", C.c_double),
                ("cx", C.c_double), ("cy", C.c_double)]


class Pose(C.Structure):
    _fields_ = [("R", C.POINTER(Matd)), ("t", C.POINTER(Matd))]


class AtPose(C.Structure):
    _fields_ = [("R", C.c_double * 9), ("t", C.c_double * 3), ("err", C.c_double), ("R2", C.c_double * 9),
                ("t2", C.c_double * 3), ("err2", C.c_double)]


def _bind(L):
    L.matd_create_data.restype = C.POINTER(Matd)
    L.matd_create_data.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.estimate_tag_pose.argtypes = [C.POINTER(Info), C.POINTER(Pose)]
    L.estimate_tag_pose.restype = C.c_double
    L.estimate_tag_pose_orthogonal_iteration.argtypes = [C.POINTER(Info), C.POINTER(C.c_double), C.POINTER(Pose),
                                                         C.POINTER(C.c_double), C.POINTER(Pose), C.c_int]
    L.estimate_pose_for_tag_homography.argtypes = [C.POINTER(Info), C.POINTER(Pose)]
    return L


def _info(L, d):
    H = (C.c_double * 9)(*d.H)
    det = ApDet(None, d.id, d.hamming, d.decision_margin, L.matd_create_data(3, 3, H), (C.c_double * 2)(*d.c),
                ((C.c_double * 2) * 4)(*[(C.c_double * 2)(*q) for q in d.p]))
    return Info(C.pointer(det), *CAM), det


def _close(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.all(np.abs(a - b) <= TOL * np.maximum(1.0, np.abs(b)))


def _frames():
    return [synth.make_frame(synth.CONFIGS["1080p"], s)[0] for s in range(3)]


@pytest.fixture(scope="module")
def libs():
    R = O.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref not built")
    return _bind(C.CDLL(AT.LIB_PATH)), _bind(R)


def test_batched_poses_match_reference(libs):
    mine, ref = libs
    L = AT.lib()
    L.at_estimate_poses.argtypes = [C.c_void_p] + [C.c_double] * 5 + [C.c_void_p]
    L.at_estimate_poses.restype = C.c_int
    det = AT.Detector(["tag36h11"], 2)
    n = two = 0
    for img in _frames():
        dets = det.detect(img)
        out = (AtPose * max(1, len(dets)))()
        assert L.at_estimate_poses(C.cast(det._td, C.c_void_p), *CAM, out) == 0
        for d, p in zip(dets, out):
            info, keep = _info(ref, d)
            e1, e2 = C.c_double(), C.c_double()
            p1, p2 = Pose(), Pose()
            ref.estimate_tag_pose_orthogonal_iteration(C.byref(info), C.byref(e1), C.byref(p1), C.byref(e2),
                                                       C.byref(p2), 50)
            assert _close(p.R, p1.R.contents.data[:9]) and _close(p.t, p1.t.contents.data[:3])
            assert abs(p.err - e1.value) <= TOL * max(1e-12, abs(e1.value))
            assert bool(p2.R) == (p.err2 != float("inf"))
            if p2.R:
                two += 1
                assert _close(p.R2, p2.R.contents.data[:9]) and _close(p.t2, p2.t.contents.data[:3])
            n += 1
    assert n >= 60 and two >= n // 2


def test_upstream_pose_api_matches_reference(libs):
    mine, ref = libs
    det = AT.Detector(["tag36h11"], 2)
    dets = det.detect(_frames()[0])[:8]
    assert dets
    for d in dets:
        ia, ka = _info(mine, d)
        ib, kb = _info(ref, d)
        pa, pb = Pose(), Pose()
        ea = mine.estimate_tag_pose(C.byref(ia), C.byref(pa))
        eb = ref.estimate_tag_pose(C.byref(ib), C.byref(pb))
        assert abs(ea - eb) <= TOL * max(1e-12, abs(eb))
        assert _close(pa.R.contents.data[:9], pb.R.contents.data[:9])
        assert _close(pa.t.contents.data[:3], pb.t.contents.data[:3])
        ha, hb = Pose(), Pose()
        mine.estimate_pose_for_tag_homography(C.byref(ia), C.byref(ha))
        ref.estimate_pose_for_tag_homography(C.byref(ib), C.byref(hb))
        assert _close(ha.R.contents.data[:9], hb.R.contents.data[:9])
        assert _close(ha.t.contents.data[:3], hb.t.contents.data[:3])
