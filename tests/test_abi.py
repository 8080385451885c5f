"""CPU tests of the C-ABI boundary: the library loads, exports every entry
point that include/apriltag_fast.h declares, and keeps the reference's
struct layouts. No compute call is made (there is no GPU here)."""
import ctypes as C
import os
import re

import pytest

import apriltags_fast_b200 as AT
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "apriltag_fast.h")
UPSTREAM_HEADERS = [os.path.join(ROOT, "include", h) for h in (
    "apriltag.h", "apriltag_pose.h", "common/matd.h", "common/image_u8.h", "tag16h5.h", "tag25h9.h", "tag36h10.h", "tag36h11.h",
    "tagCircle21h7.h", "tagCircle49h12.h", "tagCustom48h12.h", "tagStandard41h12.h", "tagStandard52h13.h",
    "common/pjpeg.h", "common/image_u8x3.h")]


def declared_functions(path=HEADER, prefix=r"at_\w+"):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"static inline[^{]*\{.*?\n\}", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(" + prefix + r")\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_all_declared_symbols():
    L = C.CDLL(AT.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 23
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_library_exports_the_upstream_api():
    L = C.CDLL(AT.LIB_PATH)
    names = []
    for h in UPSTREAM_HEADERS:
        names += declared_functions(h, r"(?:apriltag|matd|image_u8|tag|estimate|pjpeg)\w+")
    assert "apriltag_detector_detect" in names and "tag36h11_create" in names and len(names) >= 38
    assert "estimate_tag_pose" in names and "pjpeg_to_u8_baseline" in names and "image_u8x3_create" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_upstream_struct_layouts_match_reference(tmp_path):
    """include/apriltag.h keeps the reference apriltag.h layouts (x86-64):
    the numbers below were printed by tests/upstream_layout.c compiled
    against the reference's own apriltag.h."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    exe = str(tmp_path / "layout")
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe,
                           os.path.join(ROOT, "tests", "upstream_layout.c")])
    out = subprocess.check_output([exe]).decode().split("\n")
    assert out[0] == ("family 72 ncodes 0 codes 8 wab 16 tw 20 rb 24 nbits 28 bx 32 by 40 h 48 name 56 impl 64")
    assert out[1] == ("detector 160 nthreads 0 qd 4 qs 8 re 12 ds 16 debug 24 qtp 28 tp 56 nedges 64 nsegments 68 "
                      "nquads 72 tf 80 wp 88 mutex 96 fast 136 fb 144 fc 152")
    assert out[2] == "detection 112 family 0 id 8 hamming 12 dm 16 H 24 c 32 p 48"
    assert out[3] == "qtp 28 zarray 24 matd 16 image_u8 24 timeprofile 16"
    assert out[4] == "info 48 det 0 tagsize 8 fx 16 fy 24 cx 32 cy 40 pose 16 R 0 t 8"
    # common/pjpeg.h and common/image_types.h of the reference
    assert out[5] == ("pjpeg 24 error 0 width 4 height 8 nc 12 comps 16 component 32 w 0 h 4 stride 8 data 16 "
                      "id 24 hv 25 sx 26 sy 27 tq 28 tda 29 u8x3 24")
    assert out[6] == "errors 1 6 8 10 flags 1 2"


def test_struct_layouts_match_reference():
    # fast/apriltag_fast.h: at_detection 168 B (H@16, c@88, p@104),
    # at_detector 160 B, at_family 584 B
    assert C.sizeof(AT.CDetection) == 168
    assert AT.CDetection.H.offset == 16 and AT.CDetection.c.offset == 88 and AT.CDetection.p.offset == 104
    assert C.sizeof(AT.CDetector) == 160
    assert AT.CDetector.qtp.offset == 28 and AT.CDetector.detections.offset == 56
    assert AT.CDetector.timing.offset == 80 and AT.CDetector.internal.offset == 152
    assert C.sizeof(AT.Family) == 584
    assert C.sizeof(O.Detection) == 168 and C.sizeof(O.Family) == 584


@pytest.mark.parametrize("name", AT.FAMILY_NAMES)
def test_builtin_family_tables(name):
    f = AT.family(name)
    assert f.name.decode() == name
    R = O.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref not built")
    r = R.at_family_by_name(name.encode()).contents
    for fld in ("ncodes", "nbits", "h", "width_at_border", "total_width", "reversed_border"):
        assert getattr(f, fld) == getattr(r, fld), fld
    assert list(f.bit_x) == list(r.bit_x) and list(f.bit_y) == list(r.bit_y)
    assert [f.codes[i] for i in range(f.ncodes)] == [r.codes[i] for i in range(r.ncodes)]
