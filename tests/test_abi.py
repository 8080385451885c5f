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


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(at_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_all_declared_symbols():
    L = C.CDLL(AT.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 23
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


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
