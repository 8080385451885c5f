"""GPU parity: the CUDA detector, called through its C ABI, against the CPU
oracle on the same inputs. Integer, byte and index results must be equal;
the floating point results too (bit-exact: the tolerance is zero), since
the kernels round every operation as the reference does."""
import os

import numpy as np
import pytest

import apriltags_fast_b200 as AT
from apriltags_fast_b200 import synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = H.golden_cases()


def gpu_detect(img, fams, bits, prm):
    det = AT.Detector()
    for f, b in zip(fams, bits):
        assert det.add_family(f, b)
    for k, v in prm.items():
        det.set(k, v)
    dets = det.detect(img)
    return det, [d.key() for d in dets]


def oracle_detect(img, fams, bits, prm, order=O.ORDER_CANON):
    return O.detect(img, [H.oracle_family(f) for f in fams], bits, O.default_params(**prm), order=order)


def oracle_pixel_labels(r, min_px):
    """The oracle's labels per pixel, renumbered as the GPU numbers nodes
    (run i of row y: y*qw + i; last-column node of row y: qw*qh + y)."""
    qw, qh = r.qw, r.qh
    nruns = len(r.run_start)
    ro = r.row_off.astype(np.int64)

    def gpu_id(L):
        L = int(L)
        if L >= nruns:
            return qw * qh + (L - nruns)
        y = int(np.searchsorted(ro, L, side="right")) - 1
        return y * qw + (L - ro[y])

    out = np.full((qh, qw), 0xffffffff, np.uint32)
    for y in range(qh):
        for n in range(ro[y], ro[y + 1]):
            if r.comp_pixels[n] >= min_px:
                out[y, r.run_start[n]:r.run_end[n] + 1] = gpu_id(r.label[n])
        v = nruns + y
        if r.comp_pixels[v] >= min_px:
            out[y, qw - 1] = gpu_id(r.label[v])
    return out


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_golden_cases_gpu(case):
    """Each golden case: GPU detections == oracle (same order), the quad
    count too, and the reference's golden hex lines as a multiset."""
    name, fam, ham, prm = case
    lines = []
    for path, im in zip(H.IMAGES, H.golden_images()):
        det, g = gpu_detect(im, [fam], [ham], prm)
        r = oracle_detect(im, [fam], [ham], prm)
        assert det.nquads == len(r.quads)
        assert g == r.dets
        lines += [O.hex_line(path, d) for d in g]
    assert sorted(lines) == sorted(H.golden_hex(name))


@pytest.mark.parametrize("img_i", [0, 1])
def test_stage_parity_default(img_i):
    """Every stage of the default configuration on the reference's images."""
    im = H.golden_images()[img_i]
    det, g = gpu_detect(im, ["tag36h11"], [1], {})
    r = oracle_detect(im, ["tag36h11"], [1], {})
    assert np.array_equal(det.diag("quad_image"), r.qim)
    assert np.array_equal(det.diag("threshold"), r.thresh)
    assert np.array_equal(det.diag("labels"), oracle_pixel_labels(r, 24))
    assert np.array_equal(det.diag("points"), r.pts)
    assert np.array_equal(det.diag("clusters"), r.cstart[:-1])
    q = det.diag("quads")
    assert len(q) == len(r.quads)
    for a, b in zip(q, r.quads):
        assert tuple(map(tuple, a["p"].tolist())) == b[0] and int(a["reversed_border"]) == b[1]
    assert g == r.dets


def _synth_case(name, seed, **over):
    cfg = synth.CONFIGS[name]
    for k, v in over.items():
        setattr(cfg, k, v)
    img, truth = synth.make_frame(cfg, seed)
    return cfg, img, truth


@pytest.mark.parametrize("seed", range(4))
def test_synthetic_640(seed):
    cfg, img, truth = _synth_case("640x480", seed)
    det, g = gpu_detect(img, list(cfg.families), [2], {})
    r = oracle_detect(img, list(cfg.families), [2], {})
    assert det.nquads == len(r.quads)
    assert g == r.dets
    assert len(g) == len(truth)


@pytest.mark.parametrize("seed", range(2))
def test_synthetic_1080p(seed):
    cfg, img, truth = _synth_case("1080p", seed)
    det, g = gpu_detect(img, list(cfg.families), [2], {})
    r = oracle_detect(img, list(cfg.families), [2], {})
    assert det.nquads == len(r.quads)
    assert np.array_equal(det.diag("threshold"), r.thresh)
    assert np.array_equal(det.diag("points"), r.pts)
    assert g == r.dets


@pytest.mark.parametrize("dec", [2.0, 1.0])
def test_large_frame_two_families(dec):
    cfg, img, truth = _synth_case("4032x3024", 7)
    fams = list(cfg.families)
    det, g = gpu_detect(img, fams, [2, 2], {"quad_decimate": dec})
    r = oracle_detect(img, fams, [2, 2], {"quad_decimate": dec})
    assert det.nquads == len(r.quads)
    assert g == r.dets


def test_batch_equals_single():
    """A batch of uneven frames gives, per frame, what one frame alone gives."""
    imgs = []
    for i, (name, seed) in enumerate([("640x480", 11), ("1080p", 12), ("640x480", 13)]):
        imgs.append(_synth_case(name, seed)[1])
    imgs.append(H.golden_images()[1])
    det = AT.Detector(["tag36h11"], 2)
    batch = det.detect_batch(imgs)
    bq = det.last_batch_nquads
    for i, im in enumerate(imgs):
        single = det.detect(im)
        assert [d.key() for d in batch[i]] == [d.key() for d in single]
        assert bq[i] == det.nquads


def test_edge_cases():
    det = AT.Detector()
    img = H.golden_images()[0]
    assert det.detect(img) == [] and det.nquads == 0  # no families
    det.add_family("tag36h11", 1)
    assert det.detect(np.zeros((7, 100), np.uint8)) == []  # below 8 pixels
    assert det.detect(np.zeros((8, 8), np.uint8)) == []
    assert det.detect(np.full((64, 64), 200, np.uint8)) == []
    # a strided view: same as the packed copy
    big = np.zeros((480, 700), np.uint8)
    big[:, 30:670] = img
    view = big[:, 30:670]
    assert [d.key() for d in det.detect(view)] == [d.key() for d in det.detect(np.ascontiguousarray(view))]
    # device memory input, read in place
    import torch

    t = torch.from_numpy(img).cuda()
    assert [d.key() for d in det.detect(t)] == [d.key() for d in det.detect(img)]


def test_parameter_limits_fail_loudly():
    det = AT.Detector(["tag36h11"], 1)
    det.set("max_nmaxima", 40)
    with pytest.raises(RuntimeError):
        det.detect(H.golden_images()[0])
    assert not det.add_family("tag25h9", 4)


@pytest.mark.parametrize("family,bits", [("tag36h11", 2), ("tagStandard41h12", 1)])
def test_upstream_api_equals_native(tmp_path, family, bits):
    """apriltag_detector_detect (include/apriltag.h) returns exactly the
    native at_detect's detections, in the same order (apriltag.c:152-208 of
    the reference is the same wrapper), from a C program linked against the
    library."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    libdir = os.path.dirname(AT.LIB_PATH)
    exe = str(tmp_path / "upstream_detect")
    subprocess.check_call(["gcc", "-O1", "-I", os.path.join(ROOT, "include"), "-o", exe,
                           os.path.join(ROOT, "tests", "upstream_detect.c"), "-L", libdir, "-lapriltag_b200",
                           "-Wl,-rpath," + libdir])
    out = []
    for img in ("synth_640x480_000.pgm", "synth_640x480_001.pgm"):
        txt = subprocess.check_output([exe, os.path.join(H.GOLDEN, img), family, str(bits)]).decode()
        lines = txt.strip().split("\n")
        up = [l[2:] for l in lines if l.startswith("U ")]
        nat = [l[2:] for l in lines if l.startswith("N ")]
        assert up == nat and len(up) > 0
        nq = [l for l in lines if l.startswith("nquads")][0].split()
        assert nq[1] == [l for l in lines if l.startswith("native nquads")][0].split()[2]
        assert nq[3] == "9"
        assert "after clear 0" in lines
        tw = AT.family(family).total_width
        assert f"tag image {tw} {tw}" in lines
        out += up
    assert len(out) > 0
