"""GPU parity: the CUDA detector, called through its C ABI, against the CPU
oracle on the same inputs. Integer, byte and index results must be equal;
the floating point results too (bit-exact: the tolerance is zero), since
the kernels round every operation as the reference does. Detections are
compared in the reference's own output order (ORDER_REF: the order the
reference's union-find roots give same-id detections); the GPU's internal
arrays (points, clusters, quads) are in its own cluster order, which the
oracle also has (ORDER_CANON)."""
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


def oracle_detect(img, fams, bits, prm, order=O.ORDER_REF):
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
    count too, and the reference's golden hex lines, line for line."""
    name, fam, ham, prm = case
    lines = []
    for path, im in zip(H.IMAGES, H.golden_images()):
        det, g = gpu_detect(im, [fam], [ham], prm)
        r = oracle_detect(im, [fam], [ham], prm)
        assert det.nquads == len(r.quads)
        assert g == r.dets
        lines += [O.hex_line(path, d) for d in g]
    assert lines == H.golden_hex(name)


@pytest.mark.parametrize("img_i", [0, 1])
def test_stage_parity_default(img_i):
    """Every stage of the default configuration on the reference's images."""
    im = H.golden_images()[img_i]
    det, g = gpu_detect(im, ["tag36h11"], [1], {})
    r = oracle_detect(im, ["tag36h11"], [1], {}, order=O.ORDER_CANON)
    assert np.array_equal(det.diag("quad_image"), r.qim)
    assert np.array_equal(det.diag("threshold"), r.thresh)
    assert np.array_equal(det.diag("labels"), oracle_pixel_labels(r, 24))
    assert np.array_equal(det.diag("points"), r.pts)
    assert np.array_equal(det.diag("clusters"), r.cstart[:-1])
    q = det.diag("quads")
    assert len(q) == len(r.quads)
    for a, b in zip(q, r.quads):
        assert tuple(map(tuple, a["p"].tolist())) == b[0] and int(a["reversed_border"]) == b[1]
    assert g == oracle_detect(im, ["tag36h11"], [1], {}).dets


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
    r = oracle_detect(img, list(cfg.families), [2], {}, order=O.ORDER_CANON)
    assert det.nquads == len(r.quads)
    assert np.array_equal(det.diag("threshold"), r.thresh)
    assert np.array_equal(det.diag("points"), r.pts)
    assert g == oracle_detect(img, list(cfg.families), [2], {}).dets


def _dup_seeds(name, count, start=1000):
    """Seeds whose frame (codes drawn with replacement) holds two tags of
    one id."""
    cfg = synth.Config(**{**synth.CONFIGS[name].__dict__, "replacement": True})
    out, seed = [], start
    while len(out) < count:
        img, truth = synth.make_frame(cfg, seed)
        ids = [t.id for t in truth]
        if len(set(ids)) < len(ids):
            out.append((seed, img))
        seed += 1
    return cfg, out


def test_1080p_duplicate_ids_in_reference_order():
    """20 seeded 1080p frames whose tag codes are drawn with replacement
    and hold a repeated id: the GPU's detections equal the reference's own
    (oracle/_ref, the reference compiled from its sources, one thread), in
    its order. Same-id detections are ordered by the reference's union-find
    roots, so this checks the order replay on the GPU."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    cfg, frames = _dup_seeds("1080p", 20)
    det = AT.Detector(list(cfg.families), 2)
    repeated = 0
    for seed, img in frames:
        g = [d.key() for d in det.detect(img)]
        ref, nq = O.ref_detect(img, list(cfg.families), [2])
        assert det.nquads == nq, seed
        assert g == ref, seed
        ids = [d[1] for d in ref]
        repeated += len(ids) != len(set(ids))
    assert repeated >= 15  # most frames keep both copies of a repeated id


def test_order_roots_equal_the_oracle_roots():
    """Stage check of the order replay: for each component beside a quad
    whose id repeats, the root that the GPU's replay finds equals the root
    of the reference's sequential union by size, as the oracle computes it
    (fast/unionfind.c:15-45, 152-196), in the reference's node numbering."""
    cfg, frames = _dup_seeds("1080p", 6, start=3000)
    det = AT.Detector(list(cfg.families), 2)
    fams = [H.oracle_family(f) for f in cfg.families]
    checked = 0
    for seed, img in frames:
        det.detect(img)
        pairs = det.diag("order_roots")
        r = O.detect(img, fams, [2] * len(fams), O.default_params(), order=O.ORDER_REF)
        for label, root in pairs:
            assert r.label[label] == label, (seed, label)
            assert r.ref_root[label] == root, (seed, label, int(r.ref_root[label]), int(root))
        checked += len(pairs)
    assert checked >= 20


def test_1080p_duplicate_ids_batched():
    """The same frames in one batch (the order replay runs per frame)."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    cfg, frames = _dup_seeds("1080p", 8, start=2000)
    det = AT.Detector(list(cfg.families), 2)
    out = det.detect_batch([img for _, img in frames])
    for (seed, img), got in zip(frames, out):
        ref, _ = O.ref_detect(img, list(cfg.families), [2])
        assert [d.key() for d in got] == ref, seed


@pytest.mark.parametrize("family", ["tagCircle49h12", "tagCustom48h12", "tagStandard52h13", "tag16h5"])
@pytest.mark.parametrize("dec", [2.0, 1.0])
def test_family_decode_vs_reference(family, dec):
    """Families with large quick-decode tables (tagCircle49h12: 65535 codes,
    13-bit chunks; tagCustom48h12: 42211; tagStandard52h13: 48714) and the
    smallest (tag16h5): 8 tags of 90-200 px on 1280x720, three seeds, bits
    2, against the reference itself in its order."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    det = AT.Detector([family], 2, quad_decimate=dec)
    n = 0
    for seed in range(3):
        cfg = synth.Config(1280, 720, families=(family,), ntags=(8, 8), side=(90, 200), tilt_deg=40.0)
        img, truth = synth.make_frame(cfg, seed)
        g = [d.key() for d in det.detect(img)]
        ref, nq = O.ref_detect(img, [family], [2], O.default_params(quad_decimate=dec))
        assert g == ref and det.nquads == nq, seed
        n += len(g)
    assert n >= 20


@pytest.mark.parametrize("seed", range(2, 8))
def test_synthetic_1080p_more_seeds(seed):
    """More seeds of the 1080p workload, detections in the reference's order."""
    cfg, img, truth = _synth_case("1080p", seed)
    det, g = gpu_detect(img, list(cfg.families), [2], {})
    r = oracle_detect(img, list(cfg.families), [2], {})
    assert det.nquads == len(r.quads)
    assert g == r.dets


@pytest.mark.parametrize("seed", [7, 8, 9])
@pytest.mark.parametrize("dec", [2.0, 1.0])
def test_large_frame_two_families(dec, seed):
    cfg, img, truth = _synth_case("4032x3024", seed)
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
    assert not det.add_family("tag25h9", -1)


def test_family_limit_is_16():
    """The reference takes at most 16 families (fast/detector.c:45-54): the
    17th is refused and detection goes on with the first 16."""
    det = AT.Detector()
    names = list(AT.FAMILY_NAMES)
    for i in range(16):
        assert det.add_family(names[i % len(names)], 1)
    assert not det.add_family("tag36h11", 1)
    img = H.golden_images()[0]
    g = [d.key() for d in det.detect(img)]
    assert len(g) > 0
    if O.ref_lib() is not None:  # tag36h11 twice: same-id detections of two families, in the reference's order
        ref, nq = O.ref_detect(img, [names[i % len(names)] for i in range(16)], [1] * 16)
        assert g == ref and det.nquads == nq


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
        # the batch call: each copy of the image gives the single call's
        # detections, the crop none; the quad count is the batch's total
        for k in (0, 2, 3):
            assert [l[3:] for l in lines if l.startswith(f"B{k} ")] == up
        assert not [l for l in lines if l.startswith("B1 ")]
        nq = [l for l in lines if l.startswith("nquads")][0].split()
        assert int([l for l in lines if l.startswith("batch nquads")][0].split()[2]) == 3 * int(nq[1])
        # a page-locked buffer: the same detections
        assert [l[2:] for l in lines if l.startswith("R ")] == nat
        assert "registered 0 unregistered 0" in lines
        assert nq[1] == [l for l in lines if l.startswith("native nquads")][0].split()[2]
        assert nq[3] == "9"
        assert "after clear 0" in lines
        tw = AT.family(family).total_width
        assert f"tag image {tw} {tw}" in lines
        out += up
    assert len(out) > 0
