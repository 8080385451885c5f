"""CPU tests of the oracle: pinned to the reference's golden vectors and,
where the reference was compiled here (oracle/_ref), to the reference
itself on seeded synthetic frames."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import helpers as H

CASES = H.golden_cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_golden_vectors(case):
    """The oracle in the reference's order reproduces test/golden/<case>.hex
    byte for byte (the reference's own test/run_golden.sh check)."""
    name, fam, ham, prm = case
    imgs = H.golden_images()
    f = H.oracle_family(fam)
    p = O.default_params(**prm)
    lines = []
    for path, im in zip(H.IMAGES, imgs):
        r = O.detect(im, [f], [ham], p, order=O.ORDER_REF)
        lines += [O.hex_line(path, d) for d in r.dets]
    assert lines == H.golden_hex(name)


@pytest.mark.parametrize("case", CASES[:8], ids=[c[0] for c in CASES[:8]])
def test_canonical_order_same_results(case):
    """The GPU's cluster order gives the same clusters, quads and detections
    as the reference's order, up to order."""
    name, fam, ham, prm = case
    f = H.oracle_family(fam)
    p = O.default_params(**prm)
    for im in H.golden_images():
        a = O.detect(im, [f], [ham], p, order=O.ORDER_REF)
        b = O.detect(im, [f], [ham], p, order=O.ORDER_CANON)
        assert sorted(a.dets) == sorted(b.dets)
        assert len(a.quads) == len(b.quads)
        ca = sorted(tuple(a.pts[a.cstart[i]:a.cstart[i + 1]]) for i in range(len(a.cid)))
        cb = sorted(tuple(b.pts[b.cstart[i]:b.cstart[i + 1]]) for i in range(len(b.cid)))
        assert ca == cb


# --- the angle sort: the GPU's characterisation against the recursion ---

def _leaf_of(n, p):
    lo, sz = 0, n
    while sz // 2 > 5:
        half = sz // 2
        q1, q3 = half // 2, half + (sz - half) // 2
        r = p - lo
        if r < q1:
            sz = q1
        elif r < half:
            lo, sz = lo + q1, half - q1
        elif r < q3:
            lo, sz = lo + half, q3 - half
        else:
            lo, sz = lo + q3, sz - q3
    while sz > 5:
        half = sz // 2
        if p - lo >= half:
            lo, sz = lo + half, sz - half
        else:
            sz = half
    return lo, sz


_NETS = {2: [(0, 1)], 3: [(0, 1), (1, 2), (0, 1)], 4: [(0, 1), (2, 3), (0, 2), (1, 3), (1, 2)],
         5: [(0, 1), (3, 4), (1, 2), (0, 1), (0, 3), (2, 4), (1, 2), (2, 3), (1, 2)]}


def _block_order(keys):
    """Leaf networks, then sort by (block head, place in leaf)."""
    n = len(keys)
    items = []
    p = 0
    while p < n:
        lo, ln = _leaf_of(n, p)
        k = [int(x) for x in keys[lo:lo + ln]]
        for a, b in _NETS.get(ln, []):
            if (k[a] >> 32) > (k[b] >> 32):
                k[a], k[b] = k[b], k[a]
        head = None
        for t, x in enumerate(k):
            head = x if head is None or x > head else head
            items.append((head, t, x))
        p = lo + ln
    return np.array([x for _, _, x in sorted(items)], np.uint64)


@pytest.mark.parametrize("seed", range(40))
def test_angle_sort_characterisation(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 700))
    slopes = rng.integers(0, max(2, n // 6), n).astype(np.uint64)  # many equal angles
    idx = np.arange(n, dtype=np.uint64)
    keys = (slopes << np.uint64(32)) | (~idx & np.uint64(0xffffffff))
    assert np.array_equal(O.keysort(keys), _block_order(keys))


# --- the oracle against the reference itself (compiled into oracle/_ref) ---

needs_ref = pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref not built")


def _synthetic(seed, w, h, ntags, noise, fams=("tag36h11",), distractors=20):
    from apriltags_fast_b200 import synth

    cfg = synth.Config(w, h, families=fams, ntags=(ntags, ntags), side=(24, min(w, h) // 3), tilt_deg=55.0,
                       noise=noise, blur=(0.5, 1.2), distractors=distractors)
    return synth.make_frame(cfg, seed)[0]


PARAMS = [
    dict(),
    dict(quad_decimate=1.0),
    dict(quad_decimate=1.5),
    dict(quad_decimate=3.0),
    dict(quad_sigma=0.8),
    dict(quad_sigma=-0.8, quad_decimate=1.0),
    dict(refine_edges=0),
    dict(deglitch=1, quad_decimate=1.0),
    dict(max_nmaxima=4),
    dict(min_white_black_diff=20, min_cluster_pixels=8),
]


@needs_ref
@pytest.mark.parametrize("seed", range(12))
def test_oracle_equals_reference(seed):
    prm = PARAMS[seed % len(PARAMS)]
    fams = ("tag36h11",) if seed % 3 else ("tagStandard41h12", "tag36h11")
    rng = np.random.default_rng(100 + seed)
    w, h = int(rng.integers(200, 700)), int(rng.integers(150, 500))
    img = _synthetic(seed, w, h, ntags=int(rng.integers(1, 6)), noise=float(rng.uniform(1, 6)), fams=fams)
    p = O.default_params(**prm)
    bits = [2] * len(fams)
    ref, nq = O.ref_detect(img, fams, bits, p)
    r = O.detect(img, [H.oracle_family(f) for f in fams], bits, p, order=O.ORDER_REF)
    assert len(r.quads) == nq
    assert r.dets == ref


def _config_frame(name, seed, replacement=True):
    from apriltags_fast_b200 import synth

    cfg = synth.Config(**{**synth.CONFIGS[name].__dict__, "replacement": replacement})
    return cfg, synth.make_frame(cfg, seed)[0]


@needs_ref
@pytest.mark.parametrize("seed", [0, 5, 1001])
def test_oracle_equals_reference_1080p(seed):
    """The 1920x1080 workload (24 tags, 200 distractors, codes drawn with
    replacement), decimate 2, bits 2: the oracle equals the reference in
    its own order, and the quad count too."""
    cfg, img = _config_frame("1080p", seed)
    fams = list(cfg.families)
    ref, nq = O.ref_detect(img, fams, [2] * len(fams))
    r = O.detect(img, [H.oracle_family(f) for f in fams], [2] * len(fams), O.default_params(), order=O.ORDER_REF)
    assert len(r.quads) == nq and r.dets == ref and len(ref) > 10


@needs_ref
@pytest.mark.parametrize("dec", [2.0, 1.0])
def test_oracle_equals_reference_4032x3024(dec):
    """The large-frame stress workload (two families, 80 tags, 1000
    distractors, an illumination ramp) at decimate 1 and 2."""
    cfg, img = _config_frame("4032x3024", 7)
    fams = list(cfg.families)
    p = O.default_params(quad_decimate=dec)
    ref, nq = O.ref_detect(img, fams, [2, 2], p)
    r = O.detect(img, [H.oracle_family(f) for f in fams], [2, 2], p, order=O.ORDER_REF)
    assert len(r.quads) == nq and r.dets == ref and len(ref) > 20
