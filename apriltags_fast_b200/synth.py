"""Seeded synthetic AprilTag frames with the shapes of the benchmark configs.

There is no public dataset for the benchmark; these frames stand in for it:
a linear-gradient background with Gaussian noise, tags rendered from the
family code tables (a 1-module white border, as apriltag_to_image draws
them), placed by random homographies without overlap, optional filled
rectangle/ellipse distractors and an illumination ramp, a Gaussian blur,
rounded and clamped to u8. Tag codes are drawn uniformly from the
family's code table, with replacement, so ids may repeat in a frame
(Config.replacement=False draws distinct ids).

    img, truth = make_frame(CONFIGS["1080p"], seed=2)

The family tables come from the GPU library by default; `tables_from`
builds them from any at_family source (e.g. the reference's own library),
so that a frame can be made without loading the GPU library.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Config:
    width: int
    height: int
    families: tuple = ("tag36h11",)
    ntags: tuple = (4, 4)            # inclusive range
    side: tuple = (60, 140)          # tag side in pixels
    tilt_deg: float = 40.0
    noise: float = 3.0
    blur: tuple = (0.7, 0.7)         # per-tag blur sigma range (one value: global)
    distractors: int = 0
    ramp: tuple | None = None        # illumination ramp (lo, hi)
    gradient: tuple = (60.0, 190.0)
    replacement: bool = True         # draw tag codes with replacement (ids may repeat)


CONFIGS = {
    # 640x480, 4 tags of 60-140 px, tilt <= 40 deg, noise 3, blur 0.7
    "640x480": Config(640, 480),
    # 1920x1080, 24 tags of 30-220 px, tilt <= 60, noise 4, blur 0.8, 200 distractors
    "1080p": Config(1920, 1080, ntags=(24, 24), side=(30, 220), tilt_deg=60.0, noise=4.0, blur=(0.8, 0.8),
                    distractors=200),
    # 4032x3024, two families, 80 tags of 16-400 px, tilt <= 65, noise 6,
    # per-tag blur 0.5-1.5, ramp 0.4-1.0, 1000 distractors
    "4032x3024": Config(4032, 3024, families=("tagStandard52h13", "tag36h11"), ntags=(80, 80), side=(16, 400),
                        tilt_deg=65.0, noise=6.0, blur=(0.5, 1.5), distractors=1000, ramp=(0.4, 1.0)),
    # served request loop: 0-30 tag36h11 tags, otherwise as 640x480
    "serve_720p": Config(1280, 720, ntags=(0, 30)),
    "serve_1080p": Config(1920, 1080, ntags=(0, 30)),
    "serve_2160p": Config(3840, 2160, ntags=(0, 30)),
    # batched uneven frames: 0-40 tags of one family (tag36h11 or tag25h9)
    "mixed_640x480_36h11": Config(640, 480, ntags=(0, 40)),
    "mixed_640x480_25h9": Config(640, 480, families=("tag25h9",), ntags=(0, 40)),
    "mixed_1280x720_36h11": Config(1280, 720, ntags=(0, 40)),
    "mixed_1280x720_25h9": Config(1280, 720, families=("tag25h9",), ntags=(0, 40)),
    "mixed_1920x1080_36h11": Config(1920, 1080, ntags=(0, 40)),
    "mixed_1920x1080_25h9": Config(1920, 1080, families=("tag25h9",), ntags=(0, 40)),
    "mixed_3840x2160_36h11": Config(3840, 2160, ntags=(0, 40)),
    "mixed_3840x2160_25h9": Config(3840, 2160, families=("tag25h9",), ntags=(0, 40)),
}


def serve_mix(n: int, seed: int):
    """n frames of the served mix: 60% 1280x720, 30% 1920x1080, 10%
    3840x2160 (drawn per frame), each with 0-30 tag36h11 tags."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        u = rng.uniform()
        name = "serve_720p" if u < 0.6 else "serve_1080p" if u < 0.9 else "serve_2160p"
        out.append(make_frame(CONFIGS[name], seed * 100003 + i)[0])
    return out


def uneven_batch(n: int, seed: int):
    """n frames of sizes drawn uniformly from 640x480, 1280x720, 1920x1080 and
    3840x2160, each with 0-40 tags of tag36h11 or of tag25h9; returns
    (frames, family names)."""
    rng = np.random.default_rng(seed)
    frames, fams = [], []
    for i in range(n):
        size = ("640x480", "1280x720", "1920x1080", "3840x2160")[int(rng.integers(4))]
        fam = ("36h11", "25h9")[int(rng.integers(2))]
        frames.append(make_frame(CONFIGS[f"mixed_{size}_{fam}"], seed * 100003 + i)[0])
        fams.append("tag" + fam)
    return frames, fams


def tag_pattern(code: int, nbits: int, bit_x, bit_y, wab: int, tw: int, reversed_border: bool) -> np.ndarray:
    """The tag's module grid (tw x tw, 0 black / 255 white), drawn the way
    the upstream library's apriltag_to_image draws it (apriltag.c:271-297)."""
    im = np.zeros((tw, tw), np.uint8)
    wbw = wab + (0 if reversed_border else 2)
    wbs = (tw - wbw) // 2
    for i in range(wbw - 1):
        im[wbs, wbs + i] = 255
        im[wbs + i, tw - 1 - wbs] = 255
        im[tw - 1 - wbs, wbs + i + 1] = 255
        im[wbs + 1 + i, wbs] = 255
    bs = (tw - wab) // 2
    for i in range(nbits):
        if code >> (nbits - i - 1) & 1:
            im[bit_y[i] + bs, bit_x[i] + bs] = 255
    return im


def _homography(src, dst):
    A = []
    for (x, y), (u, v) in zip(src, dst):
        A.append([x, y, 1, 0, 0, 0, -u * x, -u * y, -u])
        A.append([0, 0, 0, x, y, 1, -v * x, -v * y, -v])
    _, _, vt = np.linalg.svd(np.asarray(A, float))
    H = vt[-1].reshape(3, 3)
    return H / H[2, 2]


def _tag_corners(rng, cx, cy, side, tilt_deg):
    """Corners of a square of `side` px centred at (cx, cy), rotated
    uniformly and tilted out of plane by up to tilt_deg (pinhole view)."""
    rot = rng.uniform(0, 2 * math.pi)
    tilt = math.radians(rng.uniform(0, tilt_deg))
    axis = rng.uniform(0, math.pi)
    h = side / 2.0
    sq = np.array([[-h, -h, 0], [h, -h, 0], [h, h, 0], [-h, h, 0]], float)
    c, s = math.cos(rot), math.sin(rot)
    Rz = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
    ax = np.array([math.cos(axis), math.sin(axis), 0.0])
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    Rt = np.eye(3) + math.sin(tilt) * K + (1 - math.cos(tilt)) * K @ K
    p = sq @ Rz.T @ Rt.T
    f = 4.0 * side
    z = f + p[:, 2]
    return np.stack([cx + f * p[:, 0] / z, cy + f * p[:, 1] / z], 1)


def _blur(img, sigma):
    if sigma <= 0:
        return img
    r = max(1, int(math.ceil(3 * sigma)))
    x = np.arange(-r, r + 1)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    pad = np.pad(img, ((0, 0), (r, r)), mode="edge")
    out = sum(k[i] * pad[:, i:i + img.shape[1]] for i in range(2 * r + 1))
    pad = np.pad(out, ((r, r), (0, 0)), mode="edge")
    return sum(k[i] * pad[i:i + img.shape[0], :] for i in range(2 * r + 1))


@dataclass
class TagTruth:
    family: str
    id: int
    corners: np.ndarray
    side: float


def make_frame(cfg: Config, seed: int, family_tables=None):
    """One frame (u8, h x w) and the list of TagTruth of the tags drawn.

    family_tables: name -> (codes, nbits, bit_x, bit_y, wab, tw, reversed);
    defaults to the built-in families of the library."""
    if family_tables is None:
        family_tables = {n: builtin_table(n) for n in cfg.families}
    rng = np.random.default_rng(seed)
    W, H = cfg.width, cfg.height
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float32)
    ang = rng.uniform(0, 2 * math.pi)
    t = (xx * math.cos(ang) + yy * math.sin(ang))
    t = (t - t.min()) / max(1e-6, float(t.max() - t.min()))
    img = (cfg.gradient[0] + (cfg.gradient[1] - cfg.gradient[0]) * t).astype(np.float32)

    # distractors: filled rectangles and ellipses, intensity U(0, 255)
    for _ in range(cfg.distractors):
        sz = rng.uniform(10, 150, size=2)
        x0, y0 = rng.uniform(0, W), rng.uniform(0, H)
        val = rng.uniform(0, 255)
        x1, x2 = int(max(0, x0 - sz[0] / 2)), int(min(W, x0 + sz[0] / 2))
        y1, y2 = int(max(0, y0 - sz[1] / 2)), int(min(H, y0 + sz[1] / 2))
        if x2 <= x1 or y2 <= y1:
            continue
        if rng.uniform() < 0.5:
            img[y1:y2, x1:x2] = val
        else:
            sy, sx = np.mgrid[y1:y2, x1:x2]
            m = ((sx - x0) / (sz[0] / 2)) ** 2 + ((sy - y0) / (sz[1] / 2)) ** 2 <= 1.0
            img[y1:y2, x1:x2][m] = val

    ntags = int(rng.integers(cfg.ntags[0], cfg.ntags[1] + 1))
    placed, truths = [], []
    used = {n: set() for n in cfg.families}
    tries = 0
    while len(truths) < ntags and tries < 200 * max(1, ntags):
        tries += 1
        side = rng.uniform(*cfg.side)
        r = side * 0.75 + 4
        cx, cy = rng.uniform(r, W - r), rng.uniform(r, H - r)
        if any((cx - px) ** 2 + (cy - py) ** 2 < (r + pr) ** 2 for px, py, pr in placed):
            continue
        fname = cfg.families[int(rng.integers(len(cfg.families)))]
        codes, nbits, bx, by, wab, tw, rev = family_tables[fname]
        if cfg.replacement:
            tid = int(rng.integers(len(codes)))
        else:
            if len(used[fname]) >= len(codes):
                continue
            while True:
                tid = int(rng.integers(len(codes)))
                if tid not in used[fname]:
                    break
            used[fname].add(tid)
        pat = tag_pattern(int(codes[tid]), nbits, bx, by, wab, tw, rev)
        corners = _tag_corners(rng, cx, cy, side, cfg.tilt_deg)
        # the tag's outer edge maps to the corners: module grid [0, tw]
        Hm = _homography([(0, 0), (tw, 0), (tw, tw), (0, tw)], corners)
        Hi = np.linalg.inv(Hm)
        x1, y1 = np.floor(corners.min(0)).astype(int)
        x2, y2 = np.ceil(corners.max(0)).astype(int) + 1
        x1, y1, x2, y2 = max(x1, 0), max(y1, 0), min(x2, W), min(y2, H)
        sy, sx = np.mgrid[y1:y2, x1:x2].astype(np.float64)
        q = Hi @ np.stack([sx.ravel() + 0.5, sy.ravel() + 0.5, np.ones(sx.size)])
        u, v = q[0] / q[2], q[1] / q[2]
        inside = (u >= 0) & (u < tw) & (v >= 0) & (v < tw)
        vals = pat[np.clip(v.astype(int), 0, tw - 1), np.clip(u.astype(int), 0, tw - 1)].astype(np.float32)
        sub = img[y1:y2, x1:x2].ravel()
        sub[inside] = vals[inside]
        img[y1:y2, x1:x2] = sub.reshape(y2 - y1, x2 - x1)
        placed.append((cx, cy, r))
        truths.append(TagTruth(fname, tid, corners, side))

    if cfg.ramp is not None:
        ra = rng.uniform(0, 2 * math.pi)
        t2 = (xx * math.cos(ra) + yy * math.sin(ra))
        t2 = (t2 - t2.min()) / max(1e-6, float(t2.max() - t2.min()))
        img = img * (cfg.ramp[0] + (cfg.ramp[1] - cfg.ramp[0]) * t2)
    sig = float(rng.uniform(*cfg.blur))
    img = _blur(img, sig)
    img = img + rng.normal(0.0, cfg.noise, size=img.shape)
    return np.clip(np.rint(img), 0, 255).astype(np.uint8), truths


def table_of(f):
    """(codes, nbits, bit_x, bit_y, wab, tw, reversed) of an at_family
    struct (any ctypes struct with the at_family fields)."""
    codes = np.ctypeslib.as_array(f.codes, shape=(f.ncodes,)).copy()
    return (codes, f.nbits, list(f.bit_x[:f.nbits]), list(f.bit_y[:f.nbits]), f.width_at_border, f.total_width,
            bool(f.reversed_border))


def builtin_table(name: str):
    """The table of a built-in family of the GPU library."""
    from . import family

    return table_of(family(name))


def tables_from(lookup, names):
    """name -> table for `names`, with lookup(name) giving an at_family
    struct (for example the reference library's at_family_by_name)."""
    return {n: table_of(lookup(n)) for n in names}


# --------------------------------------------------------------------------
# JPEG versions of frames (csrc/synth_jpeg.c, built beside the package)

JPEG_OPTIMIZE, JPEG_NO_DHT, JPEG_MARKERS, JPEG_ONE_DQT = 1, 2, 4, 8
_sj = None


def encode_jpeg(img, quality: int = 90, sampling=(1, 1), restart: int = 0, flags: int = 0) -> bytes:
    """Baseline JPEG of a gray (h, w) or RGB (h, w, 3) u8 image: luma
    sampling (h, v) in {1, 2}, chroma 1x1; quality 1-100 on the IJG scale
    of the Annex K tables; a restart marker every `restart` MCUs; flags:
    JPEG_OPTIMIZE (per-image optimal Huffman tables), JPEG_NO_DHT (no
    Huffman tables in the file), JPEG_MARKERS (APP0, APP13, COM),
    JPEG_ONE_DQT (one DQT segment)."""
    import ctypes as C
    import os

    global _sj
    if _sj is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsynthjpeg.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m apriltags_fast_b200.build`")
        L = C.CDLL(path)
        L.sj_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.sj_encode.restype = C.c_int64
        _sj = L
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape[:2]
    nc = 1 if img.ndim == 2 else 3
    cap = 4 * w * h * nc + 65536
    out = np.empty(cap, np.uint8)
    n = _sj.sj_encode(img.ctypes.data, w, h, img.strides[0], nc, sampling[0], sampling[1], quality, restart, flags,
                      out.ctypes.data, cap)
    if n < 0:
        raise ValueError("encode_jpeg: arguments out of range")
    return out[:n].tobytes()
