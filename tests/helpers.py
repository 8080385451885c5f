"""Shared helpers of the tests: fixtures, families and comparisons."""
import os
import shlex

import numpy as np

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
IMAGES = [f"test/images/synth_640x480_00{i}.pgm" for i in range(2)]


def read_pgm(path):
    data = open(path, "rb").read()
    toks, pos = [], 2
    while len(toks) < 3:
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            while data[pos:pos + 1] != b"\n":
                pos += 1
            continue
        s = pos
        while not data[pos:pos + 1].isspace():
            pos += 1
        toks.append(int(data[s:pos]))
    pos += 1
    w, h, _ = toks
    return np.frombuffer(data[pos:pos + w * h], np.uint8).reshape(h, w).copy()


def golden_images():
    return [read_pgm(os.path.join(GOLDEN, os.path.basename(p))) for p in IMAGES]


def golden_cases():
    """(name, family, hamming, params dict) of each case of cases.txt, read
    as the reference demo parses its flags (example/fast_demo.c:96-125)."""
    out = []
    for line in open(os.path.join(GOLDEN, "cases.txt")):
        line = line.strip()
        if not line:
            continue
        name, args = line.split("\t")
        a = shlex.split(args)
        fam, ham, prm = "tag36h11", 1, {}
        i = 0
        while i < len(a):
            if a[i] == "-x":
                i += 1
                prm["quad_decimate"] = float(a[i])
            elif a[i] == "-f":
                i += 1
                fam = a[i]
            elif a[i] == "-a":
                i += 1
                ham = int(a[i])
            elif a[i] == "-b":
                i += 1
                prm["quad_sigma"] = float(a[i])
            elif a[i] == "-0":
                prm["refine_edges"] = 0
            elif a[i] == "--deglitch":
                prm["deglitch"] = 1
            elif a[i] == "-t":
                i += 1
            i += 1
        out.append((name, fam, ham, prm))
    return out


def golden_hex(name):
    return open(os.path.join(GOLDEN, "hex", name + ".hex")).read().splitlines()


def oracle_family(name):
    """The family as an oracle struct, from the GPU library's tables (data
    only) or, failing that, from the reference built into oracle/_ref."""
    try:
        from apriltags_fast_b200 import family

        return O.Family.from_buffer_copy(bytes(family(name)))
    except Exception:
        R = O.ref_lib()
        if R is None:
            raise
        return O.Family.from_buffer_copy(bytes(R.at_family_by_name(name.encode()).contents))


def canonical(dets):
    """Detections sorted by (family, id, exact values): the order-free form."""
    return sorted(dets)
