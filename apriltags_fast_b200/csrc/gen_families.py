"""The built-in tag families as data: families.bin, and the C source the
library build makes from it.

The code tables of the AprilTag families are published data (they define
the tags, so they must be the same codes, bit positions and geometry as
the reference's tag*.c files). families.bin holds them compactly and is
committed beside this script, so building the library needs no reference
checkout:

    python gen_families.py extract <reference dir>   # tag*.c -> families.bin
    python gen_families.py csource <out.c>           # families.bin -> C (build step)

families.bin: a little-endian u32 count of families, then per family a
64-byte header (the name in 32 NUL-padded bytes; i32 ncodes, nbits, h,
width_at_border, total_width, reversed_border; 8 bytes of zeros), nbits
signed bytes of bit_x, nbits of bit_y, and ncodes codes of ceil(nbits / 8)
little-endian bytes each.
"""
import os
import re
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "families.bin")
FAMILIES = ["tag16h5", "tag25h9", "tag36h10", "tag36h11", "tagCircle21h7", "tagCircle49h12",
            "tagCustom48h12", "tagStandard41h12", "tagStandard52h13"]
HEADER = struct.Struct("<32s6i8x")  # name, ncodes, nbits, h, width_at_border, total_width, reversed


def parse_c(path):
    """One family from an AprilTag tag*.c file."""
    src = open(path).read()
    m = re.search(r"codedata\[(\d+)\]\s*=\s*\{(.*?)\};", src, re.S)
    codes = [int(c, 16) for c in re.findall(r"0x([0-9a-fA-F]+)UL", m.group(2))]
    assert len(codes) == int(m.group(1)), path

    def field(name):
        return re.search(r"tf->" + name + r"\s*=\s*([^;]+);", src).group(1).strip()

    nbits = int(field("nbits"))
    bx = {int(k): int(v) for k, v in re.findall(r"tf->bit_x\[(\d+)\]\s*=\s*(-?\d+);", src)}
    by = {int(k): int(v) for k, v in re.findall(r"tf->bit_y\[(\d+)\]\s*=\s*(-?\d+);", src)}
    assert len(bx) == nbits and len(by) == nbits, path
    f = dict(name=re.search(r'strdup\("([^"]+)"\)', field("name")).group(1), codes=codes, nbits=nbits,
             h=int(field("h")), wab=int(field("width_at_border")), tw=int(field("total_width")),
             rev=field("reversed_border") == "true", bit_x=[bx[i] for i in range(nbits)],
             bit_y=[by[i] for i in range(nbits)])
    assert int(field("ncodes")) == len(codes), path
    return f


def pack(fams):
    out = [struct.pack("<I", len(fams))]
    for f in fams:
        out.append(HEADER.pack(f["name"].encode(), len(f["codes"]), f["nbits"], f["h"], f["wab"], f["tw"],
                               int(f["rev"])))
        out.append(struct.pack(f"<{f['nbits']}b", *f["bit_x"]))
        out.append(struct.pack(f"<{f['nbits']}b", *f["bit_y"]))
        nb = (f["nbits"] + 7) // 8
        out.append(b"".join(c.to_bytes(nb, "little") for c in f["codes"]))
    return b"".join(out)


def unpack(blob):
    (n,), at, fams = struct.unpack_from("<I", blob), 4, []
    for _ in range(n):
        name, ncodes, nbits, h, wab, tw, rev = HEADER.unpack_from(blob, at)
        at += HEADER.size
        bit_x = list(struct.unpack_from(f"<{nbits}b", blob, at))
        bit_y = list(struct.unpack_from(f"<{nbits}b", blob, at + nbits))
        at += 2 * nbits
        nb = (nbits + 7) // 8
        codes = [int.from_bytes(blob[at + i * nb:at + (i + 1) * nb], "little") for i in range(ncodes)]
        at += ncodes * nb
        fams.append(dict(name=name.rstrip(b"\0").decode(), codes=codes, nbits=nbits, h=h, wab=wab, tw=tw,
                         rev=bool(rev), bit_x=bit_x, bit_y=bit_y))
    assert at == len(blob), "trailing bytes in families.bin"
    return fams


def csource(fams):
    lines = ["/* generated from families.bin by gen_families.py; do not edit */", "#include \"apriltag_fast.h\"", ""]
    for f in fams:
        n = f["name"]
        lines.append(f"static const uint64_t codes_{n}[{len(f['codes'])}] = {{")
        for i in range(0, len(f["codes"]), 6):
            lines.append("  " + ", ".join(f"0x{c:016x}ull" for c in f["codes"][i:i + 6]) + ",")
        lines.append("};")
        lines.append(f"static const at_family fam_{n} = {{\"{n}\", codes_{n}, {len(f['codes'])}, {f['nbits']}, "
                     f"{f['h']}, {f['wab']}, {f['tw']}, {'true' if f['rev'] else 'false'}, "
                     f"{{{', '.join(map(str, f['bit_x']))}}}, {{{', '.join(map(str, f['bit_y']))}}}}};")
    lines.append("const at_family *const at_builtin_families[] = {" +
                 ", ".join(f"&fam_{f['name']}" for f in fams) + ", 0};")
    return "\n".join(lines) + "\n"


def main(argv):
    if len(argv) == 3 and argv[1] == "extract":
        fams = [parse_c(os.path.join(argv[2], n + ".c")) for n in FAMILIES]
        open(DATA, "wb").write(pack(fams))
        assert unpack(open(DATA, "rb").read()) == fams
    elif len(argv) == 3 and argv[1] == "csource":
        os.makedirs(os.path.dirname(os.path.abspath(argv[2])), exist_ok=True)
        open(argv[2], "w").write(csource(unpack(open(DATA, "rb").read())))
    else:
        sys.exit(__doc__)


if __name__ == "__main__":
    main(sys.argv)
