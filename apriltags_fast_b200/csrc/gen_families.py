"""Build step: extract the tag family tables into a C source file.

The code tables of the AprilTag families are data published with the
AprilTag library; the reference ships them as tag*.c files. This script
reads those files (from the reference checkout given on the command line)
and writes one C source with each family as an ``at_family`` initialiser.
The output goes to the build folder only (it is not committed); a library
built without it has no built-in families (at_tag36h11() returns NULL).

    python gen_families.py <reference dir> <out.c>
"""
import os
import re
import sys

FAMILIES = ["tag16h5", "tag25h9", "tag36h10", "tag36h11", "tagCircle21h7", "tagCircle49h12",
            "tagCustom48h12", "tagStandard41h12", "tagStandard52h13"]


def parse(path):
    src = open(path).read()
    m = re.search(r"codedata\[(\d+)\]\s*=\s*\{(.*?)\};", src, re.S)
    codes = re.findall(r"0x([0-9a-fA-F]+)UL", m.group(2))
    assert len(codes) == int(m.group(1)), path

    def field(name):
        return re.search(r"tf->" + name + r"\s*=\s*([^;]+);", src).group(1).strip()

    nbits = int(field("nbits"))
    bx = {int(k): int(v) for k, v in re.findall(r"tf->bit_x\[(\d+)\]\s*=\s*(-?\d+);", src)}
    by = {int(k): int(v) for k, v in re.findall(r"tf->bit_y\[(\d+)\]\s*=\s*(-?\d+);", src)}
    assert len(bx) == nbits and len(by) == nbits, path
    return dict(
        name=re.search(r'strdup\("([^"]+)"\)', field("name")).group(1),
        codes=codes, nbits=nbits, h=int(field("h")), ncodes=int(field("ncodes")),
        wab=int(field("width_at_border")), tw=int(field("total_width")),
        rev=field("reversed_border") == "true",
        bit_x=[bx[i] for i in range(nbits)], bit_y=[by[i] for i in range(nbits)])


def main(refdir, out):
    lines = ["/* generated by gen_families.py from the AprilTag family tables; do not edit */",
             "#include \"apriltag_fast.h\"", ""]
    names = []
    for fam in FAMILIES:
        f = parse(os.path.join(refdir, fam + ".c"))
        assert f["ncodes"] == len(f["codes"])
        lines.append(f"static const uint64_t codes_{fam}[{len(f['codes'])}] = {{")
        for i in range(0, len(f["codes"]), 6):
            lines.append("  " + ", ".join(f"0x{c}ull" for c in f["codes"][i:i + 6]) + ",")
        lines.append("};")
        bx = ", ".join(map(str, f["bit_x"]))
        by = ", ".join(map(str, f["bit_y"]))
        lines.append(f"static const at_family fam_{fam} = {{\"{f['name']}\", codes_{fam}, {f['ncodes']}, "
                     f"{f['nbits']}, {f['h']}, {f['wab']}, {f['tw']}, {'true' if f['rev'] else 'false'}, "
                     f"{{{bx}}}, {{{by}}}}};")
        names.append(fam)
    lines.append("const at_family *const at_builtin_families[] = {" + ", ".join(f"&fam_{n}" for n in names) +
                 ", 0};")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    open(out, "w").write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
