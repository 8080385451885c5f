"""Copy the reference's own known-answer fixtures into tests/golden/.

The reference's golden test (test/run_golden.sh) runs 18 detector
configurations (test/cases.txt) on two synthetic 640x480 images
(test/images/*.pgm) and compares the hex dump of the detections byte for
byte with test/golden/*.hex. Those files are copied here unchanged so the
tests can run where the reference checkout is absent.

    python tests/golden/make_fixtures.py <reference dir>
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    os.makedirs(os.path.join(HERE, "hex"), exist_ok=True)
    for i in range(2):
        shutil.copy(os.path.join(ref, "test", "images", f"synth_640x480_00{i}.pgm"), HERE)
    shutil.copy(os.path.join(ref, "test", "cases.txt"), HERE)
    for f in sorted(os.listdir(os.path.join(ref, "test", "golden"))):
        shutil.copy(os.path.join(ref, "test", "golden", f), os.path.join(HERE, "hex", f))


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], "test", "golden")):
        sys.exit("usage: make_fixtures.py <reference checkout> (a directory with test/golden)")
    main(sys.argv[1])
