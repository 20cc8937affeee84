#!/usr/bin/env python3
"""Copy the reference's four sample decks into tests/golden/samples/.

Each deck is the reference's own end-to-end test case (bin/rt_autotest runs them and diffs
output/diagnostics.txt against reference.out): input.in, resolution.in, reference.out and,
for the Athena decks, the binary snapshot files under input_athena/.  These are fixtures
(data), copied byte for byte; the GPU box has no copy of the reference, so the tests read
them from here.

    python tests/golden/make_fixtures.py <reference_root>

reference_root is the top directory of a checkout of the reference (the one holding samples/).
"""
import os
import shutil
import sys

DECKS = ["GreyIsothermal", "NongreyAGN", "ReadFromAthena", "multiInTest"]
KEEP = {"input.in", "resolution.in", "reference.out"}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <reference_root>")
    ref = sys.argv[1]
    dst_root = os.path.join(os.path.dirname(os.path.abspath(__file__)), "samples")
    for deck in DECKS:
        src = os.path.join(ref, "samples", deck)
        dst = os.path.join(dst_root, deck)
        os.makedirs(dst, exist_ok=True)
        for name in KEEP:
            shutil.copyfile(os.path.join(src, name), os.path.join(dst, name))
        ath = os.path.join(src, "input_athena")
        if os.path.isdir(ath):
            for dirpath, _, files in os.walk(ath):
                rel = os.path.relpath(dirpath, src)
                os.makedirs(os.path.join(dst, rel), exist_ok=True)
                for f in files:
                    if f.endswith(".bin"):
                        shutil.copyfile(os.path.join(dirpath, f), os.path.join(dst, rel, f))
    print("copied", len(DECKS), "decks to", dst_root)


if __name__ == "__main__":
    main()
