"""Extract element subsets of Dalton basis-library files into this folder.

The GPU runs carry no copy of the Dalton source tree, so the few basis sets
the workloads and the parity tests use are kept here as subsets of the Dalton
basis library (``basis/<name>`` in the Dalton source tree), in the library's
own text format (``a <Z>`` blocks of ``nprim ncontr 0`` headers followed by
exponent/coefficient rows).  ``dalton_b200.basis`` parses that format.

Usage (run once, from a machine that has the Dalton sources)::

    python dalton_b200/basis_data/extract.py /path/to/dalton/basis
"""
import os
import re
import sys

SETS = ["cc-pVDZ", "cc-pVTZ", "6-31G*", "STO-3G", "aug-cc-pVDZ"]
ELEMENTS = {1, 6, 7, 8}


def subset(text, elements):
    out = []
    keep = False
    header = []
    for line in text.splitlines():
        m = re.match(r"^[aA]\s+(\d+)\s*$", line)
        if m:
            keep = int(m.group(1)) in elements
        if keep:
            out.append(line.rstrip())
        elif not out and line.startswith("$"):
            header.append(line.rstrip())
    return "\n".join(header[:1] + out) + "\n"


def main(src):
    here = os.path.dirname(os.path.abspath(__file__))
    for name in SETS:
        with open(os.path.join(src, name)) as f:
            text = f.read()
        dst = os.path.join(here, name.replace("*", "_star") + ".dalton")
        with open(dst, "w") as f:
            f.write(subset(text, ELEMENTS))
        print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract.py <path to the basis/ folder of a Dalton source tree>")
    main(sys.argv[1])
