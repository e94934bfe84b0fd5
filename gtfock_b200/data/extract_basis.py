"""Extract the H, C, N, O blocks of the published basis sets the benchmarks use.

The .gbs files (EMSL Basis Set Exchange format) ship with the reference under
data/; the GPU machines do not have that tree, so the element blocks needed by
the synthetic molecules (alkanes, graphene flakes, water clusters) are copied
here verbatim, header line ("spherical"/"cartesian") included.

Run with the reference tree's data/ directory as the argument (default: the
data/ of $GTFOCK_REFERENCE, else of a checkout named `reference` beside this
repository):
    python gtfock_b200/data/extract_basis.py <reference>/data
"""
import os
import sys

ELEMENTS = ("H", "C", "N", "O")
FILES = ("sto-3g.gbs", "6-31g.gbs", "cc-pvdz.gbs")


def extract(src, dst):
    lines = open(src).read().splitlines()
    header = next(l.strip() for l in lines if l.strip())
    out = [header, ""]
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        if len(tok) == 2 and tok[0] in ELEMENTS and tok[1] == "0":
            j = i
            while lines[j].strip() != "****":
                out.append(lines[j].rstrip())
                j += 1
            out.append("****")
            i = j + 1
            continue
        i += 1
    with open(dst, "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(os.path.dirname(here))
    default = os.environ.get("GTFOCK_REFERENCE") or os.path.join(os.path.dirname(repo), "reference")
    ref = sys.argv[1] if len(sys.argv) > 1 else os.path.join(default, "data")
    for name in FILES:
        extract(os.path.join(ref, name), os.path.join(here, name))
        print("wrote", name)
