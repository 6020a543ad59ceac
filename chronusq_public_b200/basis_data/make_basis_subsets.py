"""Extract the basis-set records this package ships from the reference's .gbs library.

The reference reads Gaussian-94 style ``.gbs`` files from its ``basis/`` directory
(parser: src/basisset/basisset_read.cpp:81-330).  This package ships trimmed copies
holding only the elements its workloads and tests use, in the same text format, so
that the package parser reads them exactly as the reference reads the originals.

Usage (run once, from the repository root, where the reference is mounted):

    python chronusq_public_b200/basis_data/make_basis_subsets.py <reference>/basis

The records are copied verbatim (exponents and coefficients are published basis-set
data: Pople 1969/1973, Dunning 1989).  Header comment lines are replaced by a one-line
provenance note.
"""
import os
import sys

BASES = ["sto3g.gbs", "6-31g.gbs", "6-31g*.gbs", "cc-pvdz.gbs", "cc-pvtz.gbs"]
ELEMENTS = {"H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne"}


def extract(src_path, dst_path):
    with open(src_path) as f:
        lines = f.read().splitlines()
    records, cur = [], []
    for line in lines:
        if not line.strip() or line.startswith("!"):
            continue
        if line.strip() == "****":
            if cur:
                records.append(cur)
            cur = []
            continue
        cur.append(line.rstrip())
    if cur:
        records.append(cur)
    keep = [r for r in records if r and r[0].split()[0] in ELEMENTS]
    with open(dst_path, "w") as f:
        f.write("! subset of %s (elements %s) extracted by make_basis_subsets.py\n"
                % (os.path.basename(src_path), " ".join(sorted(ELEMENTS))))
        f.write("****\n")
        for r in keep:
            f.write("\n".join(r) + "\n****\n")
    return len(keep)


def main(src_dir):
    here = os.path.dirname(os.path.abspath(__file__))
    for b in BASES:
        n = extract(os.path.join(src_dir, b), os.path.join(here, b))
        print(b, n, "elements")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/basis")
