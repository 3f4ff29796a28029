"""Extract the basis-set tables the workloads need into ``basis_sets.json``.

The reference reads Gaussian-style basis files from its ``basisset/`` directory
at run time (src/pread.f90:611-1030).  The machine that runs the CUDA library
does not carry the reference tree, so the published exponents/coefficients of
the basis sets used by the workloads (STO-3G, 6-31G, 6-31G*, 6-31G**, cc-pVDZ)
for the first-row elements are kept in the package as JSON data.  This script
regenerates that file from a directory of basis files in the reference's text
format; it is a one-off data import, not part of the runtime.

Usage: python make_basis_json.py <basisset-dir> [out.json]
"""
import json
import os
import sys

BASES = ["STO-3G", "6-31G", "6-31Gs", "6-31Gss", "cc-pVDZ"]
ELEMENTS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne"]


def parse_file(path):
    """Parse one basis file: '****' separated element blocks of shells."""
    out = {}
    with open(path) as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    i = 0
    after_stars = False
    while i < len(lines):
        ln = lines[i]
        tag = ln[:2]
        if tag == "**":
            after_stars = True
            i += 1
            continue
        sym = ln.split()[0] if ln.split() else ""
        if after_stars and sym in ELEMENTS:
            shells = []
            i += 1
            while i < len(lines) and not lines[i].startswith("**"):
                parts = lines[i].split()
                typ, nprim, scale = parts[0], int(parts[1]), float(parts[2].replace("D", "E"))
                prims = []
                for k in range(nprim):
                    vals = [float(x.replace("D", "E")) for x in lines[i + 1 + k].split()]
                    prims.append(vals)
                shells.append([typ, scale, prims])
                i += 1 + nprim
            out[sym] = shells
            after_stars = False
            continue
        after_stars = False
        i += 1
    return out


def main():
    src = sys.argv[1]
    dst = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(__file__), "basis_sets.json")
    data = {name: parse_file(os.path.join(src, name)) for name in BASES}
    with open(dst, "w") as fh:
        json.dump(data, fh, indent=0, sort_keys=True)
    print("wrote", dst, {k: sorted(v) for k, v in data.items()})


if __name__ == "__main__":
    main()
