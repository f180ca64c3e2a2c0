"""Extract the basis-set blocks this package needs from the reference's basis library.

The reference ships Gaussian94/psi4-format basis files under ``NOPT_lib/`` and reads
them with ``basis_lib_read_gbs`` (src/basis_lib_read.cpp:57-240).  The package only
needs the correlation-consistent orbital sets and their RI/JK fitting sets for
H, C, N and O, so this script copies those element blocks verbatim (published basis
data, unchanged) into ``nopt_b200/basis/<name>.gbs``.

Run once, where the reference tree is mounted:

    python nopt_b200/basis/extract_basis.py /root/reference/NOPT_lib
"""
import os
import sys

NAMES = ["cc-pvdz", "cc-pvdz-ri", "cc-pvdz-jkfit", "cc-pvtz", "cc-pvtz-ri", "cc-pvtz-jkfit"]
ELEMENTS = ["H", "C", "N", "O"]


def extract(src_dir, name, out_dir):
    with open(os.path.join(src_dir, name + ".gbs")) as f:
        lines = f.read().splitlines()
    out = ["! element blocks H, C, N, O of NOPT_lib/%s.gbs (Basis Set Exchange data)" % name, "****"]
    i = 0
    while i < len(lines):
        if lines[i].startswith("****") and i + 1 < len(lines):
            tok = lines[i + 1].split()
            if tok and tok[0] in ELEMENTS:
                j = i + 1
                block = []
                while j < len(lines) and not lines[j].startswith("****"):
                    block.append(lines[j].rstrip())
                    j += 1
                out.extend(block)
                out.append("****")
                i = j
                continue
        i += 1
    with open(os.path.join(out_dir, name + ".gbs"), "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/NOPT_lib"
    here = os.path.dirname(os.path.abspath(__file__))
    for n in NAMES:
        extract(src, n, here)
        print("wrote", n)
