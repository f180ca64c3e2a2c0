"""Generate the known-answer fixtures that pin the oracle (tests/golden/pins.json).

The reference has no unit test of its RI Fock build; its example logs are its regression
tests ("run, then compare with benchmark.log").  Their final RI-RHF energies pin the whole
chain integrals -> metric -> RI-JK -> SCF.  This script reads, from the reference tree:
  * the input geometry of each example (deck or test driver),
  * the final converged energy (last "ITER" line before "converged") of the log,
and writes them with their source file:line.  It also reads the normalised contraction
coefficients the reference prints for the carbon shells of C2H4 (column "c" of the basis
table), which pin the basis normalisation.

    python tests/golden/make_golden.py <path of the reference tree>
"""
import json
import os
import re
import sys


def last_energy(log_path):
    with open(log_path) as f:
        lines = f.read().splitlines()
    best = None
    for i, ln in enumerate(lines):
        m = re.match(r"ITER\s+\d+\s+E=\s*(\S+)", ln)
        if m:
            best = (float(m.group(1)), i + 1, m.group(1))
        if ("converged after" in ln) and best is not None:
            return best
    return best


def xyz_from_deck(text):
    lines = [l for l in text.splitlines()]
    for i, l in enumerate(lines):
        if l.strip().lower() == "_xyz":
            n = int(lines[i + 1].split()[0])
            atoms = lines[i + 3:i + 3 + n]
            return [a.split()[0] for a in atoms], [[float(v) for v in a.split()[1:4]] for a in atoms]
        if re.match(r"^\s*\d+\s*$", l) and i > 0 and "_xyz" in lines[i - 1].lower():
            pass
    raise ValueError("no _xyz block")


def main(ref):
    pins = []
    # C2H4 / cc-pVDZ / cc-pVDZ-RI
    deck = open(os.path.join(ref, "examples/c2h4_2_2/cas.inp")).read()
    sym, xyz = xyz_from_deck(deck)
    e, line, txt = last_energy(os.path.join(ref, "examples/c2h4_2_2/benchmark.log"))
    pins.append({"name": "c2h4", "symbols": sym, "coords_ang": xyz, "basis": "cc-pvdz", "aux": "cc-pvdz-ri",
                 "energy": e, "energy_text": txt, "source": "examples/c2h4_2_2/benchmark.log:%d" % line,
                 "geometry_source": "examples/c2h4_2_2/cas.inp"})
    # C6H8 / cc-pVDZ / cc-pVDZ-RI
    deck = open(os.path.join(ref, "examples/cis/c6h8_cis.inp")).read()
    sym, xyz = xyz_from_deck(deck)
    e, line, txt = last_energy(os.path.join(ref, "examples/cis/benchmark.log"))
    pins.append({"name": "c6h8", "symbols": sym, "coords_ang": xyz, "basis": "cc-pvdz", "aux": "cc-pvdz-ri",
                 "energy": e, "energy_text": txt, "source": "examples/cis/benchmark.log:%d" % line,
                 "geometry_source": "examples/cis/c6h8_cis.inp"})
    # guanine / cc-pVDZ / cc-pVDZ-RI (geometry from the spin-projection test driver)
    drv = open(os.path.join(ref, "tests/spin_proj/run_tests.py")).read()
    blk = drv.split("'guanine': \"\"\"")[1].split('"""')[0].splitlines()[2:]
    sym = [l.split()[0] for l in blk]
    xyz = [[float(v) for v in l.split()[1:4]] for l in blk]
    e, line, txt = last_energy(os.path.join(ref, "examples/spin_proj/guanine_sa4.log"))
    pins.append({"name": "guanine", "symbols": sym, "coords_ang": xyz, "basis": "cc-pvdz", "aux": "cc-pvdz-ri",
                 "energy": e, "energy_text": txt, "source": "examples/spin_proj/guanine_sa4.log:%d" % line,
                 "geometry_source": "tests/spin_proj/run_tests.py"})
    # normalised carbon contraction coefficients printed by the reference (C2H4 log)
    log = open(os.path.join(ref, "examples/c2h4_2_2/benchmark.log")).read().splitlines()
    coef = []
    start = None
    for i, ln in enumerate(log):
        if "C (  0)" in ln and start is None and "Basis set information" in "\n".join(log[max(0, i - 8):i]):
            start = i
            break
    for ln in log[start + 1:]:
        if "C (  1)" in ln:
            break
        cols = [c.strip() for c in ln.split("|")]
        if len(cols) >= 6 and re.match(r"^-?\d+\.\d+$", cols[3] or "x"):
            coef.append({"l": None if cols[2] == "" else int(cols[2]), "alpha": float(cols[3]),
                         "c": float(cols[4]), "c_lib": float(cols[5])})
    # propagate l down the block
    cur = None
    for c in coef:
        if c["l"] is not None:
            cur = c["l"]
        c["l"] = cur
    out = {"pins": pins, "carbon_ccpvdz_norm_coefs": coef,
           "carbon_coef_source": "examples/c2h4_2_2/benchmark.log:%d" % (start + 1)}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "pins.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(pins), "energy pins and", len(coef), "coefficients")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <path of the reference tree>")
    main(sys.argv[1])
