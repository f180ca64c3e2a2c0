"""Basis-set reader for Gaussian94/psi4 ``.gbs`` files.

Mirrors the reference's ``basis_lib_read_gbs`` (src/basis_lib_read.cpp:57-240): element
blocks are delimited by ``****``; each shell line is ``<L> <nprim> <scale>`` followed by
``nprim`` lines of ``exponent coefficient`` (Fortran ``D`` exponents accepted, as with the
reference's ``D_change``).  ``SP`` shells are rejected, as the reference does
(src/basis_lib_read.cpp:213-216).  The orbital basis of the reference is Cartesian with an
optional spherical (D5) projection; the auxiliary basis is spherical
(src/inp_par_read.cpp:2550-2585).  Energies are identical between a spherical orbital basis
and the reference's Cartesian+D5 treatment, so this package works with spherical shells.
"""
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_L = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5}


class Shell:
    __slots__ = ("l", "exps", "coefs", "center", "atom")

    def __init__(self, l, exps, coefs, center, atom):
        self.l, self.exps, self.coefs, self.center, self.atom = l, list(exps), list(coefs), tuple(center), atom

    def nfunc(self, pure=True):
        return 2 * self.l + 1 if pure else (self.l + 1) * (self.l + 2) // 2


def _to_float(tok):
    return float(tok.replace("D", "E").replace("d", "e"))


def read_gbs(name):
    """Return {element: [(l, [exps], [coefs]), ...]} for a library name or a path."""
    path = name if os.path.sep in name or name.endswith(".gbs") else os.path.join(_HERE, name.lower() + ".gbs")
    if not os.path.exists(path):
        raise FileNotFoundError("basis file not found: %s" % path)
    with open(path) as f:
        lines = [ln.rstrip() for ln in f]
    out = {}
    i = 0
    while i < len(lines):
        if lines[i].startswith("****") and i + 1 < len(lines):
            tok = lines[i + 1].split()
            if not tok or tok[0] in ("****",):
                i += 1
                continue
            el = tok[0]
            shells = []
            j = i + 2
            while j < len(lines) and not lines[j].startswith("****"):
                t = lines[j].split()
                if not t or t[0].startswith("!"):
                    j += 1
                    continue
                lab = t[0].upper()
                if lab not in _L:
                    raise ValueError("%s: unsupported shell label %r (line %d)" % (path, t[0], j + 1))
                npr = int(t[1])
                if npr < 1:
                    raise ValueError("%s: bad primitive count on line %d" % (path, j + 1))
                exps, coefs = [], []
                for k in range(npr):
                    v = lines[j + 1 + k].split()
                    exps.append(_to_float(v[0]))
                    coefs.append(_to_float(v[1]))
                shells.append((_L[lab], exps, coefs))
                j += 1 + npr
            out[el] = shells
            i = j
            continue
        i += 1
    return out


def build_shells(basis_name, symbols, coords_bohr):
    """Shells for a molecule, atom by atom in input order (as the reference appends them)."""
    lib = read_gbs(basis_name)
    shells = []
    for a, (sym, xyz) in enumerate(zip(symbols, coords_bohr)):
        key = sym.capitalize()
        if key not in lib:
            raise KeyError("element %s not in basis %s" % (sym, basis_name))
        for l, exps, coefs in lib[key]:
            shells.append(Shell(l, exps, coefs, xyz, a))
    return shells
