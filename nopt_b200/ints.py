"""ctypes front end of the host integral engine (libgto_ints.so, include/gto_ints.h).

These are the inputs of the RI-JK Fock build that the reference gets from libint2:
S, T, V (src/molecule.cpp:3757-3800), the metric (P|Q) (RI_V_calc,
src/libint_link.cpp:2049-2107) and the three-centre (mu nu|P) (calc_2el_AO_INTS_RI,
src/libint_link.cpp:2261-2350).
"""
import ctypes
import os

import numpy as np

from . import basis as _basis
from .molecules import Molecule

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

LAYOUT_NOPT_FULL = 0
LAYOUT_PACKED = 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libgto_ints.so")
        if not os.path.exists(path):
            raise RuntimeError("libgto_ints.so is not built; run python nopt_b200/build.py")
        L = ctypes.CDLL(path)
        L.gto_basis_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp]
        L.gto_basis_destroy.argtypes = [ctypes.c_void_p]
        L.gto_basis_destroy.restype = None
        L.gto_basis_nbf.argtypes = [ctypes.c_void_p]
        L.gto_basis_max_l.argtypes = [ctypes.c_void_p]
        L.gto_basis_norm_coefs.argtypes = [ctypes.c_void_p, _dp]
        L.gto_basis_shell_offsets.argtypes = [ctypes.c_void_p, _ip]
        L.gto_overlap.argtypes = [ctypes.c_void_p, _dp]
        L.gto_kinetic.argtypes = [ctypes.c_void_p, _dp]
        L.gto_nuclear.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]
        L.gto_coulomb_2c.argtypes = [ctypes.c_void_p, _dp]
        L.gto_coulomb_3c.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _dp]
        L.gto_boys.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        L.gto_atomic_density.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, _dp, _dp, _dp, _ip]
        L.gto_cart_to_sph.argtypes = [ctypes.c_int, _dp]
        L.gto_set_threads.argtypes = [ctypes.c_int]
        L.gto_set_threads.restype = None
        _LIB = L
    return _LIB


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed with code %d" % (what, rc))


class Basis:
    """A basis over a molecule's atoms (spherical shells unless pure=False)."""

    def __init__(self, shells, pure=True):
        self.shells = shells
        l = np.array([s.l for s in shells], dtype=np.int32)
        pu = np.full(len(shells), 1 if pure else 0, dtype=np.int32)
        npr = np.array([len(s.exps) for s in shells], dtype=np.int32)
        xyz = np.array([s.center for s in shells], dtype=np.float64).reshape(-1)
        ex = np.array([e for s in shells for e in s.exps], dtype=np.float64)
        co = np.array([c for s in shells for c in s.coefs], dtype=np.float64)
        h = ctypes.c_void_p()
        _check(lib().gto_basis_create(ctypes.byref(h), len(shells), _ptr(l, _ip), _ptr(pu, _ip), _ptr(npr, _ip),
                                      _ptr(xyz), _ptr(ex), _ptr(co)), "gto_basis_create")
        self._h = h
        self.nbf = lib().gto_basis_nbf(h)
        self.pure = pure
        # shell arrays as handed to the library (also the rijk_basis_t of the GPU integrals)
        self.arrays = (l, pu, npr, xyz, ex, co)

    @classmethod
    def for_molecule(cls, name, mol, pure=True):
        return cls(_basis.build_shells(name, mol.symbols, mol.coords_bohr), pure=pure)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _LIB is not None:
            _LIB.gto_basis_destroy(h)
            self._h = None

    def norm_coefs(self):
        out = np.empty(sum(len(s.exps) for s in self.shells))
        _check(lib().gto_basis_norm_coefs(self._h, _ptr(out)), "gto_basis_norm_coefs")
        return out

    def shell_offsets(self):
        out = np.empty(len(self.shells), dtype=np.int32)
        _check(lib().gto_basis_shell_offsets(self._h, _ptr(out, _ip)), "gto_basis_shell_offsets")
        return out


def overlap(b):
    S = np.empty((b.nbf, b.nbf))
    _check(lib().gto_overlap(b._h, _ptr(S)), "gto_overlap")
    return S


def kinetic(b):
    T = np.empty((b.nbf, b.nbf))
    _check(lib().gto_kinetic(b._h, _ptr(T)), "gto_kinetic")
    return T


def nuclear(b, mol):
    V = np.empty((b.nbf, b.nbf))
    Z = np.ascontiguousarray(mol.charges)
    R = np.ascontiguousarray(mol.coords_bohr.reshape(-1))
    _check(lib().gto_nuclear(b._h, len(Z), _ptr(Z), _ptr(R), _ptr(V)), "gto_nuclear")
    return V


def coulomb_2c(aux):
    V = np.empty((aux.nbf, aux.nbf))
    _check(lib().gto_coulomb_2c(aux._h, _ptr(V)), "gto_coulomb_2c")
    return V


def coulomb_3c(orb, aux, layout=LAYOUT_PACKED):
    n, na = orb.nbf, aux.nbf
    if layout == LAYOUT_NOPT_FULL:
        out = np.empty((n * n, na))
    else:
        out = np.empty((n * (n + 1) // 2, na))
    _check(lib().gto_coulomb_3c(orb._h, aux._h, layout, _ptr(out)), "gto_coulomb_3c")
    return out


def cart_to_sph(l):
    """(2l+1) x ncart(l) matrix C, Y_m = sum_c C[m][c] phi_c (gto_cart_to_sph)."""
    nc = (l + 1) * (l + 2) // 2
    out = np.empty((2 * l + 1, nc))
    _check(lib().gto_cart_to_sph(int(l), _ptr(out)), "gto_cart_to_sph")
    return out


def d5_projector(cart):
    """T (n_cart x n_sph) for a Cartesian basis: column j is spherical function j of the same shells in
    terms of the Cartesian functions, shell by shell (the role of the reference's T_D5,
    src/molecule.cpp:4551-4680).  T^T S_cart T is the overlap of the spherical basis."""
    if cart.pure:
        raise ValueError("d5_projector needs a Cartesian basis")
    nsph = sum(2 * sh.l + 1 for sh in cart.shells)
    T = np.zeros((cart.nbf, nsph))
    r = c = 0
    for sh in cart.shells:
        C = cart_to_sph(sh.l)
        T[r:r + C.shape[1], c:c + C.shape[0]] = C.T
        r += C.shape[1]
        c += C.shape[0]
    return T


def aux_slice_bounds(aux, nslices):
    """About nslices ranges [(p0, p1), ...] of aux functions covering [0, nbf), cut at shell
    boundaries (each range is then one sub-basis of whole shells)."""
    offs = list(aux.shell_offsets()) + [aux.nbf]
    target = aux.nbf / max(int(nslices), 1)
    bounds, p0 = [], 0
    for s in range(1, len(offs)):
        if offs[s] - p0 >= target or s == len(offs) - 1:
            if offs[s] > p0:
                bounds.append((p0, int(offs[s])))
                p0 = int(offs[s])
    return bounds


def coulomb_3c_aux_range(orb, aux, p0, p1, layout=LAYOUT_NOPT_FULL):
    """(mu nu|P) for the aux functions [p0, p1), which must start and end on shell boundaries:
    the three-centre integrals of the sub-basis of those shells, (n^2 or n(n+1)/2) x (p1 - p0)."""
    offs = list(aux.shell_offsets()) + [aux.nbf]
    if p0 not in offs or p1 not in offs or p1 <= p0:
        raise ValueError("aux range [%d, %d) does not fall on shell boundaries" % (p0, p1))
    sub = Basis(aux.shells[offs.index(p0):offs.index(p1)], pure=aux.pure)
    return coulomb_3c(orb, sub, layout)


def atomic_density(sym, orb_basis, aux_basis):
    """(D, rows) of one atom of element `sym` at the origin (see gto_atomic_density)."""
    from .molecules import Z_OF
    at = Molecule([sym], [[0.0, 0.0, 0.0]])
    orb = Basis.for_molecule(orb_basis, at)
    aux = Basis.for_molecule(aux_basis, at)
    n = orb.nbf
    D = np.empty((n, n))
    rows = np.empty((n, n))
    nr = ctypes.c_int(0)
    xyz = np.zeros(3)
    _check(lib().gto_atomic_density(orb._h, aux._h, float(Z_OF[sym]), _ptr(xyz), _ptr(D), _ptr(rows),
                                    ctypes.byref(nr)), "gto_atomic_density")
    return D, rows[:nr.value].copy()


def sad_guess(mol, orb_basis, aux_basis):
    """Block-diagonal superposition of atomic densities over the molecule's atoms (in basis order)
    and its factor rows, D0 = R^T R, the reference's SAD start (src/sad_guess.cpp:165-215)."""
    cache = {}
    blocks = []
    for sym in mol.symbols:
        if sym not in cache:
            cache[sym] = atomic_density(sym, orb_basis, aux_basis)
        blocks.append(cache[sym])
    n = sum(b[0].shape[0] for b in blocks)
    D = np.zeros((n, n))
    R = np.zeros((sum(b[1].shape[0] for b in blocks), n))
    o = r = 0
    for Da, Ra in blocks:
        na, nr = Da.shape[0], Ra.shape[0]
        D[o:o + na, o:o + na] = Da
        R[r:r + nr, o:o + na] = Ra
        o += na
        r += nr
    return D, R


def boys(mmax, T):
    F = np.empty(mmax + 1)
    _check(lib().gto_boys(mmax, T, _ptr(F)), "gto_boys")
    return F


def set_threads(n):
    lib().gto_set_threads(int(n))


class SystemIntegrals:
    """All inputs of an RI-RHF calculation for one molecule."""

    def __init__(self, mol, orb_basis, aux_basis, layout=LAYOUT_PACKED, ri_integrals=True):
        """ri_integrals=False skips (P|Q) and (mu nu|P) on the host (V and I3 are then None), for
        callers that form them on the GPU (FockBuilder.set_basis)."""
        self.mol = mol
        self.orb = Basis.for_molecule(orb_basis, mol)
        self.aux = Basis.for_molecule(aux_basis, mol)
        self.S = overlap(self.orb)
        self.H = kinetic(self.orb) + nuclear(self.orb, mol)
        self.V = coulomb_2c(self.aux) if ri_integrals else None
        self.layout = layout
        self.I3 = coulomb_3c(self.orb, self.aux, layout) if ri_integrals else None
        self.Enuc = mol.nuclear_repulsion()
        self.nocc = mol.nelec // 2
        self.orb_name, self.aux_name = orb_basis, aux_basis

    def sad(self):
        """(D0, factor rows) of the superposition-of-atomic-densities start."""
        return sad_guess(self.mol, self.orb_name, self.aux_name)

    @property
    def n(self):
        return self.orb.nbf

    @property
    def naux(self):
        return self.aux.nbf
