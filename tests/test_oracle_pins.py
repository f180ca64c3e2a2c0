"""Pins of the oracle and the host integral engine against the reference's own known answers.

The reference's example logs are its regression tests; their final RI-RHF energies
(cc-pVDZ / cc-pVDZ-RI, D5 spherical MOs) pin integrals + metric + RI-JK + SCF end to end.
Fixtures: tests/golden/pins.json (made by tests/golden/make_golden.py).
"""
import json
import os

import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints
from nopt_b200.basis import Shell
from nopt_b200.molecules import Molecule

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pins.json")))


def _mol(p):
    return Molecule(p["symbols"], p["coords_ang"], name=p["name"])


def test_carbon_contraction_normalisation_matches_reference_log():
    """Column "c" of the reference's basis table = libint-normalised coefficients."""
    mol = Molecule(["C"], [[0.0, 0.0, 0.0]])
    b = ints.Basis.for_molecule("cc-pvdz", mol)
    ours = b.norm_coefs()
    ref = np.array([c["c"] for c in GOLD["carbon_ccpvdz_norm_coefs"]])
    assert len(ours) == len(ref)
    np.testing.assert_allclose(ours, ref, atol=6e-7, rtol=0)  # log prints 6 decimals


@pytest.mark.parametrize("name", ["c2h4", "c6h8", "guanine"])
def test_ri_rhf_energy_pin(name):
    p = [q for q in GOLD["pins"] if q["name"] == name][0]
    mol = _mol(p)
    si = ints.SystemIntegrals(mol, p["basis"], p["aux"], layout=ints.LAYOUT_NOPT_FULL)
    Vm05, _ = O.s05_calc(si.V)
    E, MO, DM, F, it = O.scf_rhf(si.S, si.H, si.I3, Vm05, si.nocc, si.Enuc)
    # the logs stop at |dE| ~ 1e-10 with 10 printed decimals
    assert abs(E - p["energy"]) < 2e-9, (E, p["energy"])


def test_h2_sto3g_textbook_integrals():
    """H2, R = 1.4 bohr, STO-3G (Szabo & Ostlund, Table 3.x values)."""
    e = [3.42525091, 0.62391373, 0.16885540]
    c = [0.15432897, 0.53532814, 0.44463454]
    b = ints.Basis([Shell(0, e, c, (0, 0, 0), 0), Shell(0, e, c, (0, 0, 1.4), 1)])
    mol = Molecule(["H", "H"], np.array([[0, 0, 0], [0, 0, 1.4]]) / 1.889725989)
    S, T, V = ints.overlap(b), ints.kinetic(b), ints.nuclear(b, mol)
    assert abs(S[0, 1] - 0.6593) < 1e-4
    assert abs(T[0, 0] - 0.7600) < 1e-4 and abs(T[0, 1] - 0.2365) < 1e-4
    assert abs(V[0, 0] - (-1.8804)) < 1e-4 and abs(V[0, 1] - (-1.1948)) < 1e-4


def test_boys_function_against_hypergeometric():
    from scipy.special import hyp1f1
    for T in [0.0, 1e-3, 0.3, 5.7, 17.2, 35.0, 39.99, 45.0, 120.0]:
        F = ints.boys(12, T)
        ref = np.array([hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1) for m in range(13)])
        np.testing.assert_allclose(F, ref, rtol=1e-13, atol=0)


def test_spherical_shells_orthonormal_on_one_centre():
    mol = Molecule(["O"], [[0.0, 0.0, 0.0]])
    for name in ["cc-pvtz", "cc-pvtz-jkfit"]:
        b = ints.Basis.for_molecule(name, mol)
        S = ints.overlap(b)
        np.testing.assert_allclose(np.diag(S), 1.0, atol=1e-12)
        offs = list(b.shell_offsets()) + [b.nbf]
        for s, sh in enumerate(b.shells):
            blk = S[offs[s]:offs[s + 1], offs[s]:offs[s + 1]]
            np.testing.assert_allclose(blk, np.eye(2 * sh.l + 1), atol=1e-12)


def test_three_centre_matches_two_centre_for_one_centre_products():
    """(s_a s_a | P) with both s primitives on one centre equals (G|P) for the product
    Gaussian G of exponent 2a, up to the normalisation ratio."""
    a = 0.8
    mol = Molecule(["O", "H"], [[0.0, 0.0, 0.0], [0.3, -0.4, 1.1]])
    orb = ints.Basis([Shell(0, [a], [1.0], (0, 0, 0), 0)])
    aux_sh = [Shell(l, [0.9], [1.0], tuple(mol.coords_bohr[1]), 1) for l in range(5)]
    prod = ints.Basis([Shell(0, [2 * a], [1.0], (0, 0, 0), 0)] + aux_sh)
    aux = ints.Basis(aux_sh)
    I3 = ints.coulomb_3c(orb, aux)[0]
    V = ints.coulomb_2c(prod)[0, 1:]
    na = (2 * a / np.pi) ** 0.75
    nprod = (4 * a / np.pi) ** 0.75
    np.testing.assert_allclose(I3, V * na * na / nprod, rtol=1e-12, atol=1e-14)


def test_three_centre_rotational_invariance_of_fitted_energy():
    """The RI Coulomb energy of a fixed density is invariant under rigid rotation."""
    rng = np.random.default_rng(3)
    X = np.array([[0, 0, 0], [0.96, 0, 0], [-0.24, 0.93, 0]], float)
    sym = ["O", "H", "H"]
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    out = []
    for coords in (X, X @ q.T):
        mol = Molecule(sym, coords)
        si = ints.SystemIntegrals(mol, "cc-pvtz", "cc-pvtz-jkfit", layout=ints.LAYOUT_NOPT_FULL)
        Vm05, _ = O.s05_calc(si.V)
        E, MO, DM, F, it = O.scf_rhf(si.S, si.H, si.I3, Vm05, si.nocc, si.Enuc)
        out.append(E)
    assert abs(out[0] - out[1]) < 1e-9


def test_sad_guess_density_and_factor_rows():
    """The superposition of atomic densities carries n_occ electron pairs, factors as R^T R and
    starts the oracle SCF at the reference's C2H4 energy."""
    p = [q for q in GOLD["pins"] if q["name"] == "c2h4"][0]
    si = ints.SystemIntegrals(_mol(p), p["basis"], p["aux"], layout=ints.LAYOUT_NOPT_FULL)
    D0, R = si.sad()
    assert abs(np.sum(D0 * si.S) - si.nocc) < 1e-10
    np.testing.assert_allclose(R.T @ R, D0, atol=1e-12)
    Vm05, _ = O.s05_calc(si.V)
    E, MO, DM, F, it = O.scf_rhf(si.S, si.H, si.I3, Vm05, si.nocc, si.Enuc, guess=(D0, R))
    assert abs(E - p["energy"]) < 2e-9


def test_soscf_converger_restatement_reaches_reference_energy():
    """The restatement of the reference's own converger (SOSCF with L-BFGS, src/SCF.cpp:125-174)
    lands on the logged C2H4 energy from the core guess and from the SAD start."""
    p = [q for q in GOLD["pins"] if q["name"] == "c2h4"][0]
    si = ints.SystemIntegrals(_mol(p), p["basis"], p["aux"], layout=ints.LAYOUT_NOPT_FULL)
    Vm05, _ = O.s05_calc(si.V)
    E, MO, hist, conv = O.scf_soscf(si.S, si.H, si.I3, Vm05, si.nocc, si.Enuc)
    assert conv and abs(E - p["energy"]) < 2e-9, (E, p["energy"])
    Eg, _, hg, convg = O.scf_soscf(si.S, si.H, si.I3, Vm05, si.nocc, si.Enuc, guess=si.sad())
    assert convg and abs(Eg - p["energy"]) < 2e-9 and len(hg) < len(hist)


def test_gram_schmidt_rows_is_qr_with_positive_diagonal():
    """Row-wise Gram-Schmidt of I + X - X^T equals Q^T of the QR factorisation of its transpose
    with R's diagonal made positive (the form the device code uses)."""
    rng = np.random.default_rng(3)
    no, nv = 5, 9
    x = 0.1 * rng.normal(size=(no, nv))
    R = np.eye(no + nv)
    R[:no, no:] = x
    R[no:, :no] = -x.T
    Q, Rr = np.linalg.qr(R.T)
    Q = Q * np.sign(np.diag(Rr))
    np.testing.assert_allclose(O.gram_schmidt_rows(R), Q.T, atol=1e-13)


def test_cartesian_basis_with_d5_projection_reaches_the_logged_energy():
    """The reference's orbital basis is Cartesian with D5 = 1 (src/inp_par_read.cpp:2550-2552,
    src/molecule.cpp:4004-4050): the SCF in the Cartesian AO basis with the orbitals confined to
    the spherical span reaches the logged C2H4 energy; without the projection it does not."""
    p = [q for q in GOLD["pins"] if q["name"] == "c2h4"][0]
    mol = _mol(p)
    orb = ints.Basis.for_molecule(p["basis"], mol, pure=False)
    aux = ints.Basis.for_molecule(p["aux"], mol)
    S, H = ints.overlap(orb), ints.kinetic(orb) + ints.nuclear(orb, mol)
    RI = ints.coulomb_3c(orb, aux, ints.LAYOUT_NOPT_FULL)
    Vm05, _ = O.s05_calc(ints.coulomb_2c(aux))
    nocc = mol.nelec // 2
    T = ints.d5_projector(orb)
    E, MO, DM, F, it = O.scf_rhf(S, H, RI, Vm05, nocc, mol.nuclear_repulsion(), projector=T)
    assert abs(E - p["energy"]) < 2e-9, (E, p["energy"])
    E6, *_ = O.scf_rhf(S, H, RI, Vm05, nocc, mol.nuclear_repulsion())
    assert E6 < p["energy"] - 1e-4  # the full Cartesian space holds the extra s-type combinations
