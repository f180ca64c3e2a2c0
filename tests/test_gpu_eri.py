"""Parity of the GPU integral kernels with the host integral engine, through the C ABI.

rijk_eri2c / rijk_eri3c replace RI_V_calc and calc_2el_AO_INTS_RI (src/libint_link.cpp:2049-2107,
:2261-2350); rijk_set_basis replaces gen_RI_AA (src/RI.cpp:34-79) whole.  The host engine
(gto_ints.cpp, the same McMurchie-Davidson scheme) is the comparison: integrals agree to 1e-12
relative to the largest element, J and K built from either set-up to 1e-10, and the SCF energy
through the all-GPU set-up reproduces the reference's logged energy.
"""
import json
import os

import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import Molecule, water_cluster

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pins.json")))
WATER = Molecule(["O", "H", "H"], [[0.0, 0.0, 0.1173], [0.0, 0.7572, -0.4692], [0.0, -0.7572, -0.4692]],
                 name="water")


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b)))


@pytest.fixture(scope="module")
def tz():
    """Water in cc-pVTZ / cc-pVTZ-JKFIT: orbital shells to f, aux shells to g, so every class up
    to (f f|g) is exercised."""
    orb = ints.Basis.for_molecule("cc-pvtz", WATER)
    aux = ints.Basis.for_molecule("cc-pvtz-jkfit", WATER)
    return orb, aux


def test_eri2c_matches_host(tz):
    _, aux = tz
    with rijk.FockBuilder(0) as fb:
        V = fb.eri2c(aux)
    Vh = ints.coulomb_2c(aux)
    assert _rel(V, Vh) < 1e-12, _rel(V, Vh)


@pytest.mark.parametrize("layout", [rijk.LAYOUT_PACKED, rijk.LAYOUT_NOPT_FULL])
def test_eri3c_matches_host(tz, layout):
    orb, aux = tz
    with rijk.FockBuilder(0) as fb:
        I3 = fb.eri3c(orb, aux, layout)
    Ih = ints.coulomb_3c(orb, aux, layout).reshape(I3.shape)
    assert _rel(I3, Ih) < 1e-12, _rel(I3, Ih)


def test_eri_cartesian_shells_match_host():
    orb = ints.Basis.for_molecule("cc-pvtz", WATER, pure=False)
    aux = ints.Basis.for_molecule("cc-pvdz-jkfit", WATER, pure=False)
    with rijk.FockBuilder(0) as fb:
        V = fb.eri2c(aux)
        I3 = fb.eri3c(orb, aux, rijk.LAYOUT_PACKED)
    assert _rel(V, ints.coulomb_2c(aux)) < 1e-12
    assert _rel(I3, ints.coulomb_3c(orb, aux, rijk.LAYOUT_PACKED)) < 1e-12


def _jk_two_ways(si, form, nocc_extra=0):
    rng = np.random.default_rng(5)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    MO = C.T.copy()
    nocc = si.nocc + nocc_extra
    DM = O.gen_hf_dm(MO, si.n, nocc)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V, form)
        fb.set_3c(si.I3, si.n)
        Jh, Kh = fb.dm_to_f_transform_ri(DM, MO, nocc)
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(si.orb, si.aux, form)
        Jg, Kg = fb.dm_to_f_transform_ri(DM, MO, nocc)
        st = fb.stats()
    return (Jh, Kh), (Jg, Kg), st


@pytest.mark.parametrize("form", [rijk.METRIC_INVSQRT, rijk.METRIC_CHOLESKY])
def test_set_basis_matches_host_integrals_water6(form):
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    (Jh, Kh), (Jg, Kg), st = _jk_two_ways(si, form)
    assert np.max(np.abs(Jg - Jh)) < 1e-10 and np.max(np.abs(Kg - Kh)) < 1e-10
    assert st["kernels_setup_ints"] > 0 and st["ms_setup_ints"] > 0


def test_set_basis_two_row_blocks_water16():
    """(H2O)16 cc-pVDZ / JKFIT: the fitted tensor is formed in two blocks of tile rows and the
    block boundary (function 320) falls inside a p shell, which both blocks then compute."""
    si = ints.SystemIntegrals(water_cluster((4, 2, 2), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    offs = si.orb.shell_offsets()
    assert any(o < 320 < o + 3 for o, s in zip(offs, si.orb.shells) if s.l == 1)
    (Jh, Kh), (Jg, Kg), _ = _jk_two_ways(si, rijk.METRIC_INVSQRT)
    assert np.max(np.abs(Jg - Jh)) < 1e-10 and np.max(np.abs(Kg - Kh)) < 1e-10


def test_set_basis_aux_slices_sum_to_full():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=1), "cc-pvdz", "cc-pvdz-jkfit")
    rng = np.random.default_rng(2)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    MO = C.T.copy()
    DM = O.gen_hf_dm(MO, si.n, si.nocc)
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(si.orb, si.aux)
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
    h = si.naux // 3
    Js, Ks = np.zeros_like(J), np.zeros_like(K)
    for q0, q1 in [(0, h), (h, si.naux)]:
        with rijk.FockBuilder(0) as fb:
            fb.set_basis(si.orb, si.aux, rijk.METRIC_INVSQRT, q0, q1)
            j, k = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
        Js += j
        Ks += k
    assert np.max(np.abs(Js - J)) < 1e-10 and np.max(np.abs(Ks - K)) < 1e-10


def test_set_basis_reproduces_reference_energy_c2h4():
    p = [q for q in GOLD["pins"] if q["name"] == "c2h4"][0]
    mol = Molecule(p["symbols"], p["coords_ang"])
    orb = ints.Basis.for_molecule(p["basis"], mol)
    aux = ints.Basis.for_molecule(p["aux"], mol)
    S = ints.overlap(orb)
    H = ints.kinetic(orb) + ints.nuclear(orb, mol)
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(orb, aux)
        E, _, r = fb.scf(H, S, mol.nelec // 2, mol.nuclear_repulsion())
    assert r["converged"] == 1
    assert abs(E - p["energy"]) < 2e-9, (E, p["energy"])
