"""Parity of the CUDA Fock build (through the C ABI) with the CPU oracle.

FP64 form: J and K must match the oracle's restatement of DM_to_F_transform_RI
(src/RI.cpp:115-176) to 1e-9 max-abs (same metric form on both sides), and energies to
1e-10 Eh.  Inputs are the package's integrals for small molecules and seeded random
tensors for the edge cases (ragged n, n_c not a multiple of 16, n_c = 0, unsymmetric D).
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
TOL_JK = 1e-9


def _pin_mol(name):
    p = [q for q in GOLD["pins"] if q["name"] == name][0]
    return Molecule(p["symbols"], p["coords_ang"], name=name), p


@pytest.fixture(scope="module")
def c2h4():
    mol, p = _pin_mol("c2h4")
    si = ints.SystemIntegrals(mol, p["basis"], p["aux"], layout=ints.LAYOUT_PACKED)
    return si, p


def _oracle_jk(si, M, DM, MO, nocc):
    RI = O.unpack_3c(si.I3, si.n)
    if M is None:
        M, _ = O.s05_calc(si.V)
    # M^T M = V^-1 for both metric forms; the oracle's V^-1/2 sandwich uses the symmetric M
    return O.dm_to_f_transform_ri(RI, M, DM, MO, nocc, si.n)


def _random_state(n, nocc, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    DM = O.gen_hf_dm(MO, n, nocc)
    return DM, MO


@pytest.mark.parametrize("form", [rijk.METRIC_INVSQRT, rijk.METRIC_CHOLESKY])
@pytest.mark.parametrize("layout", [rijk.LAYOUT_PACKED, rijk.LAYOUT_NOPT_FULL])
def test_jk_parity_c2h4(c2h4, form, layout):
    si, _ = c2h4
    DM, MO = _random_state(si.n, si.nocc, 1)
    Jr, Kr = _oracle_jk(si, None, DM, MO, si.nocc)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V, form)
        I3 = si.I3 if layout == rijk.LAYOUT_PACKED else O.unpack_3c(si.I3, si.n)
        fb.set_3c(I3, si.n, layout)
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
    assert np.max(np.abs(J - Jr)) < TOL_JK
    assert np.max(np.abs(K - Kr)) < TOL_JK


def test_scf_energy_through_gpu_fock_matches_reference_log(c2h4):
    """The RI-RHF energy with every Fock build on the GPU equals the reference's logged
    energy (examples/c2h4_2_2/benchmark.log) and the oracle's."""
    si, p = c2h4
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V, rijk.METRIC_INVSQRT)
        fb.set_3c(si.I3, si.n)
        jk = lambda D, MO: fb.dm_to_f_transform_ri(D, MO, si.nocc)
        E, MO, DM, F, it = O.scf_rhf(si.S, si.H, None, None, si.nocc, si.Enuc, jk=jk)
    assert abs(E - p["energy"]) < 2e-9


def test_jk_parity_water_hexamer_jkfit():
    mol = water_cluster((2, 3), seed=0)
    si = ints.SystemIntegrals(mol, "cc-pvdz", "cc-pvdz-jkfit")
    assert (si.n, si.naux, si.nocc) == (144, 696, 30)
    DM, MO = _random_state(si.n, si.nocc, 2)
    Jr, Kr = _oracle_jk(si, None, DM, MO, si.nocc)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
    assert np.max(np.abs(J - Jr)) < TOL_JK
    assert np.max(np.abs(K - Kr)) < TOL_JK


@pytest.mark.parametrize("precision", [rijk.PREC_FP64, rijk.PREC_FP64_TC])
def test_two_stream_build_equals_one_stream_build(precision):
    """FP64 builds run the Coulomb pair on a second stream beside the half-transform, with capped grids
    that stride over the work; with per-kernel timing on, every kernel runs alone on full grids.  Each aux
    function's w and each element's J are summed in the same order either way: J and K are identical."""
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    DM, MO = _random_state(si.n, si.nocc, 5)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        J2, K2 = fb.dm_to_f_transform_ri(DM, MO, si.nocc, precision)
        fb.set_profiling(True)
        J1, K1 = fb.dm_to_f_transform_ri(DM, MO, si.nocc, precision)
        assert fb.stats()["profiled_stages"] > 0
    assert np.array_equal(J1, J2) and np.array_equal(K1, K2)


def _random_problem(n, naux, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(naux, naux))
    V = A @ A.T / naux + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 0.1
    return V, I3


@pytest.mark.parametrize("n,naux,nocc", [(70, 100, 13), (64, 33, 16), (1, 5, 1), (130, 257, 0), (200, 96, 97),
                                         (200, 96, 161), (180, 40, 130), (150, 70, 113), (260, 50, 160),
                                         (300, 64, 282)])
def test_jk_parity_ragged_random(n, naux, nocc):
    V, I3 = _random_problem(n, naux, n + naux)
    rng = np.random.default_rng(7)
    DM = rng.normal(size=(n, n))  # the reference uses DM as given: not symmetrised
    MO = rng.normal(size=(max(nocc, 1), n))
    Vm05, _ = O.s05_calc(V)
    Jr, Kr = O.dm_to_f_transform_ri(O.unpack_3c(I3, n), Vm05, DM, MO, nocc, n)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(V)
        fb.set_3c(I3, n)
        J, K = fb.dm_to_f_transform_ri(DM, MO, nocc)
    scale = max(1.0, np.max(np.abs(Jr)), np.max(np.abs(Kr)))
    assert np.max(np.abs(J - Jr)) < TOL_JK * scale
    assert np.max(np.abs(K - Kr)) < TOL_JK * scale
    if nocc == 0:
        assert not K.any()


def test_errors_are_status_codes_not_crashes():
    with rijk.FockBuilder(0) as fb:
        with pytest.raises(rijk.RijkError) as e:
            fb.n = 4
            fb.dm_to_f_transform_ri(np.eye(4), np.eye(4), 2)
        assert e.value.code == rijk.ERR_STATE
        with pytest.raises(rijk.RijkError) as e:
            fb.set_metric(np.eye(3), form=7)
        assert e.value.code == rijk.ERR_ARG
        with pytest.raises(rijk.RijkError) as e:
            fb.set_metric(-np.eye(3), form=rijk.METRIC_CHOLESKY)
        assert e.value.code == rijk.ERR_SOLVER
        V, I3 = _random_problem(8, 6, 0)
        fb.set_metric(V)
        with pytest.raises(rijk.RijkError) as e:
            fb.set_3c(I3[:, :5], 8)  # naux differs from the metric's
        assert e.value.code == rijk.ERR_ARG
        fb.set_3c(I3, 8)
        with pytest.raises(rijk.RijkError) as e:
            fb.dm_to_f_transform_ri(np.eye(8), np.eye(8), 17)  # n_c beyond n_ao (padded to 16)
        assert e.value.code == rijk.ERR_ARG
        with pytest.raises(rijk.RijkError) as e:
            fb.dm_to_f_transform_ri(np.eye(8), np.eye(8), 2, precision=5)
        assert e.value.code == rijk.ERR_ARG
        J, K = fb.dm_to_f_transform_ri(np.eye(8), np.eye(8), 2)  # context still usable
        assert np.isfinite(J).all() and np.isfinite(K).all()


def test_fock_energy_conventions(c2h4):
    si, _ = c2h4
    DM, MO = _random_state(si.n, si.nocc, 3)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
        for mc in (0, 1, 2):
            F, E = fb.calc_f_ao(si.H, DM, J, K, c=1.0, mc=mc, e_nuc=si.Enuc)
            Fr = O.calc_f_ao(si.H, J, K, 1.0, mc)
            assert np.max(np.abs(F - Fr)) < 1e-12
            assert abs(E - O.rhf_energy(Fr, si.H, DM, si.Enuc)) < 1e-10
