"""Active-space MO integrals (rijk_mo_ints) against the oracle's restatement of
calc_2el_MO_INTS_RI (src/RI.cpp:178-292), including the core J/K tail and the transposed
(t = 1) orbital layout; tolerance 1e-9 max-abs (FP64)."""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import Molecule, water_cluster

pytestmark = pytest.mark.gpu


def _case(si, n_core, n_act, seed, t):
    rng = np.random.default_rng(seed)
    Cq, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    MO = Cq.T.copy()
    D = O.gen_hf_dm(MO, si.n, n_core)
    act = MO[n_core:n_core + n_act]
    C1 = act.T.copy() if t else act.copy()
    Vm05, _ = O.s05_calc(si.V)
    RI = O.unpack_3c(si.I3, si.n)
    Ir, Jr, Kr = O.calc_2el_mo_ints_ri(RI, Vm05, si.n, D, MO, C1, C1, n_core, n_act, t)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        I, J, K = fb.calc_2el_mo_ints_ri(D, MO, C1, C1, n_core, n_act, t)
        I2, _, _ = fb.calc_2el_mo_ints_ri(None, MO, C1, C1, n_core, n_act, t, want_jk=False)
    assert np.max(np.abs(I - Ir)) < 1e-9
    assert np.array_equal(I, I2)
    assert np.max(np.abs(J - Jr)) < 1e-9 and np.max(np.abs(K - Kr)) < 1e-9
    # (ab|cd) symmetries of real orbitals with C1 = C2
    T4 = I.reshape(n_act, n_act, n_act, n_act)
    assert np.max(np.abs(T4 - T4.transpose(2, 3, 0, 1))) < 1e-12
    assert np.max(np.abs(T4 - T4.transpose(1, 0, 2, 3))) < 1e-10


def test_moints_c2h4_cas22():
    """The CAS(2,2) of the reference's ethylene example (examples/c2h4_2_2/cas.inp)."""
    mol = Molecule(["C", "C", "H", "H", "H", "H"],
                   [[0, 0, -0.6695], [0, 0, 0.6695], [0, -0.9289, 1.2321], [0, 0.9289, -1.2321],
                    [0, -0.9289, -1.2321], [0, 0.9289, 1.2321]])
    si = ints.SystemIntegrals(mol, "cc-pvdz", "cc-pvdz-ri")
    _case(si, 7, 2, 1, 0)


@pytest.mark.parametrize("t", [0, 1])
def test_moints_water_hexamer_cas10(t):
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    _case(si, 25, 10, 2, t)
