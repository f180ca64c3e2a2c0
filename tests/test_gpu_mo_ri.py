"""Parity of the MO-basis fitted tensors (rijk_mo_calc, rijk_mo_ints_aaag, rijk_soscf_hess_ints,
rijk_mo_tensor) with the oracle's restatements of RI_data::MO_calc (src/RI.cpp:469-587),
calc_2el_MO_INTS_AAAG_RI (src/RI.cpp:294-346) and calc_SOSCF_hess_INTS_RI (src/RI.cpp:348-450).

The tensors are compared elementwise (V^-1/2 metric, as the reference) to 1e-10; with the
Cholesky metric only their contractions over Q are compared, since the tensors themselves then
differ by a rotation of the aux index.
"""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def sys6():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=3), "cc-pvdz", "cc-pvdz-jkfit")
    RI = O.unpack_3c(si.I3, si.n)
    Vm05, _ = O.s05_calc(si.V)
    rng = np.random.default_rng(11)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    return si, RI, Vm05, C.T.copy()


def _builder(si, form=rijk.METRIC_INVSQRT):
    fb = rijk.FockBuilder(0)
    fb.set_metric(si.V, form)
    fb.set_3c(si.I3, si.n)
    return fb


@pytest.mark.parametrize("n_cor,n_act", [(25, 6), (20, 17), (0, 8)])
def test_mo_calc_matches_oracle(sys6, n_cor, n_act):
    si, RI, Vm05, VEC = sys6
    n_vac = si.n - n_cor - n_act
    ref = dict(zip(("CC", "VC", "AA", "CA", "VA"), O.mo_calc(RI, Vm05, VEC, n_cor, n_act, n_vac, si.n)))
    with _builder(si) as fb:
        got = fb.mo_calc(VEC, n_cor, n_act, n_vac)
    for k in ref:
        if ref[k].size:
            assert np.max(np.abs(got[k] - ref[k])) < TOL, k


def test_mo_calc_products_cholesky(sys6):
    """VAAA = VA AA^T (RI_data::VAAA_calc, src/RI.cpp:588-598) is metric-form independent."""
    si, RI, Vm05, VEC = sys6
    n_cor, n_act = 25, 6
    n_vac = si.n - n_cor - n_act
    _, _, AA, _, VA = O.mo_calc(RI, Vm05, VEC, n_cor, n_act, n_vac, si.n)
    with _builder(si, rijk.METRIC_CHOLESKY) as fb:
        got = fb.mo_calc(VEC, n_cor, n_act, n_vac)
    assert np.max(np.abs(got["VA"] @ got["AA"].T - VA @ AA.T)) < TOL


@pytest.mark.parametrize("n_c,n_a", [(25, 6), (10, 17)])
def test_mo_ints_aaag_matches_oracle(sys6, n_c, n_a):
    si, RI, Vm05, MO = sys6
    ref = O.mo_ints_aaag(RI, Vm05, MO, n_c, n_a, si.n)
    with _builder(si) as fb:
        got = fb.mo_ints_aaag(MO, n_c, n_a)
    assert np.max(np.abs(got - ref)) < TOL


@pytest.mark.parametrize("n_c,n_a", [(25, 6), (3, 17)])
def test_soscf_hess_ints_match_oracle(sys6, n_c, n_a):
    si, RI, Vm05, MO = sys6
    aJ, aK = O.soscf_hess_ints(RI, Vm05, MO, n_c, n_a, si.n)
    with _builder(si) as fb:
        gJ, gK = fb.soscf_hess_ints(MO, n_c, n_a)
    assert np.max(np.abs(gJ - aJ)) < TOL and np.max(np.abs(gK - aK)) < TOL


def test_mo_tensor_ragged_and_aux_slice(sys6):
    """(p a|Q) for ragged orbital counts, and an aux slice returns its columns of the full tensor."""
    si, RI, Vm05, MO = sys6
    C1, C2 = MO[:37], MO[40:53]
    ref = (C1 @ O._half(RI, Vm05, C2, si.n)[1]).reshape(37 * 13, -1)
    with _builder(si) as fb:
        got = fb.mo_tensor(C1, C2)
    assert np.max(np.abs(got - ref)) < TOL
    q0, q1 = 100, 333
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_aux_range(q0, q1)
        fb.set_3c(si.I3, si.n)
        part = fb.mo_tensor(C1, C2)
    assert part.shape == (37 * 13, q1 - q0)
    assert np.max(np.abs(part - ref[:, q0:q1])) < TOL
