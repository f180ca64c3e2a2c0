"""Element-wise parity at the benchmark workloads' sizes.

- (H2O)16 cc-pVDZ/cc-pVDZ-JKFIT (n = 384, naux = 1856, n_c = 80): FP64 J and K against the
  oracle's restatement of DM_to_F_transform_RI (src/RI.cpp:115-176) in NOPT's full-square layout
  to 1e-9, and the mixed form's K to its 2e-4 bar.
- C40H82 cc-pVDZ/cc-pVDZ-JKFIT (n = 970 padded to 1024, naux = 4686, n_c = 161): the full-square
  RI_AA (35 GB) is left out; instead three aux slices of a context (rijk_set_aux_range), with the
  Cholesky metric whose rows L^-1[Q, :] are unique, are checked against the oracle's J and K of
  the same slices from the packed fitted tensor (jk_from_b).  This pins the n >= 1024 code paths
  (the CTA-pair mixed K included) against the oracle rather than against the GPU FP64 form.
"""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import WORKLOADS

pytestmark = pytest.mark.gpu
TOL_JK = 1e-9
TOL_K_MIXED = 2e-4


def _scf_like_state(si, fb, nocc):
    """Orbitals of the first Fock matrix from the SAD start: a realistic density."""
    s_, U_ = np.linalg.eigh(si.S)
    Xo = U_[:, s_ > 1e-10] / np.sqrt(s_[s_ > 1e-10])
    D0, R0 = si.sad()
    Jg, Kg = fb.dm_to_f_transform_ri(D0, R0, R0.shape[0])
    _, Cp = np.linalg.eigh(Xo.T @ (si.H + 2 * Jg - Kg) @ Xo)
    MO = (Xo @ Cp).T.copy()
    return O.gen_hf_dm(MO, si.n, nocc), MO


def test_fp64_and_mixed_jk_h2o16_elementwise():
    fac, ob, ab = WORKLOADS["h2o16_dz"]
    si = ints.SystemIntegrals(fac(0), ob, ab)
    n, nocc = si.n, si.nocc
    Vm05, _ = O.s05_calc(si.V)
    RI = O.unpack_3c(si.I3, n)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V, rijk.METRIC_INVSQRT)
        fb.set_3c(si.I3, n)
        DM, MO = _scf_like_state(si, fb, nocc)
        J, K = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_FP64)
        Jm, Km = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_MIXED)
    Jr, Kr = O.dm_to_f_transform_ri(RI, Vm05, DM, MO, nocc, n)
    assert np.max(np.abs(J - Jr)) < TOL_JK
    assert np.max(np.abs(K - Kr)) < TOL_JK
    assert np.max(np.abs(Jm - Jr)) < 1e-4 * max(1.0, float(np.max(np.abs(Jr))))
    assert np.max(np.abs(Km - Kr)) < TOL_K_MIXED
    assert abs(float(np.sum(DM * (Km - Kr)))) < 1e-3


def test_c40h82_aux_slices_against_oracle():
    fac, ob, ab = WORKLOADS["c40h82_dz"]
    si = ints.SystemIntegrals(fac(0), ob, ab)  # packed (mu nu|P) on the host, 17.6 GB
    n, naux, nocc = si.n, si.naux, si.nocc
    Linv = O.cholesky_inverse_factor(si.V)
    rng = np.random.default_rng(40)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    DM = O.gen_hf_dm(MO, n, nocc)
    for q0, q1 in ((0, 37), (2301, 2350), (naux - 29, naux)):
        with rijk.FockBuilder(0) as fb:
            fb.set_metric(si.V, rijk.METRIC_CHOLESKY)
            fb.set_aux_range(q0, q1)
            fb.set_3c(si.I3, n)
            J, K = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_FP64)
            Jm, Km = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_MIXED)
        Bp = O.b_tensor(si.I3, Linv[q0:q1])  # (q1 - q0) x npair
        Jr, Kr = O.jk_from_b(Bp, n, DM, MO, nocc)
        assert np.max(np.abs(J - Jr)) < TOL_JK, (q0, q1)
        assert np.max(np.abs(K - Kr)) < TOL_JK, (q0, q1)
        assert np.max(np.abs(Km - Kr)) < TOL_K_MIXED, (q0, q1)
        assert np.max(np.abs(Jm - Jr)) < 1e-4 * max(1.0, float(np.max(np.abs(Jr)))), (q0, q1)
