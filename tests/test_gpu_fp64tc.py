"""The FP64 form with K on tcgen05 tensor cores (RIJK_PREC_FP64_TC): X^T split into 8 int8 digit
planes with a power-of-two exponent per row and split-K part, 36 exact s32 digit products, FP64
scaling.  It is held to the FP64 bar: J and K within 1e-9 of the oracle (relative to max|J|, max|K|
where those exceed 1), the exchange energy tr(D K) within 1e-10 relative; J is the FP64 form's own.
Cases cover ragged n, n_c = 1 and n_c off a multiple of 16, a contraction length that ends in half
a 32-wide chunk, 128-row blocks past n (n = 1000), and integrals whose magnitudes span 12 decades."""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _state(n, nocc, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    return O.gen_hf_dm(MO, n, nocc), MO


def _check(V, I3, n, nocc, DM, MO):
    Vm05, _ = O.s05_calc(V)
    Jr, Kr = O.dm_to_f_transform_ri(O.unpack_3c(I3, n), Vm05, DM, MO, nocc, n)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(V)
        fb.set_3c(I3, n)
        Jf, Kf = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_FP64)
        Jt, Kt = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_FP64_TC)
        Jt2, Kt2 = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_FP64_TC)
    assert np.array_equal(Jt, Jf)
    assert np.array_equal(Kt, Kt2)
    eK = float(np.max(np.abs(Kt - Kr)))
    assert eK < TOL * max(1.0, float(np.max(np.abs(Kr)))), eK
    ex = abs(float(np.sum(DM * (Kt - Kr))))
    assert ex < 1e-10 * max(1.0, abs(float(np.sum(DM * Kr)))), ex
    return eK, float(np.max(np.abs(Kf - Kr)))


@pytest.mark.parametrize("n,naux,nocc", [(64, 40, 16), (150, 70, 1), (200, 96, 97), (333, 211, 45), (260, 48, 192),
                                         (420, 60, 33), (580, 50, 40), (900, 36, 30), (1000, 40, 48)])
def test_fp64tc_k_ragged_random(n, naux, nocc):
    """naux * noccp = 70 * 16 ends in half a 32-wide chunk; n = 420, 580, 900 and 1000 end in a partly
    filled block of 128 rows, and n = 1000 fills 8 such blocks, the last one past npad."""
    rng = np.random.default_rng(n + naux)
    A = rng.normal(size=(naux, naux))
    V = A @ A.T / naux + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 0.1
    DM, MO = _state(n, nocc, 3)
    _check(V, I3, n, nocc, DM, MO)


def test_fp64tc_k_wide_magnitudes():
    """Pair rows scaled by 10^u, u uniform in [-6, 6]: rows of X^T differ by many binades, and small
    entries of a row sit far below its exponent."""
    n, naux, nocc = 180, 64, 30
    rng = np.random.default_rng(11)
    A = rng.normal(size=(naux, naux))
    V = A @ A.T / naux + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 10.0 ** rng.uniform(-6, 6, size=(n * (n + 1) // 2, 1))
    DM, MO = _state(n, nocc, 4)
    _check(V, I3, n, nocc, DM, MO)


def test_fp64tc_k_water_hexamer():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    DM, MO = _state(si.n, si.nocc, 2)
    eK, eKf = _check(si.V, si.I3, si.n, si.nocc, DM, MO)
    assert eK < 1e-11, (eK, eKf)


def test_fp64tc_scf_matches_fp64():
    """rijk_scf with every build in the FP64_TC form (the SAD guess build included) converges to the
    FP64 energy: the digit form is held to FP64 accuracy, so it converges on the FP64 criteria."""
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=1), "cc-pvdz", "cc-pvdz-jkfit")
    guess = si.sad()
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E64, _, r64 = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess)
        Et, _, rt = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, precision=rijk.PREC_FP64_TC)
    assert r64["converged"] and rt["converged"]
    assert rt["iterations_mixed"] == 0
    assert abs(Et - E64) < 1e-10, (Et, E64)
