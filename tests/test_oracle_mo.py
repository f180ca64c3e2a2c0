"""The oracle's MO-basis tensor restatements (reference operation order) agree with the
direct contraction of the fitted tensor, B^Q = V^-1/2 (P|mu nu): (pa|Q) = C1 B^Q C2^T."""
import numpy as np

import rijk_oracle as O


def _fixture(n=13, naux=29, seed=0):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n, naux))
    RI = (A + A.transpose(1, 0, 2)).reshape(n * n, naux)
    X = rng.normal(size=(naux, naux))
    V = X @ X.T + naux * np.eye(naux)
    Vm05, _ = O.s05_calc(V)
    B = np.einsum("qp,mnp->qmn", Vm05, RI.reshape(n, n, naux))
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    return n, RI, Vm05, B, C.T.copy()


def _pa(B, C1, C2):
    return np.einsum("pm,qmn,an->paq", C1, B, C2).reshape(C1.shape[0] * C2.shape[0], -1)


def test_mo_calc_is_the_fitted_contraction():
    n, RI, Vm05, B, VEC = _fixture()
    nc, na = 4, 3
    nv = n - nc - na
    CC, VC, AA, CA, VA = O.mo_calc(RI, Vm05, VEC, nc, na, nv, n)
    COR, ACT, VAC = VEC[:nc], VEC[nc:nc + na], VEC[nc + na:]
    for got, (C1, C2) in zip((CC, VC, AA, CA, VA), ((COR, COR), (VAC, COR), (ACT, ACT), (COR, ACT), (VAC, ACT))):
        assert np.allclose(got, _pa(B, C1, C2), atol=1e-11)


def test_aaag_and_soscf_are_the_fitted_contractions():
    n, RI, Vm05, B, MO = _fixture(seed=1)
    nc, na = 3, 4
    A = MO[nc:nc + na]
    Y = np.einsum("tm,qmn,un->qtu", A, B, A)
    Z = np.einsum("vm,qmn,xn->qvx", A, B, MO)
    ref = np.einsum("qtu,qvx->tuvx", Y, Z).reshape(na ** 3, n)
    assert np.allclose(O.mo_ints_aaag(RI, Vm05, MO, nc, na, n), ref, atol=1e-11)
    aJ, aK = O.soscf_hess_ints(RI, Vm05, MO, nc, na, n)
    pp = np.einsum("pm,qmn,pn->pq", MO, B, MO)
    assert np.allclose(aJ, np.einsum("pq,qtu->ptu", pp, Y).reshape(n, na * na), atol=1e-11)
    pt = np.einsum("pm,qmn,tn->ptq", MO, B, A)
    assert np.allclose(aK, np.einsum("ptq,puq->ptu", pt, pt).reshape(n, na * na), atol=1e-11)
