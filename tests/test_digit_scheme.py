"""The FP64_TC exchange's digit arithmetic (k_exchange_i8.cu), restated in numpy and run on the fitted
integrals of the water hexamer: each row of X^T is 2^e sum_s d_s 2^-7(s+1) with 8 balanced 7-bit
digits (k_slice_x: e = ilogb(row max) + 2, round to nearest, exact remainder), and
K = 2^(e_mu + e_nu) sum_g 2^-7(g+2) sum_{s+t=g} d_s . d_t over the groups g < 8 (k_syrk_i8).  The
digit products are integers below 2^53, so float64 matrix products form them exactly here, as the s32
tensor-core sums do on the device.  Measured against an extended-precision K: eight digits are within
2.4e-14 (FP64 BLAS: 1.6e-15).  The dropped groups hold the squares d_s^2 with 2s >= 8, always positive,
so the diagonal runs low by about kdim 2^-60 of the row scales.  Seven digits (28 products instead of
36) are within 4.9e-14, the margin for a cheaper form; six are 3.8e-10 off, too coarse for the FP64 bar."""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints
from nopt_b200.molecules import water_cluster


def slice_rows(XT, nd):
    """k_slice_x on one part: per-row exponent and nd digit planes (integer-valued doubles)."""
    m = np.max(np.abs(XT), axis=1)
    e = np.where(m > 0, np.frexp(m)[1] + 1, 0)  # ilogb(m) + 2
    r = np.ldexp(XT, -e[:, None])
    planes = []
    for _ in range(nd):
        t = r * 128.0
        d = np.rint(t)
        r = t - d
        planes.append(d)
    return planes, e


def syrk_digits(planes, e):
    nd = len(planes)
    acc = np.zeros((planes[0].shape[0],) * 2)
    for g in range(nd):
        S = sum(planes[s] @ planes[g - s].T for s in range(g + 1))
        assert np.max(np.abs(S)) < 2.0 ** 31  # the s32 accumulator's range
        acc += np.ldexp(S, -7 * (g + 2))
    return acc * np.ldexp(1.0, e[:, None] + e[None, :])


@pytest.fixture(scope="module")
def hexamer_xt():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    n, naux, nocc = si.n, si.naux, si.nocc
    Vm05, _ = O.s05_calc(si.V)
    B = (Vm05 @ O.unpack_3c(si.I3, n).T).reshape(naux, n, n)
    C = np.linalg.qr(np.random.default_rng(0).normal(size=(n, n)))[0].T[:nocc]
    X = np.einsum("im,qmn->qin", C, B)               # half-transform, (Q, i, nu)
    XT = X.transpose(2, 0, 1).reshape(n, naux * nocc)  # k = Q n_c + i contiguous per row nu
    return XT, C


@pytest.mark.parametrize("nd,tol", [(8, 1e-13), (7, 1e-13)])
def test_digit_syrk_reproduces_fp64_k(hexamer_xt, nd, tol):
    XT, C = hexamer_xt
    K = XT @ XT.T
    planes, e = slice_rows(XT, nd)
    Kd = syrk_digits(planes, e)
    D = C.T @ C
    assert np.max(np.abs(Kd - K)) < tol * np.max(np.abs(K)), np.max(np.abs(Kd - K))
    assert abs(np.sum(D * (Kd - K))) < tol * abs(np.sum(D * K))
    # the split itself: digits in [-64, 64], and after 8 digits at most 2^-57 of the row's scale 2^e left
    assert max(np.max(np.abs(p)) for p in planes) <= 64
    if nd == 8 and np.finfo(np.longdouble).nmant >= 63:  # 56 digit bits: exact in x87 extended precision
        ld = np.longdouble
        recon = sum(p.astype(ld) * ld(2.0) ** (-7 * (s + 1)) for s, p in enumerate(planes))
        recon = recon * np.ldexp(np.ones_like(e, dtype=ld), e)[:, None]
        scale = np.ldexp(np.ones_like(e, dtype=ld), e)
        assert np.all(np.max(np.abs(recon - XT.astype(ld)), axis=1) <= scale * ld(2.0) ** -57)
