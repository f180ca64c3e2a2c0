"""Mixed-precision Fock build (tcgen05, split-BF16 3-term, FP32 accumulation) against the oracle.

J is built from the same split-BF16 copy of B (hi + lo, about 17 significant bits) with fp64
accumulation and checked to 1e-4 relative to max|J|; K carries the split-BF16 error of the
three-term products, about 2^-16 relative per product, so K is checked to 2e-4 (absolute, K
entries are O(1)) and
the exchange-energy error tr(D dK) to 1e-4 Eh (split-BF16 keeps about 17 significant bits of
each operand; the SCF switches to the FP64 form for its final iterations).  Cases go from the smallest shapes (one tile row,
n_c = 8) up, so a layout fault shows on the first.
"""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import Molecule, water_cluster

pytestmark = pytest.mark.gpu
TOL_K_MIXED = 2e-4


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
        Jm, Km = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_MIXED)
        Jm2, Km2 = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_MIXED)  # reuses the split copy
    errJ = float(np.max(np.abs(Jm - Jr)))
    assert errJ < 1e-4 * max(1.0, float(np.max(np.abs(Jr)))), errJ
    assert np.array_equal(Jm, Jm2)
    errK = float(np.max(np.abs(Km - Kr)))
    assert errK < TOL_K_MIXED * max(1.0, float(np.max(np.abs(Kr)))), errK
    assert np.array_equal(Km, Km2)
    ex = abs(float(np.sum(DM * (Km - Kr))))
    return errK, ex


def test_mixed_k_c2h4_single_tile_row():
    mol = Molecule(["C", "C", "H", "H", "H", "H"],
                   [[0, 0, -0.6695], [0, 0, 0.6695], [0, -0.9289, 1.2321], [0, 0.9289, -1.2321],
                    [0, -0.9289, -1.2321], [0, 0.9289, 1.2321]])
    si = ints.SystemIntegrals(mol, "cc-pvdz", "cc-pvdz-ri")
    DM, MO = _state(si.n, si.nocc, 1)
    errK, ex = _check(si.V, si.I3, si.n, si.nocc, DM, MO)
    assert ex < 1e-4


def test_mixed_k_water_hexamer():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    DM, MO = _state(si.n, si.nocc, 2)
    errK, ex = _check(si.V, si.I3, si.n, si.nocc, DM, MO)
    assert ex < 1e-4


@pytest.mark.parametrize("n,naux,nocc", [(200, 96, 97), (64, 40, 16), (150, 70, 1), (200, 96, 161), (260, 48, 192),
                                         (1000, 40, 48), (1100, 36, 100), (300, 64, 282), (260, 48, 193),
                                         (1000, 40, 390)])
def test_mixed_k_ragged_random(n, naux, nocc):
    """n >= 1000 takes the CTA-pair SYRK (256 x 256 tiles); n = 1100 ends in a half-filled panel.
    n_c above 192 runs in orbital batches (282 -> 2 x 144, 193 -> 2 x 112, 390 -> 3 x 144)."""
    rng = np.random.default_rng(n)
    A = rng.normal(size=(naux, naux))
    V = A @ A.T / naux + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 0.1
    DM, MO = _state(n, nocc, 3)
    _check(V, I3, n, nocc, DM, MO)


def test_mixed_k_long_contraction_c40h82():
    """C40H82 cc-pVDZ/JKFIT (n = 970, naux = 4686, n_c = 161) at the first SCF density from the SAD
    start.  The CTA-pair SYRK contracts a few hundred 64-wide chunks per split; folding TMEM segments
    of four chunks into fp32 registers keeps tr(D dK) of one build near 1e-3 Eh (a single TMEM
    accumulation over each split gave 1.2e-2 Eh, 12x more)."""
    from nopt_b200.molecules import WORKLOADS
    fac, ob, ab = WORKLOADS["c40h82_dz"]
    si = ints.SystemIntegrals(fac(0), ob, ab, ri_integrals=False)
    n, nocc = si.n, si.nocc
    s_, U_ = np.linalg.eigh(si.S)
    Xo = U_[:, s_ > 1e-10] / np.sqrt(s_[s_ > 1e-10])
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(si.orb, si.aux, rijk.METRIC_INVSQRT)
        D0, R0 = si.sad()
        Jg, Kg = fb.dm_to_f_transform_ri(D0, R0, R0.shape[0])
        _, Cp = np.linalg.eigh(Xo.T @ (si.H + 2 * Jg - Kg) @ Xo)
        MO = (Xo @ Cp).T[:nocc].copy()
        DM = MO.T @ MO
        J64, K64 = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_FP64)
        Jm, Km = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_MIXED)
    dK = Km - K64
    assert float(np.max(np.abs(dK))) < 1.5e-4
    assert abs(float(np.sum(DM * dK))) < 3e-3
    assert float(np.max(np.abs(Jm - J64))) < 1e-4
