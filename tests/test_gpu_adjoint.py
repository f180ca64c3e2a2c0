"""Adjoint of the Fock build (rijk_grad) — no reference counterpart (the reference only has
finite-difference gradients, src/QM_calc.cpp:142).

Checked three ways, on C2H4 and on (H2O)16 cc-pVDZ / cc-pVDZ-JKFIT at its converged density:
  - against the oracle's closed-form FP64 gradient (oracle/rijk_oracle.adjoint_reference), to 1e-9;
  - against central finite differences (step 1e-5) of the GPU energy over 64 seeded
    perturbations of orbital coefficients, three-centre integrals and metric entries, to 1e-6;
  - through a torch.autograd.Function (test harness only) with torch.autograd.gradcheck.
The aux-chunked path that recomputes X^Q in tiles equals the stored-tensor path (also on
C40H82 after a mixed SCF).
"""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import Molecule

pytestmark = pytest.mark.gpu
H_FD = 1e-5
TOL_FD = 1e-6


@pytest.fixture(scope="module")
def c2h4():
    mol = Molecule(["C", "C", "H", "H", "H", "H"],
                   [[0, 0, -0.6695], [0, 0, 0.6695], [0, -0.9289, 1.2321], [0, 0.9289, -1.2321],
                    [0, -0.9289, -1.2321], [0, 0.9289, 1.2321]])
    si = ints.SystemIntegrals(mol, "cc-pvdz", "cc-pvdz-ri")
    rng = np.random.default_rng(5)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    return si, C.T.copy()


@pytest.mark.parametrize("form", [rijk.METRIC_INVSQRT, rijk.METRIC_CHOLESKY])
def test_grad_matches_closed_form_oracle(c2h4, form):
    si, MO = c2h4
    M = O.s05_calc(si.V)[0] if form == rijk.METRIC_INVSQRT else O.cholesky_inverse_factor(si.V)
    Er, dCr, d3r, dVr = O.adjoint_reference(si.I3, M, si.H, MO, si.nocc, si.Enuc)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V, form)
        fb.set_3c(si.I3, si.n)
        E, dC, d3, dV = fb.grad(MO, si.nocc, si.H, si.Enuc, want_3c=True, want_metric=True)
    assert abs(E - Er) < 1e-9
    assert np.max(np.abs(dC - dCr)) < 1e-9 * max(1.0, np.max(np.abs(dCr)))
    assert np.max(np.abs(d3 - d3r)) < 1e-9 * max(1.0, np.max(np.abs(d3r)))
    assert np.max(np.abs(dV - dVr)) < 1e-9 * max(1.0, np.max(np.abs(dVr)))


def test_grad_central_finite_differences_64_perturbations(c2h4):
    si, MO = c2h4
    rng = np.random.default_rng(64)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E0, dC, d3, dV = fb.grad(MO, si.nocc, si.H, si.Enuc, want_3c=True, want_metric=True)

        def energy(MO_=MO, I3_=None, V_=None):
            if I3_ is not None or V_ is not None:
                fb.set_metric(si.V if V_ is None else V_)
                fb.set_3c(si.I3 if I3_ is None else I3_, si.n)
            return fb.grad(MO_, si.nocc, si.H, si.Enuc)[0]

        errs = []
        for k in range(32):  # orbital coefficients
            i, m = rng.integers(si.nocc), rng.integers(si.n)
            P, Mn = MO.copy(), MO.copy()
            P[i, m] += H_FD
            Mn[i, m] -= H_FD
            errs.append(abs((energy(P) - energy(Mn)) / (2 * H_FD) - dC[i, m]))
        for k in range(16):  # three-centre integrals (packed pair, aux function)
            pr, q = rng.integers(si.I3.shape[0]), rng.integers(si.naux)
            P, Mn = si.I3.copy(), si.I3.copy()
            P[pr, q] += H_FD
            Mn[pr, q] -= H_FD
            errs.append(abs((energy(I3_=P) - energy(I3_=Mn)) / (2 * H_FD) - d3[pr, q]))
        for k in range(16):  # metric entries, perturbed symmetrically
            a, b = rng.integers(si.naux), rng.integers(si.naux)
            P, Mn = si.V.copy(), si.V.copy()
            for X, sgn in ((P, 1.0), (Mn, -1.0)):
                X[a, b] += sgn * H_FD
                if a != b:
                    X[b, a] += sgn * H_FD
            fd = (energy(V_=P) - energy(V_=Mn)) / (2 * H_FD)
            an = dV[a, b] if a == b else 2 * dV[a, b]
            errs.append(abs(fd - an))
    assert len(errs) == 64
    assert max(errs) < TOL_FD, max(errs)


def test_autograd_function_gradcheck():
    """A torch.autograd.Function around the C ABI (forward: energy; backward: dE/dC)."""
    import torch

    rng = np.random.default_rng(9)
    n, naux, nocc = 20, 30, 4
    A = rng.normal(size=(naux, naux))
    V = A @ A.T / naux + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 0.2
    H = rng.normal(size=(n, n))
    H = H + H.T
    fb = rijk.FockBuilder(0)
    fb.set_metric(V)
    fb.set_3c(I3, n)

    class FockEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, C):
            E, dC, _, _ = fb.grad(C.detach().cpu().numpy(), nocc, H, 0.0)
            ctx.save_for_backward(torch.from_numpy(dC))
            return torch.tensor(E, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gE):
            (dC,) = ctx.saved_tensors
            return gE * dC

    C = torch.from_numpy(rng.normal(size=(nocc, n)) * 0.5).requires_grad_(True)
    try:
        assert torch.autograd.gradcheck(FockEnergy.apply, (C,), eps=1e-6, atol=1e-6, rtol=1e-6)
    finally:
        fb.close()


def _grad_all(fb, MO, si):
    return fb.grad(MO, si.nocc, si.H, si.Enuc, want_3c=True, want_metric=True)


def _rel(a, b):
    return float(np.max(np.abs(a - b))) / max(1.0, float(np.max(np.abs(b))))


def test_grad_recompute_chunks_match_stored_tensor(c2h4):
    """Gamma over aux chunks with X^Q recomputed in tiles equals the one-chunk path that reads the
    stored half-transformed tensor."""
    si, MO = c2h4
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        ref = _grad_all(fb, MO, si)
        assert fb.stats()["grad_qchunk"] == si.naux
        fb.set_grad_chunk(17)
        got = _grad_all(fb, MO, si)
        assert fb.stats()["grad_qchunk"] == 17
    assert abs(got[0] - ref[0]) < 1e-12
    for a, b in zip(got[1:], ref[1:]):
        assert _rel(a, b) < 1e-11


@pytest.fixture(scope="module")
def water16():
    """(H2O)16 cc-pVDZ / cc-pVDZ-JKFIT at its converged FP64 density."""
    from nopt_b200.molecules import water_cluster
    si = ints.SystemIntegrals(water_cluster((4, 2, 2), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E, MO, r = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=si.sad())
    assert r["converged"] == 1
    return si, MO, E


def test_grad_water16_converged_matches_oracle_and_recompute(water16):
    si, MO, Escf = water16
    Vm05, _ = O.s05_calc(si.V)
    Er, dCr, d3r, dVr = O.adjoint_reference(si.I3, Vm05, si.H, MO, si.nocc, si.Enuc)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E, dC, d3, dV = _grad_all(fb, MO, si)
        fb.set_grad_chunk(300)  # Gamma in 7 chunks, X^Q recomputed in tiles
        Ec, dCc, d3c, dVc = _grad_all(fb, MO, si)
    assert abs(E - Escf) < 1e-9 and abs(E - Er) < 1e-9
    # dE/d(P|mu nu) = sum_Q M_QP Gamma^Q and dE/d(P|Q) carry the metric factor V^-1/2, which the GPU
    # (cuSOLVER) and the oracle (LAPACK) form independently; at naux = 1856 its conditioning puts
    # their agreement near 1e-9 relative, hence 1e-8 for these two
    assert _rel(dC, dCr) < 1e-9 and _rel(d3, d3r) < 1e-8 and _rel(dV, dVr) < 1e-8
    # chunked G rows come from GEMMs over other aux chunks (another summation order)
    assert _rel(dCc, dC) < 1e-12 and _rel(d3c, d3) < 1e-11 and _rel(dVc, dV) < 1e-11
    # converged: the occupied-virtual block of 4 F (the SCF's rotation gradient) vanishes
    g = dC @ MO[si.nocc:].T  # 4 F_ai = (4 C_occ F) C_vir^T
    assert float(np.max(np.abs(g))) < 1e-6, float(np.max(np.abs(g)))


def test_grad_water16_central_finite_differences_64(water16):
    """64 seeded perturbations at the converged (H2O)16 density, 32 of orbital coefficients and 32
    of three-centre entries (P|mu nu), central differences with step 1e-5."""
    si, MO, _ = water16
    rng = np.random.default_rng(1664)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E0, dC, d3, dV = _grad_all(fb, MO, si)

        def energy(MO_=MO, I3_=None):
            if I3_ is not None:
                fb.set_3c(I3_, si.n)
            return fb.grad(MO_, si.nocc, si.H, si.Enuc)[0]

        ec, e3 = [], []
        for k in range(32):
            i, m = rng.integers(si.nocc), rng.integers(si.n)
            P, Mn = MO.copy(), MO.copy()
            P[i, m] += H_FD
            Mn[i, m] -= H_FD
            ec.append(abs((energy(P) - energy(Mn)) / (2 * H_FD) - dC[i, m]))
        I3 = si.I3.copy()
        for k in range(32):
            pr, q = rng.integers(I3.shape[0]), rng.integers(si.naux)
            v0 = I3[pr, q]
            I3[pr, q] = v0 + H_FD
            ep = energy(I3_=I3)
            I3[pr, q] = v0 - H_FD
            em = energy(I3_=I3)
            I3[pr, q] = v0
            e3.append(abs((ep - em) / (2 * H_FD) - d3[pr, q]))
    assert len(ec) + len(e3) == 64
    assert max(ec) < TOL_FD and max(e3) < TOL_FD, (max(ec), max(e3))


def test_grad_c40h82_after_mixed_scf_recompute_path():
    """C40H82 cc-pVDZ / JKFIT: mixed SCF switching to FP64 at DIIS error 1e-5, then the adjoint
    with Gamma formed in aux chunks from X^Q recomputed in tiles; it equals the stored-tensor
    path and the orbital gradient vanishes at convergence."""
    from nopt_b200.molecules import alkane
    mol = alkane(40, 0)
    orb = ints.Basis.for_molecule("cc-pvdz", mol)
    aux = ints.Basis.for_molecule("cc-pvdz-jkfit", mol)
    S = ints.overlap(orb)
    H = ints.kinetic(orb) + ints.nuclear(orb, mol)
    nocc, enuc = mol.nelec // 2, mol.nuclear_repulsion()
    guess = ints.sad_guess(mol, "cc-pvdz", "cc-pvdz-jkfit")
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(orb, aux)
        E, MO, r = fb.scf(H, S, nocc, enuc, precision=rijk.PREC_MIXED, guess=guess)
        assert r["converged"] == 1 and r["iterations_mixed"] > 0
        Eg, dC, _, dV = fb.grad(MO, nocc, H, enuc, want_metric=True)
        fb.set_grad_chunk(1024)  # 5 chunks of the 4686 aux functions
        Ec, dCc, _, dVc = fb.grad(MO, nocc, H, enuc, want_metric=True)
        assert fb.stats()["grad_qchunk"] == 1024
    assert abs(Eg - E) < 1e-8 and abs(Ec - Eg) < 1e-10
    assert _rel(dCc, dC) < 1e-12 and _rel(dVc, dV) < 1e-11
    g = dC @ MO[nocc:r["nmo"]].T  # 4 F_ai = (4 C_occ F) C_vir^T
    assert float(np.max(np.abs(g))) < 1e-6, float(np.max(np.abs(g)))


@pytest.mark.parametrize("n,naux,nocc,chunk", [(131, 75, 13, 0), (65, 33, 1, 0), (131, 75, 13, 29), (200, 97, 37, 41)])
def test_grad_ragged_random_matches_closed_form(n, naux, nocc, chunk):
    """Odd n, naux and n_c (8-byte copies and ragged tiles in the DMMA GEMMs, the pair epilogue's edge
    rows), and aux chunks of odd size (contractions of K = 29 or 41 over the chunk)."""
    rng = np.random.default_rng(n + naux)
    A = rng.normal(size=(naux, naux))
    V = A @ A.T / naux + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 0.1
    Hm = rng.normal(size=(n, n))
    H = (Hm + Hm.T) / np.sqrt(n)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    M = O.s05_calc(V)[0]
    Er, dCr, d3r, dVr = O.adjoint_reference(I3, M, H, MO, nocc, 0.7)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(V)
        fb.set_3c(I3, n)
        if chunk:
            fb.set_grad_chunk(chunk)
        E, dC, d3, dV = fb.grad(MO, nocc, H, 0.7, want_3c=True, want_metric=True)
        assert fb.stats()["grad_qchunk"] == (chunk or naux)
    assert abs(E - Er) < 1e-9 * max(1.0, abs(Er))
    assert np.max(np.abs(dC - dCr)) < 1e-9 * max(1.0, np.max(np.abs(dCr)))
    assert np.max(np.abs(d3 - d3r)) < 1e-9 * max(1.0, np.max(np.abs(d3r)))
    assert np.max(np.abs(dV - dVr)) < 1e-9 * max(1.0, np.max(np.abs(dVr)))
