"""Adjoint of the Fock build (rijk_grad) — no reference counterpart (the reference only has
finite-difference gradients, src/QM_calc.cpp:142).

Checked three ways:
  - against the oracle's closed-form FP64 gradient (oracle/rijk_oracle.adjoint_reference), to 1e-9;
  - against central finite differences (step 1e-5) of the GPU energy over 64 seeded
    perturbations of orbital coefficients, three-centre integrals and metric entries, to 1e-6;
  - through a torch.autograd.Function (test harness only) with torch.autograd.gradcheck.
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
