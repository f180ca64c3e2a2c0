"""The SCF driver's linear algebra, restated in numpy and checked against the textbook forms on CPU:
- the DIIS step's occupied space from trace-correcting purification (TC2) of F' = X^T F X plus one
  Cholesky-QR subspace step from the previous occupied orbitals (k_scf.cu: purify_occ) gives the
  projector on the n_c lowest eigenvectors, as the reference's diagonalisation does
  (src/SCF.cpp:160-166);
- two Cholesky-QR passes give the Q of the QR factorisation with R's diagonal positive, which is what
  the reference's Gram-Schmidt of the SOSCF rotation I + X - X^T computes
  (src/converger_2_1.cpp:105-123)."""
import numpy as np
import pytest


def tc2_projector(Fp, nocc, max_steps=100):
    """TC2 as the device runs it: P0 = (b I - F')/2b with b the largest absolute row sum; each step
    P <- P^2 or 2P - P^2, whichever trace is nearer n_c; |tr P - tr P^2| is read every 4 steps from
    step 16 on, and two more steps follow once it is below 1e-8.  Returns (P, steps) or (None, steps)."""
    n = Fp.shape[0]
    b = np.max(np.sum(np.abs(Fp), axis=0))
    P = (b * np.eye(n) - Fp) / (2.0 * b)
    left = -1
    for step in range(1, max_steps + 1):
        P2 = P @ P
        t1, t2 = np.trace(P), np.trace(P2)
        P = P2 if abs(t2 - nocc) < abs(2.0 * t1 - t2 - nocc) else 2.0 * P - P2
        if left > 0:
            left -= 1
            if left == 0:
                return P, step
        elif step >= 16 and step % 4 == 0 and abs(t1 - t2) < 1e-8:
            left = 2
    return None, max_steps


def cholesky_qr2(W):
    """Two passes of W^T W = U^T U, W <- W U^-1; returns W and min/max of the first pass's diag(U)."""
    ratio = None
    for p in range(2):
        U = np.linalg.cholesky(W.T @ W).T
        if p == 0:
            d = np.abs(np.diag(U))
            ratio = d.min() / d.max()
        W = np.linalg.solve(U.T, W.T).T
    return W, ratio


def _fock(n, nocc, gap, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    occ = np.sort(rng.uniform(-20.0, -0.5, size=nocc))
    vir = np.sort(rng.uniform(-0.5 + gap, 8.0, size=n - nocc))
    e = np.concatenate([occ, vir])
    return Q @ np.diag(e) @ Q.T, Q[:, :nocc]


@pytest.mark.parametrize("n,nocc,gap", [(60, 12, 0.6), (150, 40, 0.3), (200, 90, 1.0)])
def test_tc2_and_subspace_step_give_the_aufbau_projector(n, nocc, gap):
    Fp, Cocc = _fock(n, nocc, gap, n)
    Pref = Cocc @ Cocc.T
    P, steps = tc2_projector(Fp, nocc)
    assert P is not None, steps
    assert np.max(np.abs(P - Pref)) < 1e-11, np.max(np.abs(P - Pref))
    # the previous step's occupied orbitals: the exact ones rotated a little out of the space
    rng = np.random.default_rng(1)
    V = np.linalg.qr(Cocc + 0.05 * rng.normal(size=Cocc.shape))[0]
    Q, ratio = cholesky_qr2(P @ V)
    assert ratio > 1e-6
    assert np.max(np.abs(Q.T @ Q - np.eye(nocc))) < 1e-13
    assert np.max(np.abs(Q @ Q.T - Pref)) < 1e-11


def test_subspace_step_far_from_the_new_space_is_refused():
    """V (nearly) orthogonal to the new occupied space makes P V rank deficient: the ratio test
    sends the device to the eigensolver."""
    n, nocc = 80, 10
    Fp, Cocc = _fock(n, nocc, 0.5, 7)
    P, _ = tc2_projector(Fp, nocc)
    full = np.linalg.eigh(Fp)[1]
    V = full[:, nocc:2 * nocc].copy()            # virtual orbitals of this F'
    V[:, 0] += 1e-9 * Cocc[:, 0]                 # a whisker of the occupied space
    W = P @ V
    try:
        _, ratio = cholesky_qr2(W)
        refused = not ratio > 1e-6
    except np.linalg.LinAlgError:                # potrf's info > 0 on the device
        refused = True
    assert refused


@pytest.mark.parametrize("nm,nocc,scale", [(50, 10, 0.1), (120, 30, 0.05), (90, 45, 0.02)])
def test_cholesky_qr2_is_the_positive_diagonal_qr_of_the_rotation(nm, nocc, scale):
    rng = np.random.default_rng(nm)
    x = rng.uniform(-scale, scale, size=(nocc, nm - nocc))
    R = np.eye(nm)                               # row-major R[p][q] as k_rot_build writes it
    R[:nocc, nocc:] = x
    R[nocc:, :nocc] = -x.T
    A = R.T                                      # the column-major matrix cuSOLVER / cuBLAS see
    Qh, Rh = np.linalg.qr(A)
    Qh = Qh * np.sign(np.diag(Rh))               # R's diagonal positive: unique
    Qc, _ = cholesky_qr2(A)
    assert np.max(np.abs(Qc - Qh)) < 1e-13
    assert np.max(np.abs(Qc.T @ Qc - np.eye(nm))) < 1e-14
