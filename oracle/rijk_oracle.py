"""CPU oracle for the RI-JK Fock build — TEST INFRASTRUCTURE ONLY.

It is the oracle the tests compare against.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU baseline leg may import it; the product path (nopt_b200/, librijk.so) never does.

It restates, in numpy (float64 throughout, OpenBLAS dgemm underneath), the reference's
algorithm for the hot path in the reference's own operation order:

  * DM_to_F_transform_RI          src/RI.cpp:115-176
  * CASSCF inactive J/K tail      src/RI.cpp:235-287 (same algorithm, D_core / C_core)
  * MO-basis tensors: calc_2el_MO_INTS_RI src/RI.cpp:178-292, calc_2el_MO_INTS_AAAG_RI :294-346,
    calc_SOSCF_hess_INTS_RI :348-450, RI_data::MO_calc :469-587
  * S05_calc  (metric V^-1/2)     src/matr.cpp:372-401
  * gen_HF_DM (D = sum_i C_i C_i^T, normalised to 1)   src/SCF.cpp:63-73
  * calc_F_AO (F = H + (2J - K) c, mc = 0/1/2)        src/molecule.cpp:4407-4438
  * RHF energy E = tr(F D) + tr(H D) + V_nuc          src/SCF.cpp:134, E_1el_calc src/doCI_matr.cpp:38-47
  * orbital gradient 4 F_ai                           src/converger_2_1.cpp:55-62

Parity is pinned end to end: the RI-RHF energies this oracle reaches with the package's
integral engine are checked against the reference's example logs
(examples/c2h4_2_2/benchmark.log, examples/cis/benchmark.log) in tests/test_oracle_pins.py.
"""
import numpy as np


# ------------------------------------------------------------------ metric ------
def s05_calc(V):
    """V^-1/2 and V^+1/2 as S05_calc (src/matr.cpp:372-401): eigendecomposition, eigenvalues
    <= 0 dropped (the reference prints a warning and leaves the diagonal entry zero)."""
    w, U = np.linalg.eigh(V)
    m = np.zeros_like(w)
    p = np.zeros_like(w)
    pos = w > 0.0
    p[pos] = np.sqrt(w[pos])
    m[pos] = 1.0 / p[pos]
    Vm05 = (U * m) @ U.T
    Vp05 = (U * p) @ U.T
    return Vm05, Vp05


def cholesky_inverse_factor(V):
    """L^-1 with V = L L^T (the Cholesky form of the metric; J and K agree with the V^-1/2
    form in exact arithmetic since L^-T L^-1 = V^-1 = V^-1/2 V^-1/2)."""
    L = np.linalg.cholesky(V)
    return np.linalg.solve(L, np.eye(V.shape[0]))


# --------------------------------------------------------------- RI tensors ------
def unpack_3c(I3_packed, n):
    """Packed (mu>=nu) three-centre array [(mu(mu+1)/2+nu), P] -> NOPT's RI_AA layout
    [(mu*n+nu), P] (src/RI.cpp:69-71, src/libint_link.cpp:2320)."""
    naux = I3_packed.shape[1]
    full = np.empty((n, n, naux))
    iu = np.tril_indices(n)
    full[iu[0], iu[1]] = I3_packed
    full[iu[1], iu[0]] = I3_packed
    return full.reshape(n * n, naux)


def dm_to_f_transform_ri(RI_AA, Vm05, DM, MO, n_c, n_ao):
    """J, K exactly as DM_to_F_transform_RI (src/RI.cpp:115-176).

    RI_AA: (n*n, naux) raw (mu nu|P), aux fastest.  Vm05: V^-1/2.  DM: n x n row-major
    (not symmetrised).  MO: rows are orbitals (n_c rows used).  Returns (J, K), K unscaled.
    """
    naux = RI_AA.shape[1]
    RI_J = DM.reshape(1, n_ao * n_ao) @ RI_AA            # :122-126  1 x naux
    RI_J2 = Vm05 @ RI_J.reshape(naux, 1)                  # :128-132
    RI_J = Vm05 @ RI_J2                                   # :134-138
    J = (RI_AA @ RI_J).reshape(n_ao, n_ao)                # :140-144
    MOc = np.ascontiguousarray(MO[:n_c])
    RI_CA = MOc @ RI_AA.reshape(n_ao, n_ao * naux)        # :146-150  (i, nu, P)
    RI_CA2 = RI_CA.reshape(n_c * n_ao, naux) @ Vm05       # :152-156
    T = RI_CA2.reshape(n_c, n_ao, naux).transpose(1, 0, 2).reshape(n_ao, n_c * naux)  # :158-164
    K = T @ T.T                                           # :167-171
    return J, K


# --------------------------------------------------- aux-sliced restatement ------
# DM_to_F_transform_RI (src/RI.cpp:115-176) with the raw three-centre tensor held one slice of aux
# functions at a time, for sizes whose full-square RI_AA (n^2 naux doubles) exceeds host memory.
# The reference's stages and their order are kept; each is cut along the aux index:
#   set-up (once per density):  RI_J = vec(D)^T RI_AA and RI_CA = MO RI_AA, slice by slice
#                               (:122-126, :146-150), then RI_J <- V^-1/2 V^-1/2 RI_J (:128-138);
#   one slice [p0, p1):         the slice's RI_J and RI_CA columns again (the same products),
#                               RI_CA2 columns Q in the slice = RI_CA V^-1/2[:, Q] (:152-156),
#                               their transpose (:158-164), K_s = T T^T (:167-171) and
#                               J_s = RI_AA[:, slice] RI_J[slice] (:140-144).
# Every product of a full build belongs to exactly one slice, so a slice carries (p1 - p0) / naux
# of the build's arithmetic, and J = sum_s J_s, K = sum_s K_s over slices that cover [0, naux).

def sliced_setup(raw_slice, bounds, Vm05, DM, MO, n_c, n_ao):
    """RI_CA (n_c, n_ao, naux) and the fitted Coulomb coefficients V^-1/2 V^-1/2 RI_J from every
    slice.  raw_slice(p0, p1) returns RI_AA[:, p0:p1] as an (n_ao^2, p1 - p0) array."""
    naux = Vm05.shape[0]
    MOc = np.ascontiguousarray(MO[:n_c])
    RI_CA = np.empty((n_c, n_ao, naux))
    RI_J = np.empty(naux)
    for p0, p1 in bounds:
        A = raw_slice(p0, p1)
        RI_J[p0:p1] = DM.reshape(1, n_ao * n_ao) @ A                              # :122-126
        RI_CA[:, :, p0:p1] = (MOc @ A.reshape(n_ao, n_ao * (p1 - p0))).reshape(n_c, n_ao, p1 - p0)  # :146-150
    RI_Jv = Vm05 @ (Vm05 @ RI_J)                                                  # :128-138
    return RI_CA, RI_Jv


def sliced_step(A, p0, p1, RI_CA, RI_Jv, Vm05, DM, MO, n_c, n_ao):
    """The share of aux slice [p0, p1) of one build; A = RI_AA[:, p0:p1].  Returns (J_s, K_s):
    J_s sums the raw aux functions P of the slice, K_s the fitted aux functions Q of the slice."""
    s = p1 - p0
    naux = Vm05.shape[0]
    MOc = np.ascontiguousarray(MO[:n_c])
    RI_J = DM.reshape(1, n_ao * n_ao) @ A                                         # :122-126
    RI_CA[:, :, p0:p1] = (MOc @ A.reshape(n_ao, n_ao * s)).reshape(n_c, n_ao, s)  # :146-150
    RI_CA2 = RI_CA.reshape(n_c * n_ao, naux) @ Vm05[:, p0:p1]                     # :152-156
    T = RI_CA2.reshape(n_c, n_ao, s).transpose(1, 0, 2).reshape(n_ao, n_c * s)    # :158-164
    K = T @ T.T                                                                   # :167-171
    J = (A @ RI_Jv[p0:p1]).reshape(n_ao, n_ao)                                    # :140-144
    return J, K, RI_J


def calc_2el_mo_ints_ri(RI_AA, Vm05, n_ao, DM_D, MO_VEC, MO_VEC1, MO_VEC2, n_c, n_a, t=0):
    """calc_2el_MO_INTS_RI (src/RI.cpp:178-292): active integrals MO_INTS (n_a^2 x n_a^2) in the
    reference's (b a | d c) order, then the core J, K of DM_D / MO_VEC (None when DM_D is None)."""
    naux = RI_AA.shape[1]
    C1 = MO_VEC1.T if t else MO_VEC1                                  # n_a x n_ao
    C2 = MO_VEC2.T if t else MO_VEC2
    RI_aA = C1 @ RI_AA.reshape(n_ao, n_ao * naux)                     # :197-201  (a, nu, P)
    RI_aA2 = RI_aA.reshape(n_a * n_ao, naux) @ Vm05                  # :203-207
    T = RI_aA2.reshape(n_a, n_ao, naux).transpose(1, 0, 2)            # :209-215  (nu, a, Q)
    RI_aa = C2 @ T.reshape(n_ao, n_a * naux)                          # :217-221  (b, a, Q)
    R = RI_aa.reshape(n_a * n_a, naux)
    MO_INTS = R @ R.T                                                 # :223-227
    if DM_D is None:
        return MO_INTS, None, None
    J, K = dm_to_f_transform_ri(RI_AA, Vm05, DM_D, MO_VEC, n_c, n_ao)  # :235-287
    return MO_INTS, J, K


def _half(RI_AA, Vm05, C, n_ao):
    """(tA|K) -> the reference's transposed (A t|K) buffer: T[b][(a, k)] = sum_mu C[a,mu] (mu b|P) Vm05[P,k]
    (the dgemm pair and OpenMP transpose repeated at src/RI.cpp:305-323, :361-379, :480-498)."""
    naux = RI_AA.shape[1]
    na = C.shape[0]
    RI_aA = C @ RI_AA.reshape(n_ao, n_ao * naux)
    RI_aA2 = RI_aA.reshape(na * n_ao, naux) @ Vm05
    T = RI_aA2.reshape(na, n_ao, naux).transpose(1, 0, 2).reshape(n_ao, na * naux)
    return RI_aA2, T


def mo_calc(RI_AA, Vm05, VEC, n_cor, n_act, n_vac, n_ao):
    """RI_data::MO_calc (src/RI.cpp:469-587): the CC, VC, AA, CA, VA tensors, each [(p n2 + a)][k]."""
    naux = RI_AA.shape[1]
    COR, ACT = VEC[:n_cor], VEC[n_cor:n_cor + n_act]
    VAC = VEC[n_cor + n_act:n_cor + n_act + n_vac]
    _, T = _half(RI_AA, Vm05, COR, n_ao)                              # :480-498
    CC = (COR @ T).reshape(n_cor * n_cor, naux)                       # :500-506
    VC = (VAC @ T).reshape(n_vac * n_cor, naux)                       # :508-514
    _, T = _half(RI_AA, Vm05, ACT, n_ao)                              # :521-539
    AA = (ACT @ T).reshape(n_act * n_act, naux)                       # :541-547
    CA = (COR @ T).reshape(n_cor * n_act, naux)                       # :548-554
    VA = (VAC @ T).reshape(n_vac * n_act, naux)                       # :555-561
    return CC, VC, AA, CA, VA


def mo_ints_aaag(RI_AA, Vm05, MO_VEC, n_c, n_a, n_ao):
    """calc_2el_MO_INTS_AAAG_RI (src/RI.cpp:294-346): MO_INTS[(t u v)][x] = (tu|vx), x < n_ao."""
    naux = RI_AA.shape[1]
    CA = MO_VEC[n_c:n_c + n_a]
    RI_aA2, T = _half(RI_AA, Vm05, CA, n_ao)                          # :305-323
    RI_aa = (CA @ T).reshape(n_a * n_a, naux)                         # :325-330
    aaag2 = RI_aa @ RI_aA2.T                                          # :332-337  (tu | v A)
    return aaag2.reshape(n_a ** 3, n_ao) @ MO_VEC[:n_ao].T            # :338-343


def soscf_hess_ints(RI_AA, Vm05, MO_VEC, n_c, n_a, n_ao):
    """calc_SOSCF_hess_INTS_RI (src/RI.cpp:348-450): aa_J[p][(t u)] = (pp|tu), aa_K[p][(t u)] = (pt|pu)."""
    naux = RI_AA.shape[1]
    C = MO_VEC[:n_ao]
    CA = MO_VEC[n_c:n_c + n_a]
    _, T = _half(RI_AA, Vm05, CA, n_ao)                               # :361-379
    RI_aa = (CA @ T).reshape(n_a * n_a, naux)                         # :381-386
    TMP = np.einsum("pi,pj->pij", C, C).reshape(n_ao, n_ao * n_ao)    # :389-393
    RI_pp = TMP @ RI_AA                                               # :394-399
    RI_pp_2 = RI_pp @ Vm05.T                                          # :404-407
    aa_J = RI_pp_2 @ RI_aa.T                                          # :410-413
    RI_aA2 = (C @ T).reshape(n_ao, n_a, naux)                         # :416-421  (p, a, k)
    aa_K = np.einsum("pik,pjk->pij", RI_aA2, RI_aA2).reshape(n_ao, n_a * n_a)  # :423-428
    return aa_J, aa_K


def gen_hf_dm(MO, n, n_el):
    """D[i,j] = sum_k MO[k,i] MO[k,j] over k < n_el (src/SCF.cpp:63-73)."""
    C = MO[:n_el]
    return C.T @ C


def e_1el(X, DM):
    """E_1el_calc (src/doCI_matr.cpp:38-47): sum_ij DM[i + n j] X[i n + j] = sum(DM^T * X)."""
    return float(np.sum(DM.T * X))


def calc_f_ao(H, J, K, c=1.0, mc=0):
    """calc_F_AO (src/molecule.cpp:4418-4430)."""
    if mc in (0, 2):
        return H + (2.0 * J - K) * c
    return H + (J - K) * (2.0 * c)


def rhf_energy(F, H, DM, Enuc):
    """E = tr(F D) + tr(H D) + V_nuc  (src/SCF.cpp:134)."""
    return e_1el(F, DM) + e_1el(H, DM) + Enuc


def orbital_gradient_max(F, MO, n_occ):
    """max |4 F^MO_ai| (src/converger_2_1.cpp:55-62), F^MO = C F C^T (src/SCF.cpp:136-137)."""
    Fmo = MO @ F @ MO.T
    return float(np.max(np.abs(4.0 * Fmo[n_occ:, :n_occ]))) if Fmo.shape[0] > n_occ else 0.0


# ------------------------------------------------------------ factored form ------
def b_tensor(I3_packed, M):
    """B^Q_{mu nu} = sum_P M_QP (P|mu nu) on the packed pair list: (npair, naux) -> (naux, npair)."""
    return M @ I3_packed.T


def jk_from_b(Bp, n, DM, MO, n_c):
    """J, K from a packed fitted tensor B (naux x npair, mu>=nu).  Same quantities as
    dm_to_f_transform_ri with B = V^-1/2 (P|mu nu); used at sizes where the full-square
    RI_AA of the reference does not fit in host memory."""
    naux = Bp.shape[0]
    il = np.tril_indices(n)
    Dsym = DM + DM.T
    Dsym[np.diag_indices(n)] *= 0.5
    w = Bp @ Dsym[il]
    Jp = Bp.T @ w
    J = np.zeros((n, n))
    J[il] = Jp
    J[il[1], il[0]] = Jp
    C = np.ascontiguousarray(MO[:n_c])
    K = np.zeros((n, n))
    full = np.zeros((n, n))
    for q in range(naux):
        full[il] = Bp[q]
        full[il[1], il[0]] = Bp[q]
        X = C @ full
        K += X.T @ X
    return J, K


# ----------------------------------------------------------------- adjoint ------
def energy_from_mo(RI_AA, Vm05, H, MO, n_c, Enuc):
    """E(C) of the reference's RHF (src/SCF.cpp:134) with D = C^T C from the first n_c rows."""
    n = H.shape[0]
    DM = gen_hf_dm(MO, n, n_c)
    J, K = dm_to_f_transform_ri(RI_AA, Vm05, DM, MO, n_c, n)
    F = calc_f_ao(H, J, K)
    return rhf_energy(F, H, DM, Enuc), F


def adjoint_reference(I3_packed, M, H, MO, n_c, Enuc):
    """E and its derivatives from the closed forms, for a metric factor M with M^T M = V^-1:
    E = 2 tr(HD) + 2 sum_Q w_Q^2 - sum_Q |Y^Q|^2 + Enuc, w_Q = <B^Q, D>, Y^Q = C B^Q C^T;
    dE/dC = 4 C F; Gamma^Q = 4 w_Q D - 2 C^T Y^Q C; dE/d(P|mu nu) = sum_Q M_QP Gamma^Q
    (x2 for a packed off-diagonal pair); dE/d(P|Q) = -M^T G M, G = 1/2 <Gamma^Q, B^R>."""
    n = H.shape[0]
    naux = M.shape[0]
    Bf = np.zeros((naux, n, n))
    Bp = M @ I3_packed.T
    il = np.tril_indices(n)
    Bf[:, il[0], il[1]] = Bp
    Bf[:, il[1], il[0]] = Bp
    Bm = Bf.reshape(naux, n * n)
    C = MO[:n_c]
    D = C.T @ C
    w = Bm @ D.reshape(-1)                                   # <B^Q, D>
    X = np.matmul(C[None], Bf)                               # X^Q = C B^Q        (naux, n_c, n)
    Y = np.matmul(X, C.T[None])                              # Y^Q = C B^Q C^T    (naux, n_c, n_c)
    J = (w @ Bm).reshape(n, n)
    Xm = X.reshape(naux * n_c, n)
    K = Xm.T @ Xm                                            # sum_Q X^Q^T X^Q
    F = H + 2 * J - K
    E = 2 * np.sum(H * D) + 2 * np.sum(w * w) - np.sum(Y * Y) + Enuc
    dC = 4 * C @ F
    Gam = 4 * w[:, None, None] * D[None] - 2 * np.matmul(np.matmul(C.T[None], Y), C[None])
    Gm = Gam.reshape(naux, n * n)
    d3f = (M.T @ Gm).reshape(naux, n, n)                     # sum_Q M_QP Gamma^Q
    fac = np.where(il[0] == il[1], 1.0, 2.0)
    d3 = (d3f[:, il[0], il[1]] * fac).T.copy()
    G = 0.5 * Gm @ Bm.T
    dV = -M.T @ G @ M
    return E, dC, d3, dV


# --------------------------------------------------------------------- SCF ------
def scf_rhf(S, H, RI_AA, Vm05, n_occ, Enuc, conv_dm=1e-10, max_iter=100, diis_n=8, jk=None, guess=None,
            projector=None):
    """Restricted HF with DIIS on F D S - S D F, using the reference's J/K, F and E
    conventions.  Returns (E, MO, DM, F, iterations).  `jk(DM, MO, n_rows) -> (J, K)` overrides
    the Fock build (default: dm_to_f_transform_ri on RI_AA/Vm05); `guess = (D0, R)` starts from
    the Fock matrix of D0 = R^T R instead of the core Hamiltonian.  `projector` T (n x n_proj)
    confines the orbitals to its columns' span: every diagonalisation is the generalised problem
    (T^T F T) V = (T^T S T) V e with MO = V^T T^T, as diag_X_AO_in_MO with D5 = 1
    (src/molecule.cpp:4004-4050)."""
    n = S.shape[0]
    T = np.eye(n) if projector is None else projector
    s, U = np.linalg.eigh(T.T @ S @ T)
    keep = s > 1e-10
    X = T @ (U[:, keep] / np.sqrt(s[keep]))
    if jk is None:
        jk = lambda D, MO, nr=n_occ: dm_to_f_transform_ri(RI_AA, Vm05, D, MO, nr, n)

    def diag(F):
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        return (X @ Cp).T  # rows are orbitals

    if guess is not None:
        J0, K0 = jk(guess[0], guess[1], guess[1].shape[0])
        MO = diag(calc_f_ao(H, J0, K0))
    else:
        MO = diag(H)
    DM = gen_hf_dm(MO, n, n_occ)
    focks, errs = [], []
    E = 0.0
    for it in range(1, max_iter + 1):
        J, K = jk(DM, MO)
        F = calc_f_ao(H, J, K)
        E = rhf_energy(F, H, DM, Enuc)
        err = X.T @ (F @ DM @ S - S @ DM @ F) @ X
        focks.append(F)
        errs.append(err)
        if len(focks) > diis_n:
            focks.pop(0)
            errs.pop(0)
        m = len(focks)
        Bm = -np.ones((m + 1, m + 1))
        Bm[m, m] = 0.0
        for i in range(m):
            for j in range(m):
                Bm[i, j] = np.sum(errs[i] * errs[j])
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        try:
            coef = np.linalg.solve(Bm, rhs)[:m]
        except np.linalg.LinAlgError:
            coef = np.zeros(m)
            coef[-1] = 1.0
        Fd = sum(c * f for c, f in zip(coef, focks))
        MO = diag(Fd)
        DMn = gen_hf_dm(MO, n, n_occ)
        rms = float(np.sqrt(np.mean((DMn - DM) ** 2)))
        DM = DMn
        if rms < conv_dm:
            J, K = jk(DM, MO)
            F = calc_f_ao(H, J, K)
            E = rhf_energy(F, H, DM, Enuc)
            return E, MO, DM, F, it
    return E, MO, DM, F, max_iter


# ----------------------------------------------------- SOSCF converger ------
def lbfgs_step(st, g, h, x_max=0.1):
    """l_bfgs_engine::step as the reference builds it (LBFGS_RETURN_STEP, LBFGS_CALC_HESS with a
    no-op Hessian callback; src/l-bfgs_2_1.cpp:30-126, Makefile DEFINITIONS): two-loop recursion
    over the accepted curvature pairs with the diagonal Hessian h (not inverted), step scaled so
    that no angle exceeds x_max.  `st` holds the engine state between calls."""
    m = st["m"]
    if st["step"] == 0:
        st["pairs"] = 0
    if m > 0 and st["step"] > 0:                                        # :44-61
        y = g - st["gprev"]
        sy, yy = float(st["last"] @ y), float(y @ y)
        if sy > np.finfo(float).eps * yy:
            k = st["pairs"] % m
            st["Y"][k], st["S"][k], st["rho"][k] = y, st["last"].copy(), 1.0 / sy
            st["pairs"] += 1
    P = st["pairs"]
    vec = min(P, m)
    q = g.copy()
    st["gprev"] = g.copy()
    alpha = np.zeros(vec)
    for i in range(vec):                                                # :75-82
        k = (P - i - 1) % m
        alpha[i] = st["rho"][k] * float(st["S"][k] @ q)
        q -= alpha[i] * st["Y"][k]
    s = q / h                                                           # :85
    for i in range(vec):                                                # :87-95
        k = (P - vec + i) % m
        beta = st["rho"][k] * float(st["Y"][k] @ s)
        s += (alpha[vec - i - 1] - beta) * st["S"][k]
    smax = float(np.max(np.abs(s))) if s.size else 0.0
    zoom = -x_max / smax if smax > x_max else -1.0                      # :96-102
    x = s * zoom                                                        # :105-107
    st["last"] = x.copy()                                               # :118-121
    st["step"] += 1
    return x


def gram_schmidt_rows(R):
    """ortogonalization (src/matr.cpp:1001-1016): rows made orthonormal in order."""
    R = R.copy()
    for i in range(R.shape[0]):
        R[i] /= np.sqrt(R[i] @ R[i])
        R[i + 1:] -= np.outer(R[i + 1:] @ R[i], R[i])
    return R


def scf_soscf(S, H, RI_AA, Vm05, n_occ, Enuc, e_conv=1e-10, g_conv=1e-7, max_iter=100, jk=None, guess=None,
              lindep=1e-10):
    """The reference's RHF loop (src/SCF.cpp:125-174) with its SOSCF engine
    (src/converger_2_1.cpp:55-125): g_ia = 4 F_ai and H_ia = 4 (e_a - e_i) in the MO basis,
    L-BFGS step, orbitals rotated by the Gram-Schmidt-orthonormalised I + X - X^T; the first
    iteration diagonalises instead unless a guess was given; converged on max|g| < g_conv or
    |dE| < e_conv.  Canonical orthogonalisation X and the starts are those of scf_rhf.
    Returns (E, MO, history [(E, max|g|) per Fock build], converged)."""
    n = S.shape[0]
    s, U = np.linalg.eigh(S)
    keep = s >= lindep
    X = U[:, keep] / np.sqrt(s[keep])
    if jk is None:
        jk = lambda D, MO, nr=n_occ: dm_to_f_transform_ri(RI_AA, Vm05, D, MO, nr, n)

    def diag(F):
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        return (X @ Cp).T

    if guess is not None:
        J0, K0 = jk(guess[0], guess[1], guess[1].shape[0])
        MO = diag(calc_f_ao(H, J0, K0))
    else:
        MO = diag(H)
    nm = MO.shape[0]
    nv = nm - n_occ
    m = min(nm, 20, max_iter)
    st = {"m": m, "step": 0, "pairs": 0, "gprev": np.zeros(n_occ * nv), "last": np.zeros(n_occ * nv),
          "Y": np.zeros((m, n_occ * nv)), "S": np.zeros((m, n_occ * nv)), "rho": np.zeros(m)}
    E_old, hist, converged = 1e15, [], False
    for it in range(max_iter):
        DM = gen_hf_dm(MO, n, n_occ)
        J, K = jk(DM, MO)
        F = calc_f_ao(H, J, K)
        E = rhf_energy(F, H, DM, Enuc)
        Fmo = MO @ F @ MO.T
        g = 4.0 * Fmo[n_occ:, :n_occ].T.reshape(-1)                      # orb_grad_calc
        e = np.diag(Fmo)
        h = 4.0 * (e[None, n_occ:] - e[:n_occ, None]).reshape(-1)       # orb_hess_calc
        gmax = float(np.max(np.abs(g))) if g.size else 0.0
        hist.append((E, gmax))
        if gmax < g_conv or abs(E - E_old) < e_conv:
            converged = True
            break
        if it == 0 and guess is None:
            MO = diag(F)
            E_old = E
            continue
        x = lbfgs_step(st, g, h)
        R = np.eye(nm)
        R[:n_occ, n_occ:] = x.reshape(n_occ, nv)
        R[n_occ:, :n_occ] = -x.reshape(n_occ, nv).T
        MO = gram_schmidt_rows(R) @ MO
        E_old = E
    return E, MO, hist, converged
