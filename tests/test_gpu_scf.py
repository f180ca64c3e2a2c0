"""RHF on the GPU (rijk_scf): FP64 energies against the reference's logged RI-RHF energies, and
the mixed-precision SCF (mixed Fock builds until the DIIS error falls below 1e-5, FP64 after)
against the FP64 SCF to 1e-8 Eh."""
import json
import os

import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import Molecule, water_cluster

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pins.json")))


def _pin(name):
    p = [q for q in GOLD["pins"] if q["name"] == name][0]
    return ints.SystemIntegrals(Molecule(p["symbols"], p["coords_ang"]), p["basis"], p["aux"]), p


@pytest.mark.parametrize("name", ["c2h4", "c6h8", "guanine"])
def test_gpu_scf_reproduces_reference_energy(name):
    si, p = _pin(name)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E, MO, r = fb.scf(si.H, si.S, si.nocc, si.Enuc)
        Eg, _, rg = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=si.sad())
    assert r["converged"] == 1 and rg["converged"] == 1
    assert abs(Eg - E) < 1e-9
    assert abs(E - p["energy"]) < 2e-9, (E, p["energy"])
    # orbitals are S-orthonormal, one per row as the reference's MO_VEC
    C = MO[:r["nmo"]]
    assert np.max(np.abs(C @ si.S @ C.T - np.eye(r["nmo"]))) < 1e-9


def test_gpu_scf_mixed_then_fp64_matches_fp64():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E64, _, r64 = fb.scf(si.H, si.S, si.nocc, si.Enuc, precision=rijk.PREC_FP64)
        Em, _, rm = fb.scf(si.H, si.S, si.nocc, si.Enuc, precision=rijk.PREC_MIXED)
    assert r64["converged"] and rm["converged"]
    assert rm["iterations_mixed"] > 0
    assert abs(Em - E64) < 1e-8, (Em, E64)
    # the host DIIS loop of the oracle over the same GPU Fock builds agrees too
    Vm05, _ = O.s05_calc(si.V)
    Eo, *_ = O.scf_rhf(si.S, si.H, O.unpack_3c(si.I3, si.n), Vm05, si.nocc, si.Enuc)
    assert abs(E64 - Eo) < 1e-9


def test_gpu_scf_long_alkane_full_size():
    """C40H82 cc-pVDZ / cc-pVDZ-JKFIT (n = 970, naux = 4686, n_c = 161), from the SAD start:
    the core-Hamiltonian start diverges for this chain, the SAD start converges; mixed builds
    followed by FP64 reach the FP64 energy to 1e-8 Eh."""
    from nopt_b200.molecules import alkane
    si = ints.SystemIntegrals(alkane(40, 0), "cc-pvdz", "cc-pvdz-jkfit")
    assert (si.n, si.naux, si.nocc) == (970, 4686, 161)
    guess = si.sad()
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E64, _, r64 = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess)
        Em, _, rm = fb.scf(si.H, si.S, si.nocc, si.Enuc, precision=rijk.PREC_MIXED, guess=guess)
    assert r64["converged"] and rm["converged"]
    assert rm["iterations_mixed"] > 0
    assert abs(Em - E64) < 1e-8
    assert -1562.6 < E64 < -1562.5


def test_gpu_soscf_follows_the_reference_converger():
    """rijk_scf with the SOSCF converger takes the reference's iterates.  From the core start the
    C2H4 trajectory is chaotic (rounding differences grow about tenfold every two iterations past
    iteration ~15; any change in the order of a sum in J, K or the converger's algebra moves the later
    gaps by a few times), so the per-build energies and max |4 F_ai| are compared while rounding still
    dominates: against the oracle's restatement of the reference loop fed by the same J/K (the
    converger alone), to 1e-10 for 15 builds and 1e-9 for 19, and fed by the oracle's own J/K for 10
    builds.  Both runs land on the logged energy."""
    import rijk_oracle as O
    si, p = _pin("c2h4")
    RI = O.unpack_3c(si.I3, si.n)
    Vm05, _ = O.s05_calc(si.V)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E, MO, r = fb.scf(si.H, si.S, si.nocc, si.Enuc, converger=rijk.CONV_SOSCF)
        jk = lambda D, C, nr=si.nocc: fb.dm_to_f_transform_ri(D, C[:nr], nr)
        _, _, hist_same, _ = O.scf_soscf(si.S, si.H, RI, Vm05, si.nocc, si.Enuc, jk=jk, max_iter=19)
    Eo, _, hist, conv = O.scf_soscf(si.S, si.H, RI, Vm05, si.nocc, si.Enuc)
    assert r["converged"] == 1 and conv
    assert abs(E - p["energy"]) < 2e-9, (E, p["energy"])
    gh = r["history"]

    def gap(h, k):
        return (max(abs(gh[i][0] - h[i][0]) for i in range(k)), max(abs(gh[i][1] - h[i][1]) for i in range(k)))

    dE, dg = gap(hist_same, 15)
    assert dE < 1e-10 and dg < 1e-10, (dE, dg)
    dE, dg = gap(hist_same, 19)
    assert dE < 1e-9 and dg < 1e-9, (dE, dg)
    dE, dg = gap(hist, 10)
    assert dE < 1e-9 and dg < 1e-9, (dE, dg)
    C = MO[:r["nmo"]]
    assert np.max(np.abs(C @ si.S @ C.T - np.eye(r["nmo"]))) < 1e-9


def test_gpu_soscf_sad_and_mixed_reach_the_diis_energy():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=2), "cc-pvdz", "cc-pvdz-jkfit")
    guess = si.sad()
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        Ed, _, rd = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess)
        Es, _, rs = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, converger=rijk.CONV_SOSCF)
        Em, _, rm = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, converger=rijk.CONV_SOSCF,
                           precision=rijk.PREC_MIXED)
    assert rd["converged"] and rs["converged"] and rm["converged"]
    assert abs(Es - Ed) < 1e-8 and abs(Em - Ed) < 1e-8, (Ed, Es, Em)
    assert rm["iterations_mixed"] > 0
    assert rs["diis_err"] < 1e-7 or abs(rs["history"][-1][0] - rs["history"][-2][0]) < 1e-10


@pytest.mark.parametrize("start", ["sad", "core"])
def test_gpu_scf_diis_then_soscf(start):
    """RIJK_CONV_DIIS_SOSCF: DIIS over mixed builds, then from the switch on the reference's SOSCF
    step over FP64 builds, started from every orbital of the extrapolated Fock matrix the density
    came from.  It reaches the FP64 DIIS energy to 1e-8 Eh; with FP64 builds throughout it is DIIS."""
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=2), "cc-pvdz", "cc-pvdz-jkfit")
    guess = si.sad() if start == "sad" else None
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        Ed, _, rd = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess)
        E64, _, r64 = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, converger=rijk.CONV_DIIS_SOSCF)
        Eh, MO, rh = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, converger=rijk.CONV_DIIS_SOSCF,
                            precision=rijk.PREC_MIXED)
    assert rd["converged"] and r64["converged"] and rh["converged"]
    assert E64 == Ed and r64["iterations"] == rd["iterations"]
    assert abs(Eh - Ed) < 1e-8, (Ed, Eh)
    h = rh["history"]
    nmix = rh["iterations_mixed"]
    assert nmix > 0 and all(x[2] == 1 for x in h[:nmix]) and all(x[2] == 0 for x in h[nmix:])
    # the SOSCF phase ends on its own test: max |4 F_ai| < 1e-7 or |dE| < 1e-10
    assert h[-1][1] < 1e-7 or abs(h[-1][0] - h[-2][0]) < 1e-10
    C = MO[:rh["nmo"]]
    assert np.max(np.abs(C @ si.S @ C.T - np.eye(rh["nmo"]))) < 1e-9


@pytest.mark.parametrize("precision", [rijk.PREC_FP64, rijk.PREC_MIXED])
def test_gpu_scf_purified_densities_match_eigenvectors(precision):
    """DIIS densities from TC2 purification of X^T F X (the default) against the eigenvector step of
    the reference: the same iterates to rounding, so the same build count and energy to 1e-10 Eh.
    With FP64 builds the per-iteration energies and DIIS errors agree to 1e-9.  A split-BF16 build
    moves by up to its own rounding (about 1e-5 Eh here, against an error of about 1e-3 Eh per
    build) when D changes by one rounding, and the FP64 phase starts from where the mixed one
    ended, so the mixed run is held to its final energy and build counts."""
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=3), "cc-pvdz", "cc-pvdz-jkfit")
    guess = si.sad()
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        Ee, _, re_ = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, precision=precision, purify=False)
        Ep, MO, rp = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, precision=precision)
    assert re_["converged"] and rp["converged"]
    assert re_["purified"] == 0 and rp["purified"] > 0
    assert rp["iterations"] == re_["iterations"] and rp["iterations_mixed"] == re_["iterations_mixed"]
    assert abs(Ep - Ee) < 1e-10, (Ep, Ee)
    if precision == rijk.PREC_FP64:
        for (a, b, _), (c, d, _) in zip(rp["history"], re_["history"]):
            assert abs(a - c) < 1e-9 and abs(b - d) < 1e-9 * max(1.0, abs(d)), (a, c, b, d)
    C = MO[:rp["nmo"]]
    assert np.max(np.abs(C @ si.S @ C.T - np.eye(rp["nmo"]))) < 1e-9


def test_gpu_scf_fp64_phase_on_int8_tensor_cores():
    """fp64_phase=PREC_FP64_TC: after the mixed phase the builds are FP64_TC ones (K from exact int8
    digit products), FP64-accurate, so the run ends on the FP64 energy; other values are refused."""
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=4), "cc-pvdz", "cc-pvdz-jkfit")
    guess = si.sad()
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        E64, _, r64 = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess)
        Et, _, rt = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess, precision=rijk.PREC_MIXED,
                           converger=rijk.CONV_DIIS_SOSCF, fp64_phase=rijk.PREC_FP64_TC)
        with pytest.raises(rijk.RijkError) as e:
            fb.scf(si.H, si.S, si.nocc, si.Enuc, precision=rijk.PREC_MIXED, fp64_phase=rijk.PREC_MIXED)
        assert e.value.code == rijk.ERR_ARG
    assert r64["converged"] and rt["converged"] and rt["iterations_mixed"] > 0
    assert abs(Et - E64) < 1e-9, (Et, E64)


@pytest.mark.parametrize("converger", [rijk.CONV_DIIS, rijk.CONV_SOSCF])
def test_gpu_scf_cartesian_basis_with_d5_projection(converger):
    """The reference's setting: a Cartesian orbital basis (src/inp_par_read.cpp:2550-2552) with the
    orbitals confined to the spherical span (D5 = 1, src/molecule.cpp:4004-4050).  The Fock builds
    run on Cartesian integrals formed on the GPU; rijk_scf with the Cartesian->spherical projector
    reaches the logged C2H4 energy with both convergers, the orbitals lie in the projector's span,
    and without the projector the energy is that of the larger Cartesian space."""
    p = [q for q in GOLD["pins"] if q["name"] == "c2h4"][0]
    mol = Molecule(p["symbols"], p["coords_ang"])
    orb = ints.Basis.for_molecule(p["basis"], mol, pure=False)
    aux = ints.Basis.for_molecule(p["aux"], mol)
    S, H = ints.overlap(orb), ints.kinetic(orb) + ints.nuclear(orb, mol)
    T = ints.d5_projector(orb)
    nocc, Enuc = mol.nelec // 2, mol.nuclear_repulsion()
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(orb, aux)
        E, MO, r = fb.scf(H, S, nocc, Enuc, converger=converger, projector=T)
        E6, _, r6 = fb.scf(H, S, nocc, Enuc, converger=converger)
    assert r["converged"] == 1 and r6["converged"] == 1
    assert r["nmo"] == T.shape[1] and r6["nmo"] == orb.nbf
    assert abs(E - p["energy"]) < 2e-9, (E, p["energy"])
    assert E6 < p["energy"] - 1e-4
    C = MO[:r["nmo"]]
    assert np.max(np.abs(C @ S @ C.T - np.eye(r["nmo"]))) < 1e-9
    # in the span of T: C = Z T^T for Z = C S T (T^T S T)^-1
    Z = C @ S @ T @ np.linalg.inv(T.T @ S @ T)
    assert np.max(np.abs(Z @ T.T - C)) < 1e-9
    assert not np.any(MO[r["nmo"]:])
