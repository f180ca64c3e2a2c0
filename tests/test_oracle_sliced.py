"""The aux-sliced restatement of DM_to_F_transform_RI (the CPU arm at sizes whose full-square
RI_AA does not fit in host memory) against the plain restatement.

Each slice's three-centre integrals come from the integral engine's sub-basis of whole aux
shells; the slices' J and K partials must sum to the J and K of the whole build (src/RI.cpp:115-176).
"""
import numpy as np

import rijk_oracle as O
from nopt_b200 import ints
from nopt_b200.molecules import water_cluster


def _state(n, nocc, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    return O.gen_hf_dm(MO, n, nocc), MO


def test_aux_slice_bounds_cover_the_basis_on_shell_boundaries():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit", ri_integrals=False)
    offs = set(int(x) for x in si.aux.shell_offsets()) | {si.naux}
    for ns in (1, 3, 7, 40):
        b = ints.aux_slice_bounds(si.aux, ns)
        assert b[0][0] == 0 and b[-1][1] == si.naux
        assert all(p1 == q0 for (_, p1), (q0, _) in zip(b, b[1:]))
        assert all(p0 in offs and p1 in offs and p1 > p0 for p0, p1 in b)


def test_sliced_jk_sums_to_the_full_build():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit",
                              layout=ints.LAYOUT_NOPT_FULL)
    n, nocc = si.n, si.nocc
    DM, MO = _state(n, nocc, 3)
    DM = DM + 0.01 * np.random.default_rng(4).normal(size=DM.shape)  # D used as given, not symmetrised
    Vm05, _ = O.s05_calc(si.V)
    Jr, Kr = O.dm_to_f_transform_ri(si.I3, Vm05, DM, MO, nocc, n)
    bounds = ints.aux_slice_bounds(si.aux, 4)
    assert len(bounds) >= 3

    def raw(p0, p1):
        return ints.coulomb_3c_aux_range(si.orb, si.aux, p0, p1)

    np.testing.assert_array_equal(raw(*bounds[1]), si.I3[:, bounds[1][0]:bounds[1][1]])
    RI_CA, RI_Jv = O.sliced_setup(raw, bounds, Vm05, DM, MO, nocc, n)
    J = np.zeros((n, n))
    K = np.zeros((n, n))
    for p0, p1 in bounds:
        Js, Ks, _ = O.sliced_step(raw(p0, p1), p0, p1, RI_CA, RI_Jv, Vm05, DM, MO, nocc, n)
        J += Js
        K += Ks
    assert np.max(np.abs(J - Jr)) < 1e-11 * max(1.0, np.max(np.abs(Jr)))
    assert np.max(np.abs(K - Kr)) < 1e-11 * max(1.0, np.max(np.abs(Kr)))


def test_d5_projector_maps_cartesian_overlap_to_spherical():
    """T^T S_cart T = S_sph, T^T H_cart T = H_sph: the projected Cartesian space is the spherical one."""
    from nopt_b200.molecules import Molecule
    mol = Molecule(["O", "H", "H"], [[0, 0, 0.1173], [0, 0.7572, -0.4692], [0, -0.7572, -0.4692]])
    for name in ("cc-pvdz", "cc-pvtz"):
        cart = ints.Basis.for_molecule(name, mol, pure=False)
        sph = ints.Basis.for_molecule(name, mol, pure=True)
        T = ints.d5_projector(cart)
        assert T.shape == (cart.nbf, sph.nbf)
        Sc, Ss = ints.overlap(cart), ints.overlap(sph)
        np.testing.assert_allclose(T.T @ Sc @ T, Ss, atol=1e-13)
        Hc = ints.kinetic(cart) + ints.nuclear(cart, mol)
        Hs = ints.kinetic(sph) + ints.nuclear(sph, mol)
        np.testing.assert_allclose(T.T @ Hc @ T, Hs, atol=1e-12)
