"""The fitted tensor on disk (rijk_save / rijk_load): a loaded context gives bit-identical J, K
and gradients; damaged, truncated or foreign files are refused with RIJK_ERR_ARG and leave the
context as it was."""
import os

import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=4), "cc-pvdz", "cc-pvdz-jkfit")
    rng = np.random.default_rng(9)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    MO = C.T.copy()
    return si, MO, O.gen_hf_dm(MO, si.n, si.nocc)


def test_round_trip_is_bit_identical(system, tmp_path):
    si, MO, DM = system
    path = str(tmp_path / "b.rijk")
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(si.orb, si.aux, rijk.METRIC_CHOLESKY)
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
        E, dC, d3, dV = fb.grad(MO, si.nocc, si.H, si.Enuc, want_3c=True, want_metric=True)
        fb.save(path)
    assert os.path.getsize(path) > 8 * si.naux * si.naux
    with rijk.FockBuilder(0) as fb:
        fb.load(path)
        assert (fb.n, fb.naux) == (si.n, si.naux)
        J2, K2 = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
        E2, dC2, d32, dV2 = fb.grad(MO, si.nocc, si.H, si.Enuc, want_3c=True, want_metric=True)
        Jm, Km = fb.dm_to_f_transform_ri(DM, MO, si.nocc, precision=rijk.PREC_MIXED)
    assert np.array_equal(J, J2) and np.array_equal(K, K2)
    assert E == E2 and np.array_equal(dC, dC2) and np.array_equal(d3, d32) and np.array_equal(dV, dV2)
    assert np.max(np.abs(Km - K)) < 2e-4


def test_aux_slice_round_trip(system, tmp_path):
    si, MO, DM = system
    path = str(tmp_path / "slice.rijk")
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(si.orb, si.aux, rijk.METRIC_INVSQRT, 50, 400)
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
        fb.save(path)
    with rijk.FockBuilder(0) as fb:
        fb.load(path)
        J2, K2 = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
    assert np.array_equal(J, J2) and np.array_equal(K, K2)


def test_damaged_files_are_refused(system, tmp_path):
    si, MO, DM = system
    good = str(tmp_path / "good.rijk")
    with rijk.FockBuilder(0) as fb:
        fb.set_basis(si.orb, si.aux)
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
        fb.save(good)
        data = open(good, "rb").read()
        flipped = bytearray(data)
        flipped[len(data) // 2] ^= 0x40
        cases = {"flip": bytes(flipped), "short": data[:len(data) - 4096], "foreign": b"not a tensor" * 100}
        for name, blob in cases.items():
            p = str(tmp_path / (name + ".rijk"))
            open(p, "wb").write(blob)
            with pytest.raises(rijk.RijkError) as e:
                fb.load(p)
            assert e.value.code == rijk.ERR_ARG, name
            J2, K2 = fb.dm_to_f_transform_ri(DM, MO, si.nocc)  # context unchanged
            assert np.array_equal(J, J2) and np.array_equal(K, K2), name
        with pytest.raises(rijk.RijkError):
            fb.load(str(tmp_path / "missing.rijk"))
