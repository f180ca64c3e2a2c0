"""The fitted tensor from three-centre integrals handed over in blocks of orbital rows
(rijk_begin_3c / rijk_add_3c_block), for callers whose (mu nu|P) does not fit in host memory at once.

The blocks fill the same device staging as rijk_set_3c, chunk by chunk of whole 64-row tile rows, so
the fitted tensor, and every build from it, is bit-identical to rijk_set_3c's.  Blocks are cut at rows
that are not tile boundaries, and the large-naux case makes the staging hold one tile row per chunk, so
blocks straddle chunk boundaries.  Call-order errors are refused with the context left consistent.
"""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu


def _state(n, nocc, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    return O.gen_hf_dm(MO, n, nocc), MO


@pytest.mark.parametrize("layout", [rijk.LAYOUT_PACKED, rijk.LAYOUT_NOPT_FULL])
def test_streamed_blocks_equal_set_3c_water_hexamer(layout):
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    n, nocc = si.n, si.nocc
    I3 = si.I3 if layout == rijk.LAYOUT_PACKED else O.unpack_3c(si.I3, n)
    DM, MO = _state(n, nocc, 1)
    bounds = [(0, 7), (7, 70), (70, 71), (71, 128), (128, n)]
    out = {}
    for how in ("whole", "streamed"):
        with rijk.FockBuilder(0) as fb:
            fb.set_metric(si.V)
            if how == "whole":
                fb.set_3c(I3, n, layout)
            else:
                fb.set_3c_streamed(I3, n, bounds, layout)
            out[how] = fb.dm_to_f_transform_ri(DM, MO, nocc)
            out[how + "_mixed"] = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_MIXED)
    for a, b in zip(out["whole"] + out["whole_mixed"], out["streamed"] + out["streamed_mixed"]):
        assert np.array_equal(a, b)
    Vm05, _ = O.s05_calc(si.V)
    Jr, Kr = O.dm_to_f_transform_ri(O.unpack_3c(si.I3, n), Vm05, DM, MO, nocc, n)
    assert np.max(np.abs(out["streamed"][0] - Jr)) < 1e-9 and np.max(np.abs(out["streamed"][1] - Kr)) < 1e-9


def test_streamed_blocks_straddle_staging_chunks_and_aux_slice():
    """n = 300, naux = 7100: the staging holds one 64-row tile row per chunk (5 chunks), and blocks of
    100 rows straddle them; on an aux slice as well."""
    n, naux, nocc = 300, 7100, 23
    rng = np.random.default_rng(2)
    A = rng.normal(size=(naux, 64))
    V = A @ A.T / 64 + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 0.05
    DM, MO = _state(n, nocc, 3)
    bounds = [(0, 100), (100, 200), (200, 300)]
    for q in (None, (1000, 1733)):
        res = []
        for streamed in (False, True):
            with rijk.FockBuilder(0) as fb:
                fb.set_metric(V)
                if q:
                    fb.set_aux_range(*q)
                if streamed:
                    fb.set_3c_streamed(I3, n, bounds)
                else:
                    fb.set_3c(I3, n)
                res.append(fb.dm_to_f_transform_ri(DM, MO, nocc))
        assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_streamed_blocks_refuse_bad_order_and_premature_use():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    n = si.n
    DM, MO = _state(n, si.nocc, 4)
    with rijk.FockBuilder(0) as fb:
        with pytest.raises(rijk.RijkError) as e:
            fb.begin_3c(n, si.naux)  # no metric yet
        assert e.value.code == rijk.ERR_STATE
        fb.set_metric(si.V)
        with pytest.raises(rijk.RijkError) as e:
            fb.add_3c_block(0, 10, si.I3[:55])  # no stream started
        assert e.value.code == rijk.ERR_STATE
        fb.begin_3c(n, si.naux)
        fb.add_3c_block(0, 10, si.I3[:55])
        with pytest.raises(rijk.RijkError) as e:
            fb.add_3c_block(11, 20, si.I3[66:210])  # skips row 10
        assert e.value.code == rijk.ERR_ARG
        with pytest.raises(rijk.RijkError) as e:
            fb.dm_to_f_transform_ri(DM, MO, si.nocc)  # the tensor is not complete
        assert e.value.code == rijk.ERR_STATE
        fb.set_3c(si.I3, n)  # abandons the stream; the whole-tensor set-up works after it
        J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
        with pytest.raises(rijk.RijkError) as e:
            fb.add_3c_block(10, 20, si.I3[55:210])
        assert e.value.code == rijk.ERR_STATE
    Vm05, _ = O.s05_calc(si.V)
    Jr, Kr = O.dm_to_f_transform_ri(O.unpack_3c(si.I3, n), Vm05, DM, MO, si.nocc, n)
    assert np.max(np.abs(J - Jr)) < 1e-9 and np.max(np.abs(K - Kr)) < 1e-9
