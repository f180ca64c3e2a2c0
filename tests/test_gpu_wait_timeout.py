"""The bounded device-side wait and its error path, made to run out without any fault.

rijk_selftest_wait_timeout launches one warp that allocates TMEM, waits on an mbarrier nothing
arrives on for a short cycle limit, raises the context's timeout bit, frees the TMEM and returns.
rijk_sync must then report RIJK_ERR_TIMEOUT with a message, and the context must stay usable: the
next Fock builds (FP64 and the tcgen05 mixed form, which allocates TMEM again) match the oracle.
"""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu


def test_wait_runs_out_reports_timeout_and_context_stays_usable():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    n, nocc = si.n, si.nocc
    rng = np.random.default_rng(7)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    DM = O.gen_hf_dm(MO, n, nocc)
    Vm05, _ = O.s05_calc(si.V)
    Jr, Kr = O.dm_to_f_transform_ri(O.unpack_3c(si.I3, n), Vm05, DM, MO, nocc, n)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, n)
        fb.sync()
        with pytest.raises(rijk.RijkError) as e:
            fb.selftest_wait_timeout(10)  # below the accepted range
        assert e.value.code == rijk.ERR_ARG
        for _ in range(2):  # twice: the error word is cleared after it is reported
            fb.selftest_wait_timeout(2_000_000)  # about a millisecond of SM clock
            with pytest.raises(rijk.RijkError) as e:
                fb.sync()
            assert e.value.code == rijk.ERR_TIMEOUT
            assert "wait ran out" in fb.last_error()
            fb.sync()  # reported once, then clear
            J, K = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_FP64)
            assert np.max(np.abs(J - Jr)) < 1e-9 and np.max(np.abs(K - Kr)) < 1e-9
            Jm, Km = fb.dm_to_f_transform_ri(DM, MO, nocc, rijk.PREC_MIXED)
            assert np.max(np.abs(Km - Kr)) < 2e-4
