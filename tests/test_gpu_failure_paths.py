"""Failure paths made on the host, without any GPU fault, and the metrics log.

rijk_selftest_alloc_failure lets the k-th device allocation of a context fail with RIJK_ERR_ALLOC, as an
exhausted cudaMalloc would.  For every k up to the number of allocations a call makes, the call must
return RIJK_ERR_ALLOC or succeed, never anything else, and with allocations allowed again the same
context must give the oracle's results: set-up, FP64 and mixed Fock builds, the SCF and the adjoint.
The JSON-lines metrics log (RIJK_LOG) is checked in a child process, since it is opened once per process.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def hexamer():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    rng = np.random.default_rng(8)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    MO = C.T.copy()
    DM = O.gen_hf_dm(MO, si.n, si.nocc)
    Vm05, _ = O.s05_calc(si.V)
    Jr, Kr = O.dm_to_f_transform_ri(O.unpack_3c(si.I3, si.n), Vm05, DM, MO, si.nocc, si.n)
    return si, DM, MO, Jr, Kr


def _run_with_failures(call, setup=None, max_k=96):
    """call(fb) under an allocation refused after k successes, k = 0, 1, ...: each attempt on a fresh
    context either fails with ERR_ALLOC or succeeds; after a failure the same call on the same context,
    allocations allowed again, must succeed.  Returns the number of allocation points met."""
    for k in range(max_k):
        with rijk.FockBuilder(0) as fb:
            if setup:
                setup(fb)
            fb.selftest_alloc_failure(k)
            try:
                call(fb)
                fb.selftest_alloc_failure(-1)
                return k
            except rijk.RijkError as e:
                assert e.code == rijk.ERR_ALLOC, (k, e.code, fb.last_error())
                assert "injected" in fb.last_error()
            fb.selftest_alloc_failure(-1)
            call(fb)  # the context is usable again
    raise AssertionError("the call kept allocating past %d buffers" % max_k)


def test_allocation_failures_in_setup_and_builds(hexamer):
    si, DM, MO, Jr, Kr = hexamer
    n, nocc = si.n, si.nocc

    def setup(fb):
        fb.set_metric(si.V)
        fb.set_3c(si.I3, n)

    def check(fb, prec, tolK):
        J, K = fb.dm_to_f_transform_ri(DM, MO, nocc, prec)
        assert np.max(np.abs(J - Jr)) < (1e-9 if prec != rijk.PREC_MIXED else 1e-4 * np.max(np.abs(Jr)))
        assert np.max(np.abs(K - Kr)) < tolK

    assert _run_with_failures(setup) >= 2  # the metric factor and the fitted tensor
    assert _run_with_failures(lambda fb: check(fb, rijk.PREC_FP64, 1e-9), setup) >= 5
    assert _run_with_failures(lambda fb: check(fb, rijk.PREC_MIXED, 2e-4), setup) >= 5
    assert _run_with_failures(lambda fb: check(fb, rijk.PREC_FP64_TC, 1e-9), setup) >= 5


def test_allocation_failures_in_scf_and_adjoint(hexamer):
    si = hexamer[0]
    n, nocc = si.n, si.nocc
    Eref = {}

    def setup(fb):
        fb.set_metric(si.V)
        fb.set_3c(si.I3, n)

    def scf(fb):
        E, MO, r = fb.scf(si.H, si.S, nocc, si.Enuc)
        assert r["converged"] == 1
        Eref.setdefault("scf", E)
        assert abs(E - Eref["scf"]) < 1e-10

    def grad(fb):
        E, dC, d3, dV = fb.grad(hexamer[2], nocc, si.H, si.Enuc, want_3c=True, want_metric=True)
        Eref.setdefault("grad", E)
        assert abs(E - Eref["grad"]) < 1e-10

    assert _run_with_failures(scf, setup) >= 10
    assert _run_with_failures(grad, setup) >= 10


def test_metrics_log_lines(tmp_path):
    log = tmp_path / "rijk.jsonl"
    code = r"""
import sys
sys.path.insert(0, %r)
import numpy as np
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster
si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
rng = np.random.default_rng(1)
C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
MO = C.T.copy()
with rijk.FockBuilder(0) as fb:
    fb.set_metric(si.V)
    fb.set_3c(si.I3, si.n)
    fb.dm_to_f_transform_ri(MO[:si.nocc].T @ MO[:si.nocc], MO, si.nocc)
    fb.dm_to_f_transform_ri(MO[:si.nocc].T @ MO[:si.nocc], MO, si.nocc, rijk.PREC_MIXED)
    fb.scf(si.H, si.S, si.nocc, si.Enuc)
""" % ROOT
    env = dict(os.environ, RIJK_LOG=str(log))
    subprocess.run([sys.executable, "-c", code], check=True, env=env, timeout=600)
    lines = [json.loads(x) for x in log.read_text().splitlines()]
    builds = [x for x in lines if x["call"] == "rijk_fock"]
    scfs = [x for x in lines if x["call"] == "rijk_scf"]
    assert [b["precision"] for b in builds] == ["fp64", "mixed"]
    assert all(b["n"] == 144 and b["naux"] == 696 and b["n_c"] == 30 and b["ms"] > 0 and b["flops"] > 0 for b in builds)
    assert len(scfs) == 1 and scfs[0]["converged"] == 1 and scfs[0]["iterations"] > 1
