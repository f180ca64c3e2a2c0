"""The allocation-free Coulomb entry point, rijk_coulomb_noalloc.

It is for callers that cannot let the library call cudaMalloc while their iterations run
(a program that hands all of its GPU memory to its own pool, or one that must not add an
allocation inside its loop).  Its working space is a fixed 32 MiB device array inside the
library, so this checks:
  - J matches the oracle's restatement of the reference's J and the ordinary entry point
    (rijk_fock_device) on two calls in a row with different densities (the shared scratch
    keeps the previous call's contents);
  - the calls leave the device's free memory unchanged; they run before any ordinary build, so
    no buffer of the ordinary path can hide an allocation;
  - too large a system is refused with a clear error.
The file sorts last so that a run stopping at the first failure has already run the rest.
"""
import ctypes

import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu
TOL_JK = 1e-9


def _noalloc(L):
    f = L.rijk_coulomb_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _state(n, nocc, seed):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, n)))
    MO = C.T.copy()
    return O.gen_hf_dm(MO, n, nocc), MO


def test_noalloc_coulomb_matches_oracle_and_fock_device_on_two_calls():
    import torch
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    n, nocc = si.n, si.nocc
    dev = torch.device("cuda", 0)
    f = _noalloc(rijk.lib())
    Vm05, _ = O.s05_calc(si.V)
    RI = O.unpack_3c(si.I3, n)
    states = [_state(n, nocc, seed) for seed in (11, 12)]
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, n)
        dDs = [torch.from_numpy(DM).to(dev) for DM, _ in states]
        dJs = [torch.full((n, n), float("nan"), dtype=torch.float64, device=dev) for _ in states]
        torch.cuda.synchronize(dev)
        free0 = torch.cuda.mem_get_info(dev)[0]
        for call, ((DM, MO), dD, dJ) in enumerate(zip(states, dDs, dJs)):
            rc = f(fb._h, dD.data_ptr(), dJ.data_ptr())
            assert rc == rijk.OK, fb.last_error()
            torch.cuda.synchronize(dev)
            assert torch.cuda.mem_get_info(dev)[0] == free0, "device memory changed across rijk_coulomb_noalloc"
            Jr, _ = O.dm_to_f_transform_ri(RI, Vm05, DM, MO, nocc, n)
            err = float(np.max(np.abs(dJ.cpu().numpy() - Jr)))
            assert err < TOL_JK, ("oracle", call, err)
        # the ordinary entry point on the same densities, after the allocation-free calls
        for call, ((DM, MO), dD, dJ) in enumerate(zip(states, dDs, dJs)):
            dMO = torch.from_numpy(MO[:nocc].copy()).to(dev)
            dJ_ref = torch.empty((n, n), dtype=torch.float64, device=dev)
            dK_ref = torch.empty((n, n), dtype=torch.float64, device=dev)
            fb.fock_device(dD.data_ptr(), dMO.data_ptr(), nocc, dJ_ref.data_ptr(), dK_ref.data_ptr())
            torch.cuda.synchronize(dev)
            err = float((dJ - dJ_ref).abs().max())
            assert err < TOL_JK, ("fock_device", call, err)


def test_noalloc_coulomb_refuses_sizes_beyond_its_scratch():
    n, naux = 2000, 4  # 32 x 32 tile rows: two copies of the packed tiles exceed 32 MiB
    rng = np.random.default_rng(0)
    V = np.eye(naux) * 2.0
    I3 = rng.normal(size=(n * (n + 1) // 2, naux))
    f = _noalloc(rijk.lib())
    import torch
    dev = torch.device("cuda", 0)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(V)
        fb.set_3c(I3, n)
        dD = torch.zeros((n, n), dtype=torch.float64, device=dev)
        dJ = torch.zeros((n, n), dtype=torch.float64, device=dev)
        rc = f(fb._h, dD.data_ptr(), dJ.data_ptr())
        assert rc == rijk.ERR_ARG
        assert "scratch" in fb.last_error()
