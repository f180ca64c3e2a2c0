"""Aux-index slices on the GPU (rijk_set_aux_range): two contexts holding [0, q1) and
[q1, naux) give partial J, K and active integrals that sum to the full ones (FP64 and the
int8-digit FP64_TC K to 1e-9, mixed to its tolerance).  This is the arithmetic of the multi-GPU sharding in
nopt_b200.parallel, checked on one GPU without collectives."""
import numpy as np
import pytest

import rijk_oracle as O
from nopt_b200 import ints, rijk
from nopt_b200.molecules import water_cluster

pytestmark = pytest.mark.gpu


def test_two_aux_slices_sum_to_full():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    rng = np.random.default_rng(4)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    MO = C.T.copy()
    DM = O.gen_hf_dm(MO, si.n, si.nocc)
    q1 = 301
    out = {}
    for name, rng_ in (("full", None), ("a", (0, q1)), ("b", (q1, si.naux))):
        with rijk.FockBuilder(0) as fb:
            fb.set_metric(si.V)
            if rng_:
                fb.set_aux_range(*rng_)
            fb.set_3c(si.I3, si.n)
            J, K = fb.dm_to_f_transform_ri(DM, MO, si.nocc)
            Jm, Km = fb.dm_to_f_transform_ri(DM, MO, si.nocc, rijk.PREC_MIXED)
            act = MO[si.nocc - 2:si.nocc + 2]
            I, _, _ = fb.calc_2el_mo_ints_ri(None, MO, act, act, 0, 4, want_jk=False)
            _, Kt = fb.dm_to_f_transform_ri(DM, MO, si.nocc, rijk.PREC_FP64_TC)
            out[name] = (J, K, Jm, Km, I, Kt)
    f, a, b = out["full"], out["a"], out["b"]
    assert np.max(np.abs(a[0] + b[0] - f[0])) < 1e-9
    assert np.max(np.abs(a[1] + b[1] - f[1])) < 1e-9
    assert np.max(np.abs(a[4] + b[4] - f[4])) < 1e-9
    assert np.max(np.abs(a[3] + b[3] - f[1])) < 2e-4
    # the int8 digit form of K on each slice: digit exponents per slice, FP64 partials that sum
    assert np.max(np.abs(a[5] + b[5] - f[1])) < 1e-9
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        with pytest.raises(rijk.RijkError) as e:
            fb.set_aux_range(5, 5)
        assert e.value.code == rijk.ERR_ARG
        fb.set_aux_range(0, 10)
        fb.set_3c(si.I3, si.n)
        with pytest.raises(rijk.RijkError) as e:
            fb.scf(si.H, si.S, si.nocc, si.Enuc)
        assert e.value.code == rijk.ERR_STATE


def test_sharded_builder_nccl_device_path_one_rank():
    """The NCCL path of ShardedFockBuilder.dm_to_f_transform_ri (D and the orbitals up once, the
    partial build into one device buffer, one all-reduce, J and K down once) in a one-rank NCCL
    group on this GPU, against the plain builder."""
    import socket

    import torch
    import torch.distributed as dist
    from nopt_b200.parallel import ShardedFockBuilder
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    rng = np.random.default_rng(9)
    C, _ = np.linalg.qr(rng.normal(size=(si.n, si.n)))
    MO = C.T.copy()
    DM = O.gen_hf_dm(MO, si.n, si.nocc)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    try:
        with rijk.FockBuilder(0) as fb, rijk.FockBuilder(0) as ref:
            sb = ShardedFockBuilder(fb)
            sb.setup(si.V, si.I3, si.n)
            assert sb.slice == (0, si.naux)
            J, K = sb.dm_to_f_transform_ri(DM, MO, si.nocc)
            ref.set_metric(si.V)
            ref.set_3c(si.I3, si.n)
            Jr, Kr = ref.dm_to_f_transform_ri(DM, MO, si.nocc)
        assert np.max(np.abs(J - Jr)) < 1e-12 and np.max(np.abs(K - Kr)) < 1e-12
    finally:
        dist.destroy_process_group()
