"""Aux-index slices on the GPU (rijk_set_aux_range): two contexts holding [0, q1) and
[q1, naux) give partial J, K and active integrals that sum to the full ones (FP64 and the
int8-digit FP64_TC K to 1e-9, mixed to its tolerance).  This is the arithmetic of the multi-GPU sharding in
nopt_b200.parallel, checked on one GPU without collectives.

The aux-sharded SCF runs here as two host threads, one context and one slice each, whose J/K
reduction meets on the host (a barrier with a time limit, the sum formed in the same order by both):
the kernels of the two contexts never wait on each other.  The NCCL reduction of
ShardedFockBuilder.scf runs in a one-rank group."""
import threading

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


@pytest.mark.parametrize("backend", ["nccl", "gloo"])
def test_sharded_builder_one_rank(backend):
    """ShardedFockBuilder in a one-rank group on this GPU, against the plain builder.  NCCL: the
    device path of dm_to_f_transform_ri (D and the orbitals up once, the partial build into one
    device buffer, one all-reduce, J and K down once) and the SCF's all-reduce on the build's
    stream.  gloo: the host reductions of both."""
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
    dist.init_process_group(backend, init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    try:
        with rijk.FockBuilder(0) as fb, rijk.FockBuilder(0) as ref:
            sb = ShardedFockBuilder(fb)
            sb.setup(si.V, si.I3, si.n)
            assert sb.slice == (0, si.naux)
            J, K = sb.dm_to_f_transform_ri(DM, MO, si.nocc)
            ref.set_metric(si.V)
            ref.set_3c(si.I3, si.n)
            Jr, Kr = ref.dm_to_f_transform_ri(DM, MO, si.nocc)
            # the sharded SCF: rijk_scf with the all-reduce of [J | K] on its stream after each build
            Es, MOs, rs = sb.scf(si.H, si.S, si.nocc, si.Enuc, guess=si.sad())
            Er, MOr, rr = ref.scf(si.H, si.S, si.nocc, si.Enuc, guess=si.sad())
        assert np.max(np.abs(J - Jr)) < 1e-12 and np.max(np.abs(K - Kr)) < 1e-12
        assert rs["converged"] and rs["iterations"] == rr["iterations"]
        assert abs(Es - Er) < 1e-11
    finally:
        dist.destroy_process_group()


def _host_reducer(rank, parts, barrier):
    """reduce_jk for one of two threads: the stream's partial [J | K] to the host, both parts summed
    in rank order once both are there, the sum written back before the library goes on."""
    import torch
    from nopt_b200.parallel import device_tensor

    def reduce_jk(ptr, count, stream):
        torch.cuda.ExternalStream(stream).synchronize()
        t = device_tensor(ptr, count, torch.device("cuda", 0))
        parts[rank] = t.cpu()
        barrier.wait()
        total = parts[0] + parts[1]
        barrier.wait()  # both sums formed before either thread's next build overwrites its part
        t.copy_(total)
        torch.cuda.current_stream().synchronize()
    return reduce_jk


@pytest.mark.parametrize("precision,converger", [(rijk.PREC_FP64, rijk.CONV_DIIS),
                                                 (rijk.PREC_MIXED, rijk.CONV_DIIS_SOSCF)])
def test_scf_on_two_aux_slices(precision, converger):
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")
    guess = si.sad()
    kw = dict(precision=precision, converger=converger, guess=guess)
    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_3c(si.I3, si.n)
        Ef, MOf, rf = fb.scf(si.H, si.S, si.nocc, si.Enuc, **kw)
    q1 = 301
    parts, out = [None, None], [None, None]
    barrier = threading.Barrier(2, timeout=120)

    def rank_main(rank, q0, q1_):
        try:
            with rijk.FockBuilder(0) as b:
                b.set_metric(si.V)
                b.set_aux_range(q0, q1_)
                b.set_3c(si.I3, si.n)
                out[rank] = b.scf(si.H, si.S, si.nocc, si.Enuc, reduce_jk=_host_reducer(rank, parts, barrier), **kw)
        except BaseException as e:  # the other thread's barrier then breaks and ends its SCF too
            out[rank] = e
            barrier.abort()

    threads = [threading.Thread(target=rank_main, args=(0, 0, q1)),
               threading.Thread(target=rank_main, args=(1, q1, si.naux))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    for o in out:
        if isinstance(o, BaseException):
            raise o
    (Ea, MOa, ra), (Eb, MOb, rb) = out
    # the ranks take the same steps on the same reduced J and K: identical results
    assert Ea == Eb and ra["iterations"] == rb["iterations"] and np.array_equal(MOa, MOb)
    assert ra["converged"] and rf["converged"]
    # FP64: the full-range SCF to rounding; mixed: its FP64 phase ends at the FP64 energy
    assert abs(Ea - Ef) < (1e-9 if precision == rijk.PREC_FP64 else 1e-8), (Ea, Ef)


def test_scf_reduce_failure_is_a_status():
    si = ints.SystemIntegrals(water_cluster((2, 3), seed=0), "cc-pvdz", "cc-pvdz-jkfit")

    def broken(ptr, count, stream):
        raise ValueError("collective failed")

    with rijk.FockBuilder(0) as fb:
        fb.set_metric(si.V)
        fb.set_aux_range(0, 200)
        fb.set_3c(si.I3, si.n)
        with pytest.raises(ValueError):
            fb.scf(si.H, si.S, si.nocc, si.Enuc, reduce_jk=broken)
        assert "reduce_jk" in fb.last_error()
        # the context stays usable
        DM = np.eye(si.n) * 0.1
        J, K = fb.dm_to_f_transform_ri(DM, np.eye(si.n)[:si.nocc], si.nocc)
        assert np.isfinite(J).all() and np.isfinite(K).all()

