"""Aux-index sharding of the Fock build (nopt_b200.parallel), world size 2 on CPU (gloo).

Each rank holds one slice of Q; its partial J, K come from a local builder, and one all-reduce
gives the full matrices.  On CPU the local builder is the oracle restricted to the slice (the
GPU builder is exercised on one GPU in tests/test_gpu_shard.py); the sum over ranks must equal
the oracle's full J, K."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import rijk_oracle as O
from nopt_b200.parallel import aux_slices


class OracleSlice:
    """The oracle's J, K restricted to aux functions [q0, q1) of B = V^-1/2 (P|mu nu)."""

    def set_metric(self, V, form=0):
        self.M, _ = O.s05_calc(V)

    def set_aux_range(self, q0, q1):
        self.q0, self.q1 = q0, q1

    def set_3c(self, I3, n, layout=1):
        self.n = n
        self.Bp = (self.M @ I3.T)[self.q0:self.q1]

    def dm_to_f_transform_ri(self, DM, MO, n_c, precision=0):
        return O.jk_from_b(self.Bp, self.n, DM, MO, n_c)


def _problem(seed=3, n=23, naux=31, nocc=5):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(naux, naux))
    V = A @ A.T / naux + np.eye(naux)
    I3 = rng.normal(size=(n * (n + 1) // 2, naux)) * 0.2
    DM = rng.normal(size=(n, n))
    MO = rng.normal(size=(nocc, n))
    return V, I3, DM, MO, n, nocc


def _worker(rank, world, port, out_q):
    import torch.distributed as dist
    from nopt_b200.parallel import ShardedFockBuilder
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    V, I3, DM, MO, n, nocc = _problem()
    sb = ShardedFockBuilder(OracleSlice())
    sb.setup(V, I3, n)
    J, K = sb.dm_to_f_transform_ri(DM, MO, nocc)
    out_q.put((rank, sb.slice, J, K))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_aux_slices_cover_range():
    for naux, world in [(10, 3), (4448, 8), (7, 7), (5, 1)]:
        sl = aux_slices(naux, world)
        assert sl[0][0] == 0 and sl[-1][1] == naux
        assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
        sizes = [b - a for a, b in sl]
        assert max(sizes) - min(sizes) <= 1


def test_sharded_jk_world2_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    V, I3, DM, MO, n, nocc = _problem()
    Vm05, _ = O.s05_calc(V)
    Jr, Kr = O.dm_to_f_transform_ri(O.unpack_3c(I3, n), Vm05, DM, MO, nocc, n)
    slices = sorted(r[1] for r in res)
    assert slices == [(0, 16), (16, 31)]
    for _, _, J, K in res:
        np.testing.assert_allclose(J, Jr, atol=1e-11)
        np.testing.assert_allclose(K, Kr, atol=1e-11)
