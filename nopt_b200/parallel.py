"""Aux-index (Q) sharding of the Fock build over the ranks of a torch.distributed group.

J = sum_Q B^Q w_Q and K = sum_Q X^Q^T X^Q are sums over the auxiliary index Q, so each rank
holds the fitted tensor for one contiguous slice of Q (rijk_set_aux_range) and computes that
slice's partial J and K; one all-reduce (sum) of the two n x n matrices is the only exchange.
B, the expensive part (n^2 naux / 2 doubles), is divided; the metric factor (naux^2) and the
n x n matrices are replicated.  Over NVLink the exchange is 2 n^2 doubles per build (55 MB at
n = 1856), small next to the per-rank contraction.

The local builder is any object with the FockBuilder methods set_metric, set_aux_range, set_3c,
fock_device / dm_to_f_transform_ri (nopt_b200.rijk.FockBuilder on the rank's GPU).
"""
import numpy as np


def aux_slices(naux, world):
    """Contiguous, balanced [q0, q1) slices of range(naux), one per rank."""
    base, extra = divmod(naux, world)
    out, q = [], 0
    for r in range(world):
        w = base + (1 if r < extra else 0)
        out.append((q, q + w))
        q += w
    return out


class ShardedFockBuilder:
    def __init__(self, local, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.local = local
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.slice = None

    def setup(self, V, I3, n, metric_form=0, layout=1):
        naux = V.shape[0]
        self.slice = aux_slices(naux, self.world)[self.rank]
        self.local.set_metric(V, metric_form)
        self.local.set_aux_range(*self.slice)
        self.local.set_3c(I3, n, layout)
        self.n = n

    def _allreduce(self, *tensors):
        for t in tensors:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)

    def fock_device(self, dD, dMO, n_c, dJ, dK, precision=0):
        """Device tensors (torch, on this rank's GPU): partial build on the local stream, then the
        all-reduce on the same stream (NCCL)."""
        self.local.fock_device(dD.data_ptr(), dMO.data_ptr(), n_c, dJ.data_ptr(), dK.data_ptr(), precision)
        self._allreduce(dJ, dK)

    def dm_to_f_transform_ri(self, DM, MO, n_c, precision=0):
        """Host arrays in and out (the drop-in semantics of DM_to_F_transform_RI)."""
        import torch
        J, K = self.local.dm_to_f_transform_ri(DM, MO, n_c, precision)
        backend = self.dist.get_backend(self.group)
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        tJ = torch.from_numpy(np.ascontiguousarray(J)).to(dev)
        tK = torch.from_numpy(np.ascontiguousarray(K)).to(dev)
        self._allreduce(tJ, tK)
        return tJ.cpu().numpy(), tK.cpu().numpy()
