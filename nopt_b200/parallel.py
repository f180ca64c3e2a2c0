"""Aux-index (Q) sharding of the Fock build over the ranks of a torch.distributed group.

J = sum_Q B^Q w_Q and K = sum_Q X^Q^T X^Q are sums over the auxiliary index Q, so each rank
holds the fitted tensor for one contiguous slice of Q (rijk_set_aux_range) and computes that
slice's partial J and K; one all-reduce (sum) of the two n x n matrices is the only exchange.
B, the expensive part (n^2 naux / 2 doubles), is divided; the metric factor (naux^2) and the
n x n matrices are replicated.  Over NVLink the exchange is 2 n^2 doubles per build (55 MB at
n = 1856), small next to the per-rank contraction.

The SCF shards the same way: every rank runs rijk_scf on its slice with the same arguments, and after
each Fock build the library hands the partial [J | K] (one device array) to a callback that sums it over
the ranks; the rest of every iteration is replicated, and identical on every rank.

The local builder is any object with the FockBuilder methods set_metric, set_aux_range, set_3c,
fock_device / dm_to_f_transform_ri / scf (nopt_b200.rijk.FockBuilder on the rank's GPU).
"""
import numpy as np


class DeviceArray:
    """float64 device memory at a raw pointer, as torch.as_tensor takes it without a copy (the CUDA
    array interface, version 2: no stream attached; the caller orders the work)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 2}


def device_tensor(ptr, count, device):
    import torch
    return torch.as_tensor(DeviceArray(ptr, count), device=device)


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
        """Host arrays in and out (the drop-in semantics of DM_to_F_transform_RI).  Over NCCL: D and
        the orbitals go up once, the partial build writes J and K into one device buffer, one
        all-reduce sums it across the ranks, and J and K come down once -- the host traffic of a
        one-GPU rijk_fock.  Over gloo (CPU ranks) the local builder's host J and K are summed."""
        import torch
        backend = self.dist.get_backend(self.group)
        if backend != "nccl":
            J, K = self.local.dm_to_f_transform_ri(DM, MO, n_c, precision)
            tJ = torch.from_numpy(np.ascontiguousarray(J))
            tK = torch.from_numpy(np.ascontiguousarray(K))
            self._allreduce(tJ, tK)
            return tJ.numpy(), tK.numpy()
        n = self.n
        dev = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.current_stream(dev)
        self.local.set_stream(stream.cuda_stream)  # the build and the collective on one stream
        dD = torch.from_numpy(np.ascontiguousarray(DM, dtype=np.float64)).to(dev)
        rows = max(int(n_c), 1)
        MOh = np.ascontiguousarray(MO[:rows], dtype=np.float64) if n_c > 0 else np.zeros((1, n))
        dMO = torch.from_numpy(MOh).to(dev)
        jk = torch.empty((2, n, n), dtype=torch.float64, device=dev)
        self.local.fock_device(dD.data_ptr(), dMO.data_ptr(), n_c, jk[0].data_ptr(), jk[1].data_ptr(), precision)
        self._allreduce(jk)
        out = jk.cpu().numpy()
        return out[0], out[1]

    def scf(self, H, S, n_c, e_nuc, **kw):
        """Aux-sharded RHF (rijk_scf on this rank's slice; keyword arguments as FockBuilder.scf).
        After every Fock build the partial [J | K] is summed over the group in place: over NCCL by an
        all-reduce enqueued on the build's own stream; over another backend through host memory (the
        stream synchronised first).  Every rank must call this with the same arguments."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        nccl = self.dist.get_backend(self.group) == "nccl"

        def reduce_jk(ptr, count, stream):
            t = device_tensor(ptr, count, dev)
            ext = torch.cuda.ExternalStream(stream, device=dev) if stream else torch.cuda.default_stream(dev)
            if nccl:
                with torch.cuda.stream(ext):
                    self._allreduce(t)
                return
            ext.synchronize()
            h = t.cpu()
            self._allreduce(h)
            t.copy_(h)
            torch.cuda.current_stream(dev).synchronize()

        return self.local.scf(H, S, n_c, e_nuc, reduce_jk=reduce_jk, **kw)
