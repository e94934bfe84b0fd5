"""One molecule's Fock build over several GPUs, one process per GPU.

The reference splits the quartet task space of a build over MPI ranks in a
2-D (M-block x P-block) grid, accumulates F in Global Arrays and reduces it
(pfock/pfock.c:22-154, 1373-1669).  Here every rank builds one shard of
every class launch's quartet units on its own GPU (PFock.set_shard: a
contiguous slice of each launch's unit range, its bras split by their work
model with gtf_shard_split), and one
all-reduce over the ranks' torch.distributed group sums the parts into F
-- NCCL over NVLink for device matrices, gloo for host arrays.  D is the
same on every rank (the SCF state is replicated, as in the reference where
every rank holds the purification's D blocks), so a build exchanges only F.

ShardedFock.compute_fock(D): host D in, whole F out (host).
ShardedFock.compute_fock_dev(D): D a CUDA tensor; F is all-reduced in place
in the library's device buffer (a zero-copy torch view), no host copies.
"""
import ctypes

import numpy as np

from . import PFock, load


def shard_range(nunits, shard, nshards):
    """Units [lo, hi) of shard `shard` of `nshards` of a launch of `nunits`
    equal units."""
    lo, hi = ctypes.c_longlong(), ctypes.c_longlong()
    load().gtf_shard_range(int(nunits), int(shard), int(nshards), ctypes.byref(lo), ctypes.byref(hi))
    return lo.value, hi.value


def shard_split(weights, shard, nshards):
    """Items [lo, hi) of shard `shard` of `nshards` for items of the given
    weights: the library's contiguous weighted split (gtf_shard_split), the
    one a sharded engine applies to each launch's bras."""
    w = np.ascontiguousarray(weights, dtype=np.float64)
    lo, hi = ctypes.c_longlong(), ctypes.c_longlong()
    load().gtf_shard_split(w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(w.size), int(shard),
                           int(nshards), ctypes.byref(lo), ctypes.byref(hi))
    return lo.value, hi.value


class _DeviceMatrix:
    """A library-owned n x n FP64 device matrix seen through the CUDA array
    interface, so torch.as_tensor wraps it without a copy."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n, n), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def allreduce_fock(F, group=None):
    """Sum the ranks' parts of F in place and return it.  F is a torch tensor
    (reduced where it lives: NCCL needs CUDA, gloo host or device) or a numpy
    array (reduced through a shared-memory CPU tensor on a gloo group, or a
    CUDA copy on an NCCL group)."""
    import torch
    import torch.distributed as dist
    if isinstance(F, np.ndarray):
        if dist.get_backend(group) == "nccl":
            t = torch.from_numpy(F).cuda()
            dist.all_reduce(t, group=group)
            F[...] = t.cpu().numpy()
        else:
            dist.all_reduce(torch.from_numpy(F), group=group)
        return F
    dist.all_reduce(F, group=group)
    return F


class ShardedFock:
    """A PFock engine that builds this rank's shard; F is summed over the
    ranks of `group` (default: the world)."""

    def __init__(self, basis, tolscr=1e-10, group=None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.nranks = dist.get_world_size(group)
        self.nbf = basis.nbf
        self.pf = PFock(basis, tolscr=tolscr)
        self.pf.set_shard(self.rank, self.nranks)

    def compute_fock(self, D):
        F = self.pf.compute_fock(D)
        return allreduce_fock(F, self.group)

    def compute_fock_dev(self, D):
        """D: CUDA tensor (nbf x nbf, float64, contiguous) on this rank's GPU.
        Returns a CUDA tensor viewing the library's F, summed over the ranks
        (valid until this engine's next build)."""
        import torch
        if not (D.is_cuda and D.dtype == torch.float64 and D.is_contiguous() and D.shape == (self.nbf, self.nbf)):
            raise ValueError("D must be a contiguous float64 CUDA tensor of shape (nbf, nbf)")
        # the engine reads D on its own stream, which is not ordered after
        # torch's: D must be complete before the build starts
        torch.cuda.current_stream(D.device).synchronize()
        ptr = self.pf.compute_dev(D.data_ptr())
        F = torch.as_tensor(_DeviceMatrix(ptr, self.nbf), device=D.device)
        return allreduce_fock(F, self.group)

    def close(self):
        # the engine frees F on its own stream: work of other streams (the
        # all-reduce) that uses the view must be complete
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
        self.pf.close()
