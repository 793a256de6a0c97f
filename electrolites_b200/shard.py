"""Multi-GPU J/K builds: one process per GPU, each class's task list split
across the ranks, one all-reduce of vj / vk.

Every rank holds the same plan and densities.  Rank r evaluates the tasks
r, r + size, r + 2 size, ... of every class launch (jk_plan_set_shard), so
its vj / vk are a partial sum; the J/K assembly (J_h + J_h^T, K_h + ...) is
linear, so one SUM all-reduce over the ranks' outputs gives the full
result on every rank.  vj and vk live in one buffer, so the exchange is a
single collective of n_dm * 2 * nao^2 doubles.

The reference runs on one GPU (electrolites/fastk.py:657); this is the
sharded form of its get_jk.
"""
from __future__ import annotations


def _torch():
    import torch
    return torch


def allreduce_jk(buf, group=None):
    """Sum buf over the ranks of group, in place (one collective)."""
    import torch.distributed as dist
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    return buf


class ShardedJK:
    """get_jk over the ranks of a process group.

    opt: a built VHFOpt on this rank's GPU (or any object with the same
    ``set_shard`` / ``build_jk_async`` / ``sync`` methods).  The process
    group must be initialised (NCCL for CUDA tensors)."""

    def __init__(self, opt, group=None):
        import torch.distributed as dist
        self.opt = opt
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        opt.set_shard(self.rank, self.size)

    def get_jk(self, dms, hermi=1, with_j=True, with_k=True, mixed_threshold=0.0):
        """(vj, vk) of the whole build on every rank; dms (n_dm, nao, nao) on
        this rank's device, identical on every rank."""
        torch = _torch()
        buf = torch.zeros((2,) + tuple(dms.shape), dtype=dms.dtype, device=dms.device)
        vj = buf[0] if with_j else None
        vk = buf[1] if with_k else None
        self.opt.build_jk_async(dms, hermi, with_j, with_k, vj, vk, mixed_threshold)
        self.opt.sync()
        allreduce_jk(buf, self.group)
        return (buf[0] if with_j else None), (buf[1] if with_k else None)
