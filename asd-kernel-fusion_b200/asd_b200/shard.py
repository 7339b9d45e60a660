"""Replica sharding of one ensemble over ranks, one GPU (one context) each.

Replicas never interact in the LLG step, and the correlation GEMM's K axis is
the replica axis, so rank r holds replicas [f_r, f_r+1) of the ensemble and
steps them on its own.  S(q,t) needs one exchange per evaluation: each shard
contributes its partial GEMM value (2 doubles) and its per-site replica sums
(3 N^2 doubles), both all-reduced, after which any rank forms the connected
part from the ensemble's means (asd_ctx_shard_sqt_finish).  The origin's site
sums are exchanged once.  On NCCL the all-reduces run on torch's current
stream, which is also the context's stream, so no host synchronisation is
needed between the steps.

The reference runs one process on one machine; sharding is this build's.
"""
from __future__ import annotations


def shard_range(nfile_total: int, rank: int, world: int) -> tuple[int, int]:
    """Replicas [begin, end) of rank `rank` when nfile_total are split as
    evenly as possible over `world` ranks (the first nfile_total % world ranks
    hold one more)."""
    base, extra = divmod(int(nfile_total), int(world))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


class ShardedSqt:
    """S(q,t) of an ensemble whose replicas are spread over the ranks of a
    torch.distributed group.  `ctx` holds this rank's replicas (a
    `asd_b200.Context` or an object with the same shard_* methods); buffers are
    torch tensors on `device`."""

    def __init__(self, ctx, nfile_total: int, n_sites: int, device="cuda", group=None):
        import torch

        self.ctx, self.group = ctx, group
        ctx.set_ensemble(nfile_total)
        if str(device).startswith("cuda") and hasattr(ctx, "set_stream"):
            ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        f64 = dict(dtype=torch.float64, device=device)
        self.part = torch.zeros(2, **f64)
        self.sums = torch.zeros(3 * n_sites, **f64)
        self.zsums = torch.zeros(3 * n_sites, **f64)
        self.out = torch.zeros(2, **f64)
        self.launches = 0

    def _all_reduce(self, t):
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            dist.all_reduce(t, group=self.group)

    def exchange_origin(self) -> None:
        """After set_spins(..., as_origin=True) on every rank."""
        self.ctx.shard_origin_sums(self.zsums)
        self._all_reduce(self.zsums)
        self.ctx.shard_set_origin_sums(self.zsums)

    def sqt_async(self, mode, out=None):
        """Enqueues one evaluation; the result lands in `out` (2 doubles,
        default self.out) on every rank."""
        out = self.out if out is None else out
        self.ctx.shard_sqt_async(mode, self.part, self.sums)
        n = self.ctx.last_launches() if hasattr(self.ctx, "last_launches") else 0
        self._all_reduce(self.part)
        self._all_reduce(self.sums)
        self.ctx.shard_sqt_finish(self.part, self.sums, out)
        self.launches = n + 1  # this library's kernels in the evaluation
        return out

    def sqt(self, mode) -> complex:
        o = self.sqt_async(mode).cpu()
        return complex(float(o[0]), float(o[1]))
