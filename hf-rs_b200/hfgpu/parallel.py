"""Multi-GPU Fock build: one process per GPU.

Every rank holds the whole basis, pair tables and density (a context per
GPU), builds its cost-balanced shard of the J/K work (hfg_jk_device_shard:
each launch's work queue cut into equal-cost ranges), and the partial J and
K matrices are summed with one all-reduce over the process group (NCCL over
NVLink on GPUs).  hf-rs's counterpart is its Rayon loop over shell quartets
inside one process (src/shell_integrals.rs:184-240); the sum of the shards
equals the single-GPU build because J and K are linear in the integrals.
"""


class ShardedJK:
    """J/K of one density on all ranks of `group`.

    `build(P, Ps, J, K, shard, nshards)` fills J and K with the rank's partial
    sums; by default it is the context's hfg_jk_device_shard.  J and K are
    torch tensors on this rank's device (or CPU with gloo); on return they
    hold the full J and K on every rank.
    """

    def __init__(self, rank, world, ctx=None, opts=None, nspin=1, build=None, group=None):
        self.rank, self.world, self.nspin, self.group = rank, world, nspin, group
        if build is None:
            if ctx is None:
                raise ValueError("ShardedJK needs a context or a build function")

            def build(P, Ps, J, K, shard, nshards):
                ctx.jk_device_shard(P.data_ptr(), Ps.data_ptr(), J.data_ptr(), K.data_ptr(), shard, nshards,
                                    nspin=nspin, opts=opts)
        self.build = build

    def __call__(self, P, Ps, J, K):
        import torch.distributed as dist
        self.build(P, Ps, J, K, self.rank, self.world)
        if self.world > 1:
            dist.all_reduce(J, op=dist.ReduceOp.SUM, group=self.group)
            dist.all_reduce(K, op=dist.ReduceOp.SUM, group=self.group)
        return J, K
