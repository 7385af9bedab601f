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


def aux_shard_range(rank, shard, nshards):
    """Auxiliary functions [lo, hi) of DF shard `shard` of `nshards` (the
    split hfg_df_jk_device_shard uses)."""
    return rank * shard // nshards, rank * (shard + 1) // nshards


class ShardFactorDFJK(ShardedJK):
    """DF J/K where each rank holds only its share of the factor (a DFTensor
    built with shard=rank, nshards=world), hf-rs's map-reduce over Q
    (src/df.rs:143-173) across GPUs: the rank's J and K over its rows, then
    one all-reduce.  Call with (C, None, J, K) as ShardedDFJK."""

    def __init__(self, rank, world, df_shard, nocc, mma=0, group=None):
        def build(C, _unused, J, K, shard, nshards):
            df_shard.jk_device_shard(C.data_ptr(), nocc, J.data_ptr(), K.data_ptr(), 0, 1, mma=mma)

        super().__init__(rank, world, build=build, group=group)


class ShardedDFJK(ShardedJK):
    """DF J/K of occupied coefficients on all ranks: each rank sums over its
    range of auxiliary functions (hfg_df_jk_device_shard) and one all-reduce
    adds the partial J and K (hf-rs's map-reduce over Q, src/df.rs:143-173).
    Call with (C, None, J, K): C column-major n x nocc (a torch tensor whose
    storage is the n x nocc block of a column-major matrix), J and K n x n."""

    def __init__(self, rank, world, df, nocc, mma=0, group=None):
        def build(C, _unused, J, K, shard, nshards):
            df.jk_device_shard(C.data_ptr(), nocc, J.data_ptr(), K.data_ptr(), shard, nshards, mma=mma)

        super().__init__(rank, world, build=build, group=group)
