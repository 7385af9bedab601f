"""Multi-rank Fock build on CPU: two gloo ranks each build a shard of the
J/K work and ShardedJK sums them with one all-reduce; the result equals the
single-process build.  The shards here are the oracle's bra shell-pair rows
(the hf-rs restatement), so the test needs no GPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_path, nspin):
    import torch
    import torch.distributed as dist
    import oracle as O
    from hfgpu.clusters import water_cluster
    from hfgpu.parallel import ShardedJK

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    atoms = water_cluster(2)
    basis = O.build_basis(atoms, O.load_basis("sto-3g"))
    npair = len(O.schwarz(basis))
    rng = np.random.default_rng(7)
    n = sum(1 for _ in basis)
    Pa = rng.standard_normal((n, n)); Pa = Pa + Pa.T
    Pb = rng.standard_normal((n, n)); Pb = Pb + Pb.T
    spins = [Pa] if nspin == 1 else [Pa, Pb]
    total = Pa if nspin == 1 else Pa + Pb

    def build(P, Ps, J, K, shard, nshards):
        rows = np.arange(shard, npair, nshards)
        Jp, Kp = O.direct_jk(basis, P.numpy(), [x for x in Ps.numpy()], rows=rows)
        J.copy_(torch.from_numpy(Jp))
        K.copy_(torch.from_numpy(Kp))

    J = torch.zeros((n, n), dtype=torch.float64)
    K = torch.zeros((nspin, n, n), dtype=torch.float64)
    ShardedJK(rank, world, nspin=nspin, build=build)(torch.from_numpy(total), torch.from_numpy(np.stack(spins)), J, K)
    if rank == 0:
        Jr, Kr = O.direct_jk(basis, total, spins)
        np.save(out_path, np.array([np.max(np.abs(J.numpy() - Jr)), np.max(np.abs(K.numpy() - Kr)),
                                    np.max(np.abs(Jr))]))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_fock_build_two_gloo_ranks(tmp_path):
    for nspin in (1, 2):
        out = str(tmp_path / ("res%d.npy" % nspin))
        mp.start_processes(_rank_main, args=(2, _free_port(), out, nspin), nprocs=2, join=True, start_method="spawn")
        dj, dk, scale = np.load(out)
        assert scale > 1.0
        assert dj < 1e-11 and dk < 1e-11


def _df_rank_main(rank, world, port, out_path):
    import torch
    import torch.distributed as dist
    import oracle as O
    from hfgpu.clusters import water_cluster
    from hfgpu.parallel import ShardedJK, aux_shard_range

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    atoms = water_cluster(1)
    basis = O.build_basis(atoms, O.load_basis("sto-3g"))
    aux = O.build_basis(atoms, O.load_basis("def2-svp-ri"))
    B = O.df_tensor(basis, aux)
    n, nq = len(basis), B.shape[0]
    q, _ = np.linalg.qr(np.random.default_rng(3).standard_normal((n, n)))
    C = np.ascontiguousarray(q[:, :5])

    def build(Ct, _unused, J, K, shard, nshards):
        lo, hi = aux_shard_range(nq, shard, nshards)
        Jp, Kp = O.df_jk(B[lo:hi], Ct.numpy(), n)
        J.copy_(torch.from_numpy(Jp))
        K.copy_(torch.from_numpy(Kp))

    J = torch.zeros((n, n), dtype=torch.float64)
    K = torch.zeros((n, n), dtype=torch.float64)
    ShardedJK(rank, world, build=build)(torch.from_numpy(C), None, J, K)
    if rank == 0:
        Jr, Kr = O.df_jk(B, C, n)
        np.save(out_path, np.array([np.max(np.abs(J.numpy() - Jr)), np.max(np.abs(K.numpy() - Kr)),
                                    np.max(np.abs(Jr))]))
    dist.barrier()
    dist.destroy_process_group()


def test_df_jk_sharded_over_the_auxiliary_index_two_gloo_ranks(tmp_path):
    # the DF shard decomposition (hfg_df_jk_device_shard's ranges): two ranks
    # each sum over half of the auxiliary functions, one all-reduce, equal to
    # the single-process DF J/K of the oracle
    out = str(tmp_path / "df.npy")
    mp.start_processes(_df_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    dj, dk, scale = np.load(out)
    assert scale > 0.1
    assert dj < 1e-12 and dk < 1e-12


def test_aux_shard_ranges_cover_every_auxiliary_function_once():
    from hfgpu.parallel import aux_shard_range
    for rank in (1, 7, 85, 8512):
        for nshards in (1, 2, 3, 8):
            cover = [q for s in range(nshards) for q in range(*aux_shard_range(rank, s, nshards))]
            assert cover == list(range(rank))
