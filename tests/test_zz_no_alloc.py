"""The allocation-free J/K entry point (hfg_jk_device_noalloc).

Some callers cannot allocate device memory while they run -- latency-bound
loops that cannot take cudaMalloc's device synchronisation, and host programs
whose own allocator has reserved all device memory.  This entry point serves
them from an 8 MiB device array the library reserves at load time.  These tests call it through the C ABI and check it against the
ordinary entry point, on two calls in a row (the array is shared and keeps
the previous call's contents, so the second call checks that it is cleared).
This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from hfgpu import CartesianBasis, Context, JKOptions
from hfgpu.clusters import water_cluster

pytestmark = pytest.mark.gpu


def rand_sym(n, seed):
    a = np.random.default_rng(seed).standard_normal((n, n)) * 0.3
    return a + a.T


def noalloc(ctx, opts, nspin, Pt, Ps, J, K):
    import torch
    torch.cuda.synchronize()
    rc = ctx.lib.hfg_jk_device_noalloc(ctx.h, ctypes.byref(opts), nspin, Pt.data_ptr(), Ps.data_ptr(),
                                       J.data_ptr(), K.data_ptr())
    torch.cuda.synchronize()
    return rc


@pytest.mark.parametrize("mixed", [None, 1e-6])
@pytest.mark.parametrize("nspin", [1, 2])
def test_noalloc_matches_jk_on_two_calls(nspin, mixed):
    import torch
    atoms = water_cluster(2)
    basis = CartesianBasis.build(atoms, "cc-pvdz")
    n = basis.n
    ctx = Context(basis)
    # FP64, and mixed precision (twice as many launches, so twice the counters)
    opts = JKOptions.make(mixed=mixed)
    dev = torch.device("cuda", 0)
    for call, seed in enumerate((11, 12)):
        Pa, Pb = rand_sym(n, seed), rand_sym(n, seed + 100)
        spins = [Pa] if nspin == 1 else [Pa, Pb]
        total = Pa if nspin == 1 else Pa + Pb
        J_ref, K_ref = ctx.jk(total, spins, opts=opts)  # ordinary entry point (also prepares the plan)
        Pt = torch.from_numpy(total).to(dev)
        Ps = torch.from_numpy(np.stack(spins)).to(dev)
        J = torch.full((n, n), np.nan, dtype=torch.float64, device=dev)
        K = torch.full((nspin, n, n), np.nan, dtype=torch.float64, device=dev)
        assert noalloc(ctx, opts, nspin, Pt, Ps, J, K) == 0, ctx.lib.hfg_last_error(ctx.h)
        assert np.max(np.abs(J.cpu().numpy() - J_ref)) < 1e-11, call
        assert np.max(np.abs(K.cpu().numpy() - K_ref)) < 1e-11, call
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch_and_missing_plans():
    import torch
    dev = torch.device("cuda", 0)
    small = Context(CartesianBasis.build(water_cluster(1), "cc-pvdz"))
    n = small.n
    z = torch.zeros((n, n), dtype=torch.float64, device=dev)
    rc = noalloc(small, JKOptions.make(), 1, z, z, torch.empty_like(z), torch.empty_like(z))
    assert rc == 1 and b"no launch plan" in small.lib.hfg_last_error(small.h)
    small.close()
    big = Context(CartesianBasis.build(water_cluster(32), "cc-pvdz"))  # n = 800
    n = big.n
    z = torch.zeros((n, n), dtype=torch.float64, device=dev)
    rc = noalloc(big, JKOptions.make(), 1, z, z, torch.empty_like(z), torch.empty_like(z))
    assert rc == 1 and b"8 MiB" in big.lib.hfg_last_error(big.h)
    big.close()
