"""Batched J/K builds over several molecules (hfg_jk_device_batch).

One launch per angular class and precision covers the work queues of every
molecule of the batch.  Each molecule's J and K must equal its own build
(hfg_jk, itself checked against the oracle and hf-rs's golden matrices
elsewhere) up to FP64 summation order, for molecules of different sizes and
basis sets in one batch, in FP64 and mixed precision, on two calls in a row
(the accumulators are reused and must be cleared).
"""
import numpy as np
import pytest

from hfgpu import CartesianBasis, Context, HfgError, JKOptions
from hfgpu.clusters import water_cluster

pytestmark = pytest.mark.gpu

MOLECULES = [(1, "sto-3g"), (2, "cc-pvdz"), (3, "6-31g*"), (1, "cc-pvdz"), (4, "6-31g"), (2, "sto-3g")]


def rand_sym(n, seed):
    a = np.random.default_rng(seed).standard_normal((n, n)) * 0.3
    return a + a.T


@pytest.fixture(scope="module")
def contexts():
    ctxs = [Context(CartesianBasis.build(water_cluster(w, seed=17 + i), b)) for i, (w, b) in enumerate(MOLECULES)]
    yield ctxs
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("mixed", [None, 1e-6])
def test_batch_matches_each_molecules_own_build(contexts, mixed):
    import torch
    dev = torch.device("cuda", 0)
    opts = JKOptions.make(mixed=mixed)
    for call in range(2):
        P = [rand_sym(c.n, 100 * call + i) for i, c in enumerate(contexts)]
        ref = [c.jk(p, opts=opts) for c, p in zip(contexts, P)]
        dP = [torch.from_numpy(p).to(dev) for p in P]
        dJ = [torch.full((c.n, c.n), np.nan, dtype=torch.float64, device=dev) for c in contexts]
        dK = [torch.full((c.n, c.n), np.nan, dtype=torch.float64, device=dev) for c in contexts]
        torch.cuda.synchronize()
        Context.jk_device_batch(contexts, [t.data_ptr() for t in dP], [t.data_ptr() for t in dJ],
                                [t.data_ptr() for t in dK], opts=opts)
        torch.cuda.synchronize()
        for i, (J_ref, K_ref) in enumerate(ref):
            scale = max(1.0, np.abs(J_ref).max())
            assert np.max(np.abs(dJ[i].cpu().numpy() - J_ref)) < 1e-11 * scale, (call, i)
            assert np.max(np.abs(dK[i].cpu().numpy() - K_ref[0])) < 1e-11 * scale, (call, i)


def test_batch_of_one_and_input_errors(contexts):
    import torch
    dev = torch.device("cuda", 0)
    c = contexts[1]
    P = rand_sym(c.n, 5)
    J_ref, K_ref = c.jk(P)
    dP = torch.from_numpy(P).to(dev)
    dJ = torch.empty((c.n, c.n), dtype=torch.float64, device=dev)
    dK = torch.empty_like(dJ)
    torch.cuda.synchronize()
    Context.jk_device_batch([c], [dP.data_ptr()], [dJ.data_ptr()], [dK.data_ptr()])
    torch.cuda.synchronize()
    assert np.max(np.abs(dJ.cpu().numpy() - J_ref)) < 1e-11 * np.abs(J_ref).max()
    assert np.max(np.abs(dK.cpu().numpy() - K_ref[0])) < 1e-11 * np.abs(J_ref).max()
    # one context twice would share its accumulators: rejected before any work
    with pytest.raises(HfgError, match="twice"):
        Context.jk_device_batch([c, c], [dP.data_ptr()] * 2, [dJ.data_ptr()] * 2, [dK.data_ptr()] * 2)
    with pytest.raises(HfgError, match="null pointer"):
        Context.jk_device_batch([c], [0], [dJ.data_ptr()], [dK.data_ptr()])
    with pytest.raises(ValueError):
        Context.jk_device_batch([c], [dP.data_ptr()], [], [dK.data_ptr()])
