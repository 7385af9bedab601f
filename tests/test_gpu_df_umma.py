"""The DF exchange on the tensor cores (tcgen05 kernels of df_umma.cu).

K = 2 sum_Q (B_Q C)(B_Q C)^T with BF16 or TF32 operands and FP32
accumulation, against the FP64 exchange of an FP64-stored factor (the same
as the oracle's df_jk to 1e-10, tests/test_gpu_df.py).  Stated bounds on the
relative Frobenius error of K: 1e-2 for BF16 operands (8-bit mantissas of
B, C and T, rounded), 5e-3 for TF32 (10-bit mantissas; the tensor cores
truncate the FP32 operands, which doubles the rounding error).  Also: the result does not depend on
how the auxiliary functions are chunked, it agrees with cuBLAS's GEMMs on
the same operands, and sizes that are not multiples of the tile shapes
(n < 16, odd nocc) work.
"""
import numpy as np
import pytest

from hfgpu import CartesianBasis, Context
from hfgpu.clusters import water_cluster
from hfgpu.lib import HFG_DF_BF16, HFG_DF_FP32, HFG_DF_FP64, DFTensor

pytestmark = pytest.mark.gpu

BOUND = {HFG_DF_BF16: 1e-2, HFG_DF_FP32: 5e-3}


def occ(n, nocc, seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, max(n, nocc))))
    return np.ascontiguousarray(q[:, :nocc])


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def h2o4():
    atoms = water_cluster(4)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    C = occ(ctx.n, 20, 1)
    J64, K64 = DFTensor(ctx, aux).jk(C)
    yield ctx, aux, C, J64, K64
    ctx.close()


@pytest.mark.parametrize("mma", [HFG_DF_BF16, HFG_DF_FP32])
def test_tensor_core_exchange_vs_fp64(h2o4, mma):
    ctx, aux, C, J64, K64 = h2o4
    d = DFTensor(ctx, aux, storage=HFG_DF_FP32)
    J, K = d.jk(C, mma=mma)
    assert np.all(np.isfinite(K))
    assert np.max(np.abs(K - K.T)) == 0.0  # completed from one triangle
    assert rel(K, K64) < BOUND[mma], rel(K, K64)
    assert rel(J, J64) < 1e-6  # J: FP64 accumulation over the FP32 factor
    d.close()


@pytest.mark.parametrize("mma", [HFG_DF_BF16, HFG_DF_FP32])
def test_tensor_core_exchange_agrees_with_cublas(h2o4, mma, monkeypatch):
    ctx, aux, C, _, K64 = h2o4
    d = DFTensor(ctx, aux, storage=HFG_DF_FP32)
    _, K = d.jk(C, mma=mma)
    monkeypatch.setenv("HFG_DF_K_CUBLAS", "1")
    _, Kb = d.jk(C, mma=mma)
    monkeypatch.delenv("HFG_DF_K_CUBLAS")
    # both round the same operands; they differ by accumulation order and
    # by where T is rounded
    assert rel(K, Kb) < BOUND[mma], rel(K, Kb)
    d.close()


def test_tensor_core_exchange_chunking_invariant(h2o4, monkeypatch):
    ctx, aux, C, _, _ = h2o4
    d = DFTensor(ctx, aux, storage=HFG_DF_FP32)
    _, K1 = d.jk(C, mma=HFG_DF_BF16)
    monkeypatch.setenv("HFG_DF_K_CHUNK", "7")  # ~76 chunks of 7 auxiliary functions
    _, K2 = d.jk(C, mma=HFG_DF_BF16)
    monkeypatch.delenv("HFG_DF_K_CHUNK")
    assert rel(K2, K1) < 1e-5
    d.close()


@pytest.mark.parametrize("nw,orb,auxname,nocc", [(1, "sto-3g", "def2-svp-ri", 5), (3, "6-31g*", "def2-universal-jkfit", 13),
                                                  (2, "cc-pvdz", "def2-universal-jkfit", 37)])
@pytest.mark.parametrize("mma", [HFG_DF_BF16, HFG_DF_FP32])
def test_tensor_core_exchange_odd_sizes(nw, orb, auxname, nocc, mma):
    atoms = water_cluster(nw)
    ctx = Context(CartesianBasis.build(atoms, orb))
    aux = CartesianBasis.build(atoms, auxname)
    C = occ(ctx.n, nocc, 2)
    _, K64 = DFTensor(ctx, aux).jk(C)
    _, K = DFTensor(ctx, aux, storage=HFG_DF_FP32).jk(C, mma=mma)
    assert rel(K, K64) < BOUND[mma], (ctx.n, rel(K, K64))
    ctx.close()


def test_bf16_stored_factor_on_the_tensor_cores(h2o4):
    ctx, aux, C, _, K64 = h2o4
    d = DFTensor(ctx, aux, storage=HFG_DF_BF16)
    _, K = d.jk(C, mma=HFG_DF_BF16)
    assert rel(K, K64) < 2e-2
    d.close()
