"""tcgen05 TF32 tensor-core building blocks (shared-memory descriptors, TMEM
accumulators, hi/lo split) against an FP64 product on the host."""
import numpy as np
import pytest

from spoc_b200 import api

SHAPES = [(8, 8, 16), (36, 40, 48), (42, 48, 144), (27, 32, 32)]


@pytest.mark.gpu
@pytest.mark.parametrize("K,kpad,n", SHAPES)
def test_split_tf32_product(K, kpad, n):
    rng = np.random.default_rng(K * 100 + n)
    A = rng.normal(size=(128, K)).astype(np.float32)
    B = rng.normal(size=(n, K)).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T
    d3 = api.tc_selftest(A, B, kpad, 1)
    d1 = api.tc_selftest(A, B, kpad, 0)
    e3 = np.max(np.abs(d3 - ref) / scale)
    e1 = np.max(np.abs(d1 - ref) / scale)
    assert e3 < 2e-6, e3          # three-term split: FP32-level accuracy
    assert 1e-5 < e1 < 2e-3, e1   # one TF32 product: 10-bit mantissa operands


@pytest.mark.gpu
def test_accumulate_onto_stored_tmem():
    rng = np.random.default_rng(7)
    A = rng.normal(size=(128, 36)).astype(np.float32)
    B = rng.normal(size=(48, 36)).astype(np.float32)
    D0 = rng.normal(size=(128, 48)).astype(np.float32)
    ref = D0.astype(np.float64) + A.astype(np.float64) @ B.astype(np.float64).T
    d = api.tc_selftest(A, B, 40, 1, D0)
    assert np.max(np.abs(d - ref)) < 1e-4 * np.max(np.abs(ref))
