"""Dense ring-matrix commitment C = A * W (parallel_dot_matrix_matrix,
src/arithmetic.rs:429-457) on the GPU against the CPU oracle, bit-exact."""
import numpy as np
import pytest

from helpers import rand_mod, small_signed
from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(gpu_lib, cuda):
    from salsaa_b200 import api as A
    return A


@pytest.mark.parametrize("n,m,d,q,r,digits", [
    (8, 256, 128, P.Q0, 1, 0),        # tensor cores, one column
    (8, 256, 128, P.Q0, 12, 16),      # two column groups, base-16 digits
    (16, 128, 64, P.Q1, 3, 2),        # base-2 digits
    (18, 512, 16, P.Q0, 9, 0),        # largest tensor-core key (256 byte rows)
    (16, 4096, 128, P.Q0, 2, 16),     # several element blocks
    (20, 128, 32, P.Q0, 2, 0),        # more than 18 key rows: CUDA cores
    (4, 256, 32, P.Q62, 5, 0),        # q >= 2^56: CUDA cores
])
def test_dense_commit(api, oracle, n, m, d, q, r, digits):
    rng = np.random.default_rng(n * m + r)
    A = rand_mod(rng, (n, m, d), q)
    W = small_signed(rng, (r, m, d), digits // 2, q) if digits else rand_mod(rng, (r, m, d), q)
    want = oracle.dense_commit(A, W, q)
    key = api.DenseKey(api.to_dev(A), q)
    got = api.to_host(key.commit(api.to_dev(W)))
    assert np.array_equal(got, want)
    ws = api.dev_empty((r, m, d))
    got2 = api.to_host(key.commit(api.to_dev(W), w_slot=ws))  # caller-provided workspace, second call
    assert np.array_equal(got2, want)
    key.close()


@pytest.mark.slow
@pytest.mark.parametrize("n", [8, 16])
@pytest.mark.parametrize("r", [1, 8, 32])
@pytest.mark.parametrize("b", [2, 16])
def test_dense_commit_full_size(api, oracle, n, r, b):
    """The microbench shapes: m = 2^16 ring elements of degree 128 at the 50-bit
    prime, W base-b digits in [-b/2, b/2).  The GPU computes all n x r outputs;
    the oracle recomputes the first and last key rows against three columns."""
    import torch
    q, m, d = P.Q0, 1 << 16, 128
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1000 * n + 10 * r + b)
    A = torch.randint(0, 1 << 62, (n, m, d), dtype=torch.int64, device="cuda", generator=gen) % q
    W = torch.randint(-(b // 2), b // 2, (r, m, d), dtype=torch.int64, device="cuda", generator=gen) % q
    key = api.DenseKey(A, q)
    got = api.to_host(key.commit(W))
    key.close()
    rows = sorted({0, n - 1})
    cols = sorted({0, r // 2, r - 1})
    A_s = api.to_host(A[rows])
    W_s = api.to_host(W[cols])
    del A, W
    want = oracle.dense_commit(A_s, W_s, q)
    assert np.array_equal(got[np.ix_(rows, cols)], want)


def test_dense_commit_rejects_bad_shapes(api):
    from salsaa_b200.api import SalsaaError
    with pytest.raises(SalsaaError):
        api.DenseKey(api.to_dev(np.zeros((2, 100, 16), dtype=np.uint64)), P.Q0)
