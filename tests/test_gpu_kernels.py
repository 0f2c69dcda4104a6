"""CUDA kernels against the CPU oracle, bit-exact, through the C ABI."""
import numpy as np
import pytest

from helpers import fold_challenge, proj_challenge, rand_mod, small_signed
from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(gpu_lib, cuda):
    from salsaa_b200 import api as A
    return A


@pytest.mark.parametrize("n,q", [(2, 17), (8, 65537), (16, P.Q62), (32, P.Q62), (64, P.Q62), (128, P.Q62),
                                 (256, P.Q62), (512, P.Q62), (1024, P.Q62), (2048, P.Q62), (64, P.Q0), (128, P.Q1),
                                 (256, P.Q2), (4096, P.Q62), (8192, P.Q62), (16, P.Q0), (1024, P.Q0),
                                 (4096, P.Q0)])
def test_ntt_full(api, oracle, n, q):
    rng = np.random.default_rng(n)
    x = rand_mod(rng, (37, n), q)
    want = oracle.ntt_forward(x, q)
    d = api.to_dev(x)
    api.ntt(d, n, q)
    assert np.array_equal(api.to_host(d), want)
    api.ntt(d, n, q, inverse=True)
    assert np.array_equal(api.to_host(d), x)


@pytest.mark.parametrize("d,q", [(4, 17), (16, P.Q0), (32, P.Q62), (64, P.Q62), (128, P.Q0), (256, P.Q1),
                                 (512, P.Q2), (128, P.Q62), (1024, P.Q62), (4096, P.Q62), (8192, P.Q62),
                                 (32, P.Q0), (2048, P.Q0), (4096, P.Q0)])
def test_ntt_incomplete(api, oracle, d, q):
    rng = np.random.default_rng(d)
    x = rand_mod(rng, (53, d), q)
    if d <= 2048:
        want = oracle.ring_to_slot(x, q)
    else:  # beyond the oracle's ring size: [NTT(even) | NTT(odd)] by definition
        want = np.concatenate([oracle.ntt_forward(x[:, 0::2].copy(), q), oracle.ntt_forward(x[:, 1::2].copy(), q)],
                              axis=1)
    t = api.to_dev(x)
    out = api.dev_empty(t.shape)
    api.ntt(t, d, q, incomplete=True, out=out)
    assert np.array_equal(api.to_host(out), want)
    api.ntt(out, d, q, inverse=True, incomplete=True)
    assert np.array_equal(api.to_host(out), x)


@pytest.mark.parametrize("incomplete", [False, True])
def test_ntt_unaligned_and_out_of_place(api, oracle, incomplete):
    """Buffers that are only 8-byte aligned take the generic kernel; results agree."""
    import torch
    q, n = P.Q62, 256
    rng = np.random.default_rng(17)
    x = rand_mod(rng, (9, n), q)
    want = oracle.ring_to_slot(x, q) if incomplete else oracle.ntt_forward(x, q)
    big = torch.zeros(9 * n + 1, dtype=torch.int64, device="cuda")
    big[1:] = api.to_dev(x).view(-1)
    view = big[1:].view(9, n)
    out = api.dev_empty((9, n))
    api.ntt(view, n, q, incomplete=incomplete, out=out)
    assert np.array_equal(api.to_host(out), want)
    api.ntt(view, n, q, incomplete=incomplete)  # in place, unaligned
    assert np.array_equal(api.to_host(view), want)
    api.ntt(view, n, q, inverse=True, incomplete=incomplete)
    assert np.array_equal(api.to_host(view), x)


@pytest.mark.parametrize("offset", [0, 1, 2, 4])
def test_ntt_d128_paired_layouts(api, oracle, gpu_lib, offset):
    """d = 128 incomplete transforms with FP64 butterflies: 32-byte aligned
    buffers take the paired-half kernel, 16-byte aligned ones the one-half
    kernel, 8-byte aligned ones the generic kernel; all give the oracle's
    words, in place and out of place, with partial last tiles."""
    import ctypes
    import torch
    L = gpu_lib
    q, d = P.Q0, 128
    keys = [(6, 1, inv, 0, large) for inv in (0, 1) for large in (0, 1)]
    saved = []
    for k in keys:
        v, c = ctypes.c_int(), ctypes.c_int()
        assert L.salsaa_ntt_tune_get(*k, ctypes.byref(v), ctypes.byref(c)) == 0
        saved.append((v.value, c.value))
    try:
        for k in keys:
            assert L.salsaa_ntt_tune_set(*k, 1, 0) == 0
        rng = np.random.default_rng(40 + offset)
        for count in (1, 31, 33, 100):
            x = rand_mod(rng, (count, d), q)
            want = oracle.ring_to_slot(x, q)
            big = torch.zeros(count * d + 8, dtype=torch.int64, device="cuda")
            big[offset:offset + count * d] = api.to_dev(x).view(-1)
            view = big[offset:offset + count * d].view(count, d)
            obig = torch.zeros(count * d + 8, dtype=torch.int64, device="cuda")
            out = obig[offset:offset + count * d].view(count, d)
            api.ntt(view, d, q, incomplete=True, out=out)
            assert np.array_equal(api.to_host(out), want), count
            api.ntt(out, d, q, inverse=True, incomplete=True, out=view)
            assert np.array_equal(api.to_host(view), x), count
            api.ntt(view, d, q, incomplete=True)  # in place
            assert np.array_equal(api.to_host(view), want), count
            api.ntt(view, d, q, inverse=True, incomplete=True)
            assert np.array_equal(api.to_host(view), x), count
    finally:
        for k, (v, c) in zip(keys, saved):
            L.salsaa_ntt_tune_set(*k, v, c)


@pytest.mark.parametrize("offset", [0, 1, 2, 4])
@pytest.mark.parametrize("q", [P.Q62, P.Q0])
def test_ntt_n64_paired_layouts(api, oracle, offset, q):
    """Full 64-point transforms: 32-byte aligned buffers take the paired
    kernel (two polynomials per thread), others the one-polynomial kernel;
    both give the oracle's words, with odd counts and partial last tiles."""
    import torch
    n = 64
    rng = np.random.default_rng(60 + offset)
    for count in (1, 63, 64, 65, 129):
        x = rand_mod(rng, (count, n), q)
        want = oracle.ntt_forward(x, q)
        big = torch.zeros(count * n + 8, dtype=torch.int64, device="cuda")
        big[offset:offset + count * n] = api.to_dev(x).view(-1)
        view = big[offset:offset + count * n].view(count, n)
        obig = torch.zeros(count * n + 8, dtype=torch.int64, device="cuda")
        out = obig[offset:offset + count * n].view(count, n)
        api.ntt(view, n, q, out=out)
        assert np.array_equal(api.to_host(out), want), count
        api.ntt(out, n, q, inverse=True, out=view)
        assert np.array_equal(api.to_host(view), x), count
        api.ntt(view, n, q)  # in place
        assert np.array_equal(api.to_host(view), want), count
        api.ntt(view, n, q, inverse=True)
        assert np.array_equal(api.to_host(view), x), count


def test_ntt_ragged_tiles(api, oracle):
    """Batch sizes that leave the last tile of 4096 coefficients partly empty."""
    q = P.Q0
    rng = np.random.default_rng(23)
    for count in (1, 31, 33, 95):
        x = rand_mod(rng, (count, 128), q)
        out = api.dev_empty(x.shape)
        api.ntt(api.to_dev(x), 128, q, incomplete=True, out=out)
        assert np.array_equal(api.to_host(out), oracle.ring_to_slot(x, q))
        y = rand_mod(rng, (count, 1024), P.Q62)
        t = api.to_dev(y)
        api.ntt(t, 1024, P.Q62)
        assert np.array_equal(api.to_host(t), oracle.ntt_forward(y, P.Q62))


@pytest.mark.parametrize("n,q,count", [(16, P.Q62, 7), (64, P.Q62, 65), (128, P.Q0, 33), (256, P.Q62, 17),
                                       (1024, P.Q62, 9), (4096, P.Q62, 3), (8, 65537, 5), (8192, P.Q62, 2),
                                       (1024, P.Q0, 5), (4096, P.Q0, 3), (16, P.Q1, 9)])
def test_poly_mul(api, oracle, n, q, count):
    """Batched negacyclic product against the oracle's multiply_poly, per pair."""
    rng = np.random.default_rng(n + count)
    a, b = rand_mod(rng, (count, n), q), rand_mod(rng, (count, n), q)
    got = api.to_host(api.poly_mul(api.to_dev(a), api.to_dev(b), n, q))
    for i in range(count):
        assert np.array_equal(got[i], oracle.multiply_poly(a[i], b[i], q)), i


def test_poly_mul_in_place_and_unaligned(api, oracle):
    import torch
    q, n, count = P.Q62, 64, 5
    rng = np.random.default_rng(2)
    a, b = rand_mod(rng, (count, n), q), rand_mod(rng, (count, n), q)
    want = np.stack([oracle.multiply_poly(a[i], b[i], q) for i in range(count)])
    ta, tb = api.to_dev(a), api.to_dev(b)
    api.poly_mul(ta, tb, n, q, out=ta)  # r aliases a
    assert np.array_equal(api.to_host(ta), want)
    big = torch.zeros(count * n + 1, dtype=torch.int64, device="cuda")
    big[1:] = api.to_dev(a).view(-1)
    va = big[1:].view(count, n)
    got = api.poly_mul(va, tb, n, q)  # 8-byte aligned input: three-pass path
    assert np.array_equal(api.to_host(got), want)


def test_ntt_large_batch(api, oracle):
    q, n = P.Q62, 1024
    rng = np.random.default_rng(9)
    x = rand_mod(rng, (1 << 14, n), q)
    t = api.to_dev(x)
    api.ntt(t, n, q)
    got = api.to_host(t)
    idx = rng.choice(x.shape[0], 64, replace=False)
    assert np.array_equal(got[idx], oracle.ntt_forward(x[idx], q))
    api.ntt(t, n, q, inverse=True)
    assert np.array_equal(api.to_host(t), x)


@pytest.mark.parametrize("d,q,ms,width,rows", [(16, P.Q0, 3, 64, 1), (16, P.Q0, 5, 4096, 3), (128, P.Q0, 12, 2048, 2),
                                               (256, P.Q1, 7, 1024, 4), (512, P.Q2, 4, 512, 8),
                                               (32, P.Q62, 2, 256, 2), (64, P.Q0, 3, 8192, 1),
                                               (128, P.Q0, 18, 4096, 9), (128, P.Q0, 13, 2048, 9),
                                               (256, P.Q1, 1, 128, 1), (16, P.Q0, 12, 16384, 7),
                                               (4, P.Q0, 2, 256, 3)])
def test_commit(api, oracle, d, q, ms, width, rows):
    p = P.make_params(d, q, ms, max(width, 16), 1)
    rng = np.random.default_rng(d + width)
    w = rand_mod(rng, (rows, width, d), q)
    want = oracle.commit_ck(p, 21, w)
    ctx = api.Context(p, crs_seed=21)
    got = api.to_host(ctx.parallel_dot_series_matrix(api.to_dev(w)))
    assert np.array_equal(got, want)


def test_commit_prefix_layer(api, oracle):
    """A witness narrower than WIT_LEN uses the matching expanded layer (a prefix of the powers)."""
    p = P.make_params(16, P.Q0, 3, 1 << 14, 1)
    rng = np.random.default_rng(3)
    w = small_signed(rng, (2, 4096, 16), 5, p.q)
    ctx = api.Context(p, crs_seed=4)
    got = api.to_host(ctx.parallel_dot_series_matrix(api.to_dev(w)))
    assert np.array_equal(got, oracle.commit_ck(p, 4, w))


@pytest.mark.parametrize("rows,n,d,q", [(1, 4, 4, P.Q0), (1, 1 << 12, 16, P.Q0), (3, 1 << 15, 128, P.Q0),
                                        (2, 1 << 13, 64, P.Q62), (4, 1 << 16, 256, P.Q1)])
def test_sumcheck(api, oracle, rows, n, d, q):
    from helpers import nc_challenges
    rng = np.random.default_rng(n + rows)
    w = rand_mod(rng, (rows, n), q)
    seed, rnd = 99, 3
    claims, polys = api.sum_check(api.to_dev(w), d, q, seed, rnd)
    claims, polys = api.to_host(claims), api.to_host(polys)
    nr = n.bit_length() - 1
    for rep in range(2):
        cs = nc_challenges(seed, rnd, rep, nr, q)
        for k in range(rows):
            claim, want, _ = oracle.sumcheck(w[k], q, cs)
            assert int(claims[k]) == claim
            assert np.array_equal(polys[rep, :, k, :], want)


def _check_sumcheck(api, oracle, w, d, q, seed=99, rnd=3):
    from helpers import nc_challenges
    rows, n = w.shape
    claims, polys = api.sum_check(api.to_dev(w), d, q, seed, rnd)
    claims, polys = api.to_host(claims), api.to_host(polys)
    nr = n.bit_length() - 1
    for rep in range(2):
        cs = nc_challenges(seed, rnd, rep, nr, q)
        for k in range(rows):
            claim, want, _ = oracle.sumcheck(w[k], q, cs)
            assert int(claims[k]) == claim
            assert np.array_equal(polys[rep, :, k, :], want)


@pytest.mark.parametrize("rows,n,d,q,bound", [(1, 1 << 15, 128, P.Q0, 1), (3, 1 << 16, 128, P.Q0, 1 << 24),
                                              (2, 1 << 17, 64, P.Q1, 1 << 30), (1, 1 << 20, 128, P.Q0, 1 << 25),
                                              (16, 1 << 15, 16, P.Q2, 1 << 12)])
def test_sumcheck_small(api, oracle, rows, n, d, q, bound):
    """Small centred witnesses (ternary, decomposition digits): the first
    pass runs on the tensor cores through the groups' Gram matrices."""
    rng = np.random.default_rng(n + rows + bound)
    _check_sumcheck(api, oracle, small_signed(rng, (rows, n), bound, q), d, q)


@pytest.mark.slow
@pytest.mark.parametrize("logn,bound", [(22, 1), (23, 1 << 12), (24, 1)])
def test_sumcheck_full_size(api, oracle, logn, bound):
    """Norm-check sumchecks at 2^22..2^24 coefficients (ternary, and
    decomposition-digit sized), every round polynomial of both repetitions."""
    rng = np.random.default_rng(logn)
    _check_sumcheck(api, oracle, small_signed(rng, (1, 1 << logn), bound, P.Q0), 128, P.Q0)


@pytest.mark.parametrize("outside", [0, 1, 2])
def test_sumcheck_limb_edges(api, oracle, outside):
    """Values at the ends of the four-signed-byte range stay on the tensor
    cores; one value beyond either end sends the launch to the exact pass."""
    q, n = P.Q0, 1 << 16
    rng = np.random.default_rng(5)
    w = small_signed(rng, (2, n), 3, q)
    hi, lo = 0x7F7F7F7F, 0x80808080
    w[0, 17] = hi
    w[0, 40000] = q - lo
    w[1, 3] = q - lo
    w[1, n - 1] = hi
    if outside == 1:
        w[1, 1234] = hi + 1
    elif outside == 2:
        w[0, 999] = q - lo - 1
    _check_sumcheck(api, oracle, w, 128, q)


@pytest.mark.parametrize("parts", [1, 2, 3])
def test_decompose(api, oracle, parts):
    q, d = P.Q0, 128
    rng = np.random.default_rng(parts)
    w = small_signed(rng, (2, 1024, d), 1 << 13, q)
    want, radix = oracle.decompose(w, q, parts)
    got, gr = api.decompose_matrix_by_chunks(api.to_dev(w), q, parts)
    assert int(api.to_host(gr)[0]) == radix
    assert np.array_equal(api.to_host(got), want)


def test_decompose_zero_and_full_range(api, oracle):
    q, d = P.Q0, 16
    z = np.zeros((2, 64, d), dtype=np.uint64)
    got, gr = api.decompose_matrix_by_chunks(api.to_dev(z), q, 2)
    assert int(api.to_host(gr)[0]) == 1 and not api.to_host(got).any()
    rng = np.random.default_rng(1)
    w = rand_mod(rng, (1, 64, d), q)
    want, radix = oracle.decompose(w, q, 2)
    got, gr = api.decompose_matrix_by_chunks(api.to_dev(w), q, 2)
    assert int(api.to_host(gr)[0]) == radix
    assert np.array_equal(api.to_host(got), want)


@pytest.mark.parametrize("rows,width,d,q", [(1, 256, 16, P.Q0), (2, 2048, 128, P.Q0), (4, 4096, 64, P.Q1),
                                            (8, 2048, 16, P.Q0), (2, 1024, 32, P.Q62)])
def test_project(api, oracle, rows, width, d, q):
    rng = np.random.default_rng(rows * width)
    w = rand_mod(rng, (rows, width, d), q)
    seed, rnd = 5, 2
    iz, sg = proj_challenge(seed, rnd, rows * 256)
    want = oracle.project(w, q, iz, sg)
    got = api.to_host(api.project(api.to_dev(w), q, seed, rnd))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("rows,width,d,bound", [(2, 2048, 128, 1), (8, 4096, 128, 127), (4, 2048, 256, 128),
                                                 (2, 1024, 512, 60), (1, 512, 128, 129)])
def test_project_small_values(api, oracle, rows, width, d, bound):
    """Witness values in int8 range take the tensor-core path; bound 129 forces
    the exact fallback for some values."""
    q = P.Q0
    rng = np.random.default_rng(bound + d)
    w = small_signed(rng, (rows, width, d), bound, q)
    if bound == 128:
        w[0, 0, :] = q - 128  # the int8 edge
    seed, rnd = 8, 5
    iz, sg = proj_challenge(seed, rnd, rows * 256)
    want = oracle.project(w, q, iz, sg)
    got = api.to_host(api.project(api.to_dev(w), q, seed, rnd))
    assert np.array_equal(got, want)


def test_project_too_narrow_rejected(api):
    from salsaa_b200.api import SalsaaError
    w = api.to_dev(np.zeros((4, 512, 16), dtype=np.uint64))
    with pytest.raises(SalsaaError):
        api.project(w, P.Q0, 1, 0)


@pytest.mark.parametrize("rows,width,d,q", [(2, 512, 16, P.Q0), (8, 1024, 128, P.Q0), (3, 256, 512, P.Q2),
                                            (2, 128, 32, P.Q62), (16, 256, 128, P.Q0), (5, 128, 4, P.Q1),
                                            (7, 64, 64, P.Q62)])
def test_fold(api, oracle, rows, width, d, q):
    rng = np.random.default_rng(rows + d)
    w = rand_mod(rng, (rows, width, d), q)
    c = fold_challenge(11, 0, rows, d, q)
    want = oracle.fold(w, q, c)
    got = api.to_host(api.fold(api.to_dev(w), q, api.to_dev(c)))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n,k", [(16, 32), (112, 128), (176, 128), (256, 256), (128, 64)])
def test_umma_i8_selftest(api, n, k):
    """tcgen05.mma kind::i8 with our shared-memory descriptors equals the exact integer product."""
    rng = np.random.default_rng(n * k)
    a = rng.integers(0, 256, size=(128, k), dtype=np.uint8)
    b = rng.integers(0, 256, size=(n, k), dtype=np.uint8)
    a[0, :] = 255
    b[0, :] = 255
    got = api.selftest_umma_i8(a, b)
    want = a.astype(np.int64) @ b.astype(np.int64).T
    assert np.array_equal(got.astype(np.int64), want)


# ---- HEXL-compatible tier (host buffers, GPU compute) ---------------------------
def test_hexl_compat_eltwise(api, oracle):
    q = P.Q62
    rng = np.random.default_rng(0)
    a, b = rand_mod(rng, 5000, q), rand_mod(rng, 5000, q)
    for name, op in [("eltwise_mult_mod", "mult"), ("eltwise_add_mod", "add"), ("eltwise_sub_mod", "sub")]:
        r = np.zeros_like(a)
        api.hexl_call(name, r, a, b, a.size, q)
        assert np.array_equal(r, oracle.eltwise(op, a, b, q)), name
    r = np.zeros_like(a)
    api.hexl_call("eltwise_fma_mod", r, a, 12345, b, a.size, q)
    assert np.array_equal(r, oracle.eltwise_fma(a, 12345, b, q))
    big = rng.integers(0, 2 ** 63, size=1000, dtype=np.uint64)
    r = np.zeros_like(big)
    api.hexl_call("eltwise_reduce_mod", r, big, big.size, q)
    assert np.array_equal(r, big % np.uint64(q))
    assert api.hexl_call("sum", a, a.size, q) == oracle.sum_mod(a, q)
    assert api.hexl_call("sum_sq", a, a.size, q) == oracle.sum_sq(a, q)
    assert api.hexl_call("sum_fast", a, a.size, q) == oracle.sum_mod(a, q)
    assert api.hexl_call("sum_sq_fast", a, a.size, q) == oracle.sum_sq(a, q)


def test_hexl_compat_kats(api):
    """The reference's HEXL-boundary tests (src/hexl/bindings.rs:99-148) against this library."""
    r = np.zeros(5, dtype=np.uint64)
    api.hexl_call("eltwise_mult_mod", r, np.array([1, 2, 3, 4, 5], dtype=np.uint64),
                  np.array([6, 7, 8, 9, 10], dtype=np.uint64), 5, 100)
    assert r.tolist() == [6, 14, 24, 36, 50]
    a = np.array([1, 2, 3, 1, 0, 0, 0, 0], dtype=np.uint64)
    b = np.array([8, 7, 6, 1, 0, 0, 0, 0], dtype=np.uint64)
    r = np.zeros(8, dtype=np.uint64)
    api.hexl_call("multiply_poly", r, a, b, 8, 65537)
    want = [0] * 8
    for i in range(4):
        for j in range(4):
            want[i + j] = (want[i + j] + int(a[i]) * int(b[j])) % 65537
    assert r.tolist() == want
    assert api.hexl_call("sum_sq", np.arange(1, 9, dtype=np.uint64), 8, 71) == 62


def test_hexl_compat_ntt(api, oracle):
    q = P.Q62
    rng = np.random.default_rng(4)
    for n in (4, 64, 1024):
        x = rand_mod(rng, n, q)
        y = x.copy()
        api.hexl_call("ntt_forward_in_place", y, n, q)
        assert np.array_equal(y, oracle.ntt_forward(x, q))
        api.hexl_call("ntt_inverse_in_place", y, n, q)
        assert np.array_equal(y, x)
