"""Batched uneven sumchecks (salsaa_sumcheck_batch) against the CPU oracle,
bit-exact: instance i follows sum_check (src/subroutines/fast_norm_check.rs:
135-199) with the norm-check challenge stream of (round, repetition i)."""
import numpy as np
import pytest

from helpers import nc_challenges, rand_mod, small_signed
from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(gpu_lib, cuda):
    from salsaa_b200 import api as A
    return A


def _check(api, oracle, vecs, q, seed, rnd):
    claims, polys = api.sum_check_batch([api.to_dev(v) for v in vecs], q, seed, rnd)
    claims = api.to_host(claims)
    for i, v in enumerate(vecs):
        nr = v.size.bit_length() - 1
        cs = nc_challenges(seed, rnd, i, nr, q)
        claim, want, _ = oracle.sumcheck(v, q, cs)
        assert int(claims[i]) == claim, i
        assert np.array_equal(api.to_host(polys[i]), want), i


def test_sumcheck_batch_uneven(api, oracle):
    """Tail-only, one-level and two-level instances in one batch."""
    q = P.Q0
    rng = np.random.default_rng(41)
    logs = [4, 14, 15, 16, 19, 18, 1]
    vecs = [small_signed(rng, 1 << k, 1, q) if k % 2 else rand_mod(rng, 1 << k, q) for k in logs]
    _check(api, oracle, vecs, q, seed=12, rnd=3)


def test_sumcheck_batch_64_instances(api, oracle):
    q = P.Q1
    rng = np.random.default_rng(7)
    logs = rng.integers(10, 18, size=64)
    vecs = [small_signed(rng, 1 << int(k), 1, q) for k in logs]
    _check(api, oracle, vecs, q, seed=99, rnd=0)


@pytest.mark.slow
def test_sumcheck_batch_bench_instances(api, oracle, cuda):
    """The microbench's batch: 64 ternary instances with lengths log-uniform in
    2^16..2^22 (the same seeded draw), the 50-bit prime."""
    torch = cuda
    q = P.Q0
    rng = np.random.default_rng(2024)
    logs = np.sort(rng.integers(16, 23, size=64))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    vecs = [api.to_host(torch.randint(-1, 2, (1 << int(k),), dtype=torch.int64, device="cuda", generator=gen) % q)
            for k in logs]
    _check(api, oracle, vecs, q, seed=1, rnd=0)


def test_sumcheck_batch_wide_modulus(api, oracle):
    """q >= 2^50: exact residues instead of lazy 128-bit sums."""
    q = P.Q62
    rng = np.random.default_rng(3)
    vecs = [rand_mod(rng, 1 << 17, q), rand_mod(rng, 1 << 9, q)]
    _check(api, oracle, vecs, q, seed=5, rnd=1)


def test_sumcheck_batch_matches_single_call(api, oracle):
    """Instance 0 of a batch equals repetition 0 of the single-vector entry point."""
    q = P.Q0
    rng = np.random.default_rng(8)
    w = small_signed(rng, (1, 1 << 16), 1, q)
    claims, polys = api.sum_check(api.to_dev(w), 16, q, 21, 2)
    bc, bp = api.sum_check_batch([api.to_dev(w[0])], q, 21, 2)
    assert int(api.to_host(bc)[0]) == int(api.to_host(claims)[0])
    assert np.array_equal(api.to_host(bp[0]), api.to_host(polys)[0, :, 0, :])


def test_sumcheck_batch_rejects_bad_lengths(api):
    from salsaa_b200.api import SalsaaError
    with pytest.raises(SalsaaError):
        api.sum_check_batch([api.to_dev(np.zeros(100, dtype=np.uint64))], P.Q0, 1, 0)


@pytest.mark.parametrize("n_arg,incomplete,q", [(128, True, P.Q0), (256, True, P.Q1), (512, True, P.Q2),
                                                (64, False, P.Q62), (1024, False, P.Q62), (16, False, P.Q0)])
def test_ntt_multi_uneven(api, oracle, cuda, n_arg, incomplete, q):
    """64 uneven batches (some empty, some not a whole tile) in one launch,
    forward then inverse, equal one salsaa_ntt call per batch and the oracle."""
    torch = cuda
    rng = np.random.default_rng(n_arg)
    counts = [int(c) for c in rng.integers(0, 300, size=64)]
    counts[5] = 0
    counts[7] = 1
    xs = [rand_mod(rng, (c, n_arg), q) for c in counts]
    dev = [api.to_dev(x) for x in xs]
    fwd = api.ntt_multi(dev, n_arg, q, incomplete=incomplete, outs=[api.dev_empty(d.shape) for d in dev])
    single = [api.ntt(d, n_arg, q, incomplete=incomplete, out=api.dev_empty(d.shape)) if d.numel() else d
              for d in dev]
    back = api.ntt_multi([f.clone() for f in fwd], n_arg, q, inverse=True, incomplete=incomplete)  # in place
    torch.cuda.synchronize()
    for i, c in enumerate(counts):
        f = api.to_host(fwd[i])
        assert np.array_equal(f, api.to_host(single[i])), i
        assert np.array_equal(api.to_host(back[i]), xs[i]), i
    i = 8
    want = oracle.ring_to_slot(xs[i][:3], q) if incomplete else oracle.ntt_forward(xs[i][:3], q)
    assert np.array_equal(api.to_host(fwd[i])[:3], want)


def test_ntt_multi_rejects(api):
    from salsaa_b200.api import SalsaaError
    with pytest.raises(SalsaaError):  # n = 8 is below the register path
        api.ntt_multi([api.to_dev(np.zeros((4, 8), dtype=np.uint64))], 8, P.Q0)


def test_commit_multi_uneven(api, oracle):
    """Eight witnesses of uneven widths and row counts against one context's
    key rows in one tensor-core launch equal one salsaa_commit each and the
    oracle's parallel_dot_series_matrix."""
    p = P.make_params(128, P.Q0, 12, 1 << 15, 2, False)
    ctx = api.Context(p, crs_seed=4)
    rng = np.random.default_rng(17)
    shapes = [(1, 1 << 15), (3, 1 << 12), (9, 1 << 7), (2, 1 << 14), (1, 1 << 10), (5, 1 << 13), (4, 1 << 8),
              (2, 1 << 15)]
    ws = [small_signed(rng, (r, w, p.d), 3, p.q) for r, w in shapes]
    got = ctx.parallel_dot_series_matrix_multi([api.to_dev(w) for w in ws])
    for i, w in enumerate(ws):
        single = api.to_host(ctx.parallel_dot_series_matrix(api.to_dev(w)))
        assert np.array_equal(api.to_host(got[i]), single), i
    for i in (1, 2, 6):
        assert np.array_equal(api.to_host(got[i]), oracle.commit_ck(p, 4, ws[i])), i
    ctx.close()


def test_commit_multi_rejects(api):
    from salsaa_b200.api import SalsaaError
    p = P.make_params(128, P.Q0, 12, 1 << 12, 1, False)
    ctx = api.Context(p, crs_seed=4)
    with pytest.raises(SalsaaError):  # width below one 128-element chunk
        ctx.parallel_dot_series_matrix_multi([api.to_dev(np.zeros((1, 64, 128), dtype=np.uint64))])
    ctx.close()


def _fq2_challenges(seed, rnd, inst, nr, q):
    from helpers import domain, prf_np
    r = prf_np(seed, domain(6, rnd, inst), np.arange(2 * nr, dtype=np.uint64))
    return np.array([(int(x) * q) >> 64 for x in r], dtype=np.uint64).reshape(nr, 2)


@pytest.mark.parametrize("q", [P.Q0, P.Q62])
def test_sumcheck_fq2_batch(api, oracle, q):
    """The F_{q^2} norm-check sumcheck of uneven instances (one launch per
    round level) equals the oracle's restatement, every round polynomial."""
    rng = np.random.default_rng(23)
    logs = [1, 5, 10, 12, 13, 9, 16]
    vecs = [small_signed(rng, 1 << k, 1, q) for k in logs]
    shift = api.fq2_shift(q)
    assert shift == oracle.qnr(q)
    claims, polys = api.sum_check_fq2_batch([api.to_dev(v) for v in vecs], q, 31, 2)
    claims = api.to_host(claims)
    for i, v in enumerate(vecs):
        nr = v.size.bit_length() - 1
        cs = _fq2_challenges(31, 2, i, nr, q)
        claim, want, _ = oracle.sumcheck_fq2(v, q, shift, cs)
        assert int(claims[i]) == claim, i
        assert np.array_equal(api.to_host(polys[i]), want), i


@pytest.mark.slow
def test_sumcheck_fq2_bench_instances(api, oracle, cuda):
    """The microbench's batch (64 ternary instances, 2^16..2^22) over F_{q^2}."""
    torch = cuda
    q = P.Q0
    rng = np.random.default_rng(2024)
    logs = np.sort(rng.integers(16, 23, size=64))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    dev = [torch.randint(-1, 2, (1 << int(k),), dtype=torch.int64, device="cuda", generator=gen) % q for k in logs]
    shift = api.fq2_shift(q)
    claims, polys = api.sum_check_fq2_batch(dev, q, 1, 0)
    claims = api.to_host(claims)
    for i in (0, 31, 63):
        v = api.to_host(dev[i])
        cs = _fq2_challenges(1, 0, i, v.size.bit_length() - 1, q)
        claim, want, _ = oracle.sumcheck_fq2(v, q, shift, cs)
        assert int(claims[i]) == claim
        assert np.array_equal(api.to_host(polys[i]), want)
