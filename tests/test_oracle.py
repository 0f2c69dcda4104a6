"""The CPU oracle against the reference's own known-answer tests and the
properties its property tests check (src/**/#[test]).  CPU only."""
import json
import os

import numpy as np
import pytest

from helpers import DOM_NC, domain, nc_challenges, prf_np, rand_mod, small_signed
from salsaa_b200 import params as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kats.json")


@pytest.fixture(scope="module")
def kats():
    with open(GOLDEN) as f:
        return {k["name"]: k for k in json.load(f)}


def test_kat_multiply_mod(oracle, kats):
    k = kats["multiply_mod"]
    assert oracle.mul_mod(k["a"], k["b"], k["q"]) == k["expect"]


def test_kat_eltwise_mult_mod(oracle, kats):
    k = kats["eltwise_mult_mod"]
    assert oracle.eltwise("mult", k["a"], k["b"], k["q"]).tolist() == k["expect"]


def test_kat_multiply_poly(oracle, kats):
    k = kats["multiply_poly"]
    assert oracle.multiply_poly(k["a"], k["b"], k["q"]).tolist() == k["expect"]


@pytest.mark.parametrize("name,op", [("ring_add", "add"), ("ring_sub", "sub")])
def test_kat_ring_add_sub(oracle, kats, name, op):
    k = kats[name]
    assert oracle.eltwise(op, k["a"], k["b"], k["q"]).tolist() == k["expect"]


def test_kat_ring_mul(oracle, kats):
    k = kats["ring_mul"]
    assert oracle.ring_mul(k["a"], k["b"], k["q"]).tolist() == k["expect"]


def _quad_mul(O, a, b, shift, q):
    # QuadraticExtension::mul, src/quadratic_extension.rs:30-58
    return [O.add_mod(O.mul_mod(a[0], b[0], q), O.mul_mod(shift, O.mul_mod(a[1], b[1], q), q), q),
            O.add_mod(O.mul_mod(a[0], b[1], q), O.mul_mod(a[1], b[0], q), q)]


def test_kat_quadratic_extension(oracle, kats):
    k = kats["quadratic_add"]
    assert [oracle.add_mod(x, y, k["q"]) for x, y in zip(k["a"], k["b"])] == k["expect"]
    k = kats["quadratic_mul"]
    assert _quad_mul(oracle, k["a"], k["b"], k["shift"], k["q"]) == k["expect"]


def test_slot_product_is_quadratic_extension_product(oracle):
    """The incomplete-NTT slot product equals the F_q[X]/(X^2 - zeta_i) product
    of src/cyclotomic_ring.rs:629-660 (to_and_from_quadratic_fields_with_multiplication)."""
    q, d = P.Q0, 16
    rng = np.random.default_rng(1)
    a, b = rand_mod(rng, d, q), rand_mod(rng, d, q)
    sa, sb = oracle.ring_to_slot(a, q), oracle.ring_to_slot(b, q)
    zeta = oracle.shift_factors(d, q)
    n = d // 2
    prod = oracle.ring_to_slot(oracle.ring_mul(a, b, q), q)
    for s in range(n):
        e, o = _quad_mul(oracle, [int(sa[s]), int(sa[n + s])], [int(sb[s]), int(sb[n + s])], int(zeta[s]), q)
        assert (e, o) == (int(prod[s]), int(prod[n + s]))


def test_kat_tensor(oracle, kats):
    k = kats["tensor"]
    assert oracle.tensor(k["cs"], k["q"]).tolist() == k["expect"]


def test_kat_sum_sq(oracle, kats):
    k = kats["sum_sq"]
    assert oracle.sum_sq(k["a"], k["q"]) == k["expect"]


def test_kat_split(oracle, kats):
    """test_split (src/subroutines/split.rs:109-143): constants as ring elements."""
    k = kats["split"]
    q, d = k["q"], k["d"]

    def const(v):
        x = np.zeros(d, dtype=np.uint64)
        x[0] = v % q
        return x

    def dot(row, wit):
        acc = np.zeros(d, dtype=np.uint64)
        for r, w in zip(row, wit):
            acc = oracle.eltwise("add", acc, oracle.ring_mul(const(r), const(w), q), q)
        return int(acc[0])

    assert dot(k["layers"][0], k["witness"]) == k["expect_rhs"]
    half = len(k["witness"]) // 2
    left, right = k["witness"][:half], k["witness"][half:]
    assert [left, right] == k["expect_split_witness"]
    got = [dot(k["layers"][1], left), dot(k["layers"][1], right)]
    assert got == k["expect_split_rhs"]
    # verifier_split relation with the layer's tensor factor (1, 16)
    t = k["tensors"][0]
    assert (t[0] * got[0] + t[1] * got[1]) % q == k["expect_rhs"]


def test_ntt_is_hexl_convention(oracle):
    """Forward output i is A(psi^(2*bitrev(i)+1)), psi the minimal 2n-th root."""
    q, n = P.Q62, 32
    psi = oracle.minimal_root(2 * n, q)
    assert pow(psi, n, q) == q - 1
    rng = np.random.default_rng(2)
    a = rand_mod(rng, n, q)
    A = oracle.ntt_forward(a, q)
    bits = n.bit_length() - 1
    for i in range(n):
        br = int(format(i, "0%db" % bits)[::-1], 2)
        pt = pow(psi, 2 * br + 1, q)
        assert int(A[i]) == sum(int(a[j]) * pow(pt, j, q) for j in range(n)) % q
    assert np.array_equal(oracle.ntt_inverse(A, q), a)
    # minimality: no odd power of psi is smaller
    assert all(pow(psi, 2 * i + 1, q) >= psi for i in range(n))


@pytest.mark.parametrize("d,q", [(16, P.Q0), (32, P.Q1), (64, P.Q2), (128, P.Q0), (32, P.Q62)])
def test_ring_mul_matches_schoolbook(oracle, d, q):
    rng = np.random.default_rng(d)
    a, b = rand_mod(rng, d, q), rand_mod(rng, d, q)
    r = oracle.ring_mul(a, b, q)
    z = [0] * d
    for i in range(d):
        for j in range(d):
            t = int(a[i]) * int(b[j])
            if i + j < d:
                z[i + j] = (z[i + j] + t) % q
            else:
                z[i + j - d] = (z[i + j - d] - t) % q
    assert [int(v) for v in r] == z


def test_conjugate_homomorphism(oracle):
    """multiply_conjugate, src/cyclotomic_ring.rs:662-671."""
    q, d = P.Q62, 32
    rng = np.random.default_rng(3)
    a, b = rand_mod(rng, d, q), rand_mod(rng, d, q)
    lhs = oracle.conjugate(oracle.ring_mul(a, b, q), q)
    rhs = oracle.ring_mul(oracle.conjugate(a, q), oracle.conjugate(b, q), q)
    assert np.array_equal(lhs, rhs)


def test_prf_matches_numpy_copy(oracle):
    for seed, dom in [(0, 0), (7, domain(DOM_NC, 3, 1)), (2 ** 63 + 5, 12345)]:
        idx = np.arange(50, dtype=np.uint64)
        assert [oracle.prf(seed, dom, int(i)) for i in idx] == [int(x) for x in prf_np(seed, dom, idx)]


def test_sumcheck_final_claim_is_square_of_evaluation(oracle):
    """test_sum_check (src/subroutines/fast_norm_check.rs:237-262): after all
    rounds the claim equals <w, tensor(cs)>^2."""
    q = 65537
    rng = np.random.default_rng(4)
    w = rand_mod(rng, 128, q)
    cs = rand_mod(rng, 7, q)
    claim, polys, final_v = oracle.sumcheck(w, q, cs)
    assert claim == int(sum(int(x) * int(x) for x in w) % q)
    # verifier replay
    cl = claim
    for j in range(7):
        f0, f1, f2 = (int(x) for x in polys[j])
        assert (2 * f0 + 2 * f1 + f2) % q == cl
        c = int(cs[j])
        cl = (f0 + 2 * f1 * c + f2 * c * c) % q
    ev = int(sum(int(a) * int(b) for a, b in zip(w, oracle.tensor(cs, q))) % q)
    assert ev == final_v
    assert cl == ev * ev % q


def test_decompose_round_trip(oracle):
    """test_decomp (src/subroutines/decomp.rs:69-92): composing the digits gives the input back."""
    q, d = P.Q0, 16
    rng = np.random.default_rng(5)
    w = small_signed(rng, (2, 64, d), 3000, q)
    for parts in (1, 2, 3):
        out, radix = oracle.decompose(w, q, parts)
        assert out.shape == (2 * parts, 64, d)
        shift = radix.bit_length() - 1
        comp = np.zeros_like(w)
        for r in range(2):
            for c in range(parts):
                digit = out[r * parts + c]
                comp[r] = oracle.eltwise("add", comp[r], oracle.eltwise_fma(digit, (1 << (shift * c)) % q,
                                                                            np.zeros_like(digit), q), q).reshape(64, d)
        assert np.array_equal(comp, w)


def test_fold_homomorphism(oracle):
    """test_fold (src/subroutines/fold.rs:29-56): commit(fold(w, c)) = sum_k c_k commit(w_k)."""
    p = P.make_params(16, P.Q0, 2, 64, 1)
    q, d = p.q, p.d
    rng = np.random.default_rng(6)
    w = rand_mod(rng, (3, 64, d), q)
    c = rand_mod(rng, (3, d), q)
    folded = oracle.fold(w, q, c)
    lhs = oracle.commit_ck(p, 9, folded.reshape(1, 64, d))
    com = oracle.commit_ck(p, 9, w)
    for r in range(p.module_size):
        acc = np.zeros(d, dtype=np.uint64)
        for k in range(3):
            acc = oracle.eltwise("add", acc, oracle.ring_mul(c[k], com[r, k], q), q)
        assert np.array_equal(acc, lhs[r, 0])


def test_commit_matches_power_definition(oracle):
    """parallel_dot_series_matrix on a CK row equals sum_i m^(i+1) * w_i."""
    p = P.make_params(8, P.Q62, 2, 16, 1)
    q, d = p.q, p.d
    rng = np.random.default_rng(7)
    w = rand_mod(rng, (1, 16, d), q)
    m = oracle.sample_crs(p, 3)
    com = oracle.commit_ck(p, 3, w)
    for r in range(2):
        acc = np.zeros(d, dtype=np.uint64)
        pw = m[r].copy()
        for i in range(16):
            acc = oracle.eltwise("add", acc, oracle.ring_mul(pw, w[0, i], q), q)
            pw = oracle.ring_mul(pw, m[r], q)
        assert np.array_equal(acc, com[r, 0])


def test_nc_challenges_helper(oracle):
    q = P.Q0
    got = nc_challenges(5, 2, 1, 4, q)
    dom = domain(DOM_NC, 2, 1)
    assert [int(x) for x in got] == [(oracle.prf(5, dom, j) * q) >> 64 for j in range(4)]


def test_dense_commit_matches_ring_products(oracle):
    """The oracle's dense commitment (src/arithmetic.rs:429-457) is the sum of ring products."""
    from helpers import rand_mod
    from salsaa_b200 import params as P
    q = P.Q0
    rng = np.random.default_rng(5)
    A = rand_mod(rng, (2, 4, 16), q)
    W = rand_mod(rng, (3, 4, 16), q)
    C = oracle.dense_commit(A, W, q)
    for j in range(2):
        for c in range(3):
            acc = [0] * 16
            for i in range(4):
                pr = oracle.ring_mul(A[j, i], W[c, i], q)
                acc = [(x + int(y)) % q for x, y in zip(acc, pr)]
            assert [int(v) for v in C[j, c]] == acc


def _qe(O, a, b, s, q):
    return _quad_mul(O, a, b, s, q)


@pytest.mark.parametrize("q", [P.Q0, 1000003])
def test_sumcheck_fq2_verifier_identities(oracle, q):
    """The F_{q^2} sumcheck restatement satisfies the verifier's round checks
    (verify_norm_check_2, src/subroutines/fast_norm_check.rs:352-399, with
    values in the extension): g(0) + g(1) = 2 f0 + 2 f1 + f2 equals the running
    claim, which becomes f0 + 2 f1 c + f2 c^2, and ends at the square of the
    last folded value; with real challenges it equals the F_q sumcheck."""
    O = oracle
    s = O.qnr(q)
    assert O.pow_mod(s, (q - 1) // 2, q) == q - 1
    rng = np.random.default_rng(3)
    w = small_signed(rng, 1 << 9, 1, q)
    nr = 9
    cs = rand_mod(rng, (nr, 2), q)
    claim, polys, final = O.sumcheck_fq2(w, q, s, cs)
    cur = [claim, 0]
    for j in range(nr):
        f0, f1, f2 = ([int(x) for x in polys[j, t]] for t in range(3))
        tot = [(2 * f0[k] + 2 * f1[k] + f2[k]) % q for k in range(2)]
        assert tot == cur, j
        c = [int(cs[j, 0]), int(cs[j, 1])]
        c2 = _qe(O, c, c, s, q)
        t1 = _qe(O, f1, c, s, q)
        t2 = _qe(O, f2, c2, s, q)
        cur = [(f0[k] + 2 * t1[k] + t2[k]) % q for k in range(2)]
    assert cur == _qe(O, list(final), list(final), s, q)
    # real challenges: the F_q sumcheck
    cr = np.stack([cs[:, 0], np.zeros(nr, dtype=np.uint64)], axis=1)
    claim2, polys2, _ = O.sumcheck_fq2(w, q, s, cr)
    c1, p1, _ = O.sumcheck(w, q, cs[:, 0])
    assert claim2 == c1
    assert np.array_equal(polys2[:, :, 0], p1) and not polys2[:, :, 1].any()
