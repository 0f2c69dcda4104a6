"""The library's verifier (salsaa_verify: host replay of the reference
verifier's inline checks, final statement check on the GPU) against the
oracle's verifier: same verdict on valid proofs, on proofs with one word
changed in each section, and under a wrong seed."""
import numpy as np
import pytest

from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu

CASES = {
    "snark2_d16": P.small_snark(d=16, log_len=13, rounds=2),
    "snark3_d32_q1": P.small_snark(d=32, q=P.Q1, module_size=2, log_len=14, rounds=3),
    "snark2_d128": P.make_params(128, P.Q0, 4, 1 << 13, 2, False),
    "fold_d16": P.small_folding(d=16, log_len=11),
    "fold_d128": P.make_params(128, P.Q0, 5, 1 << 12, 1, True),
}


@pytest.fixture(scope="module")
def api(gpu_lib, cuda):
    from salsaa_b200 import api as A
    return A


@pytest.mark.parametrize("name", sorted(CASES))
def test_verify_accepts_and_rejects(api, oracle, name):
    p = CASES[name]
    ctx = api.Context(p, crs_seed=5)
    proof = ctx.prove(9)
    assert ctx.verify(9, proof) == 0
    assert oracle.verify(p, 5, 9, proof) == 0
    words = proof.size // 8
    rng = np.random.default_rng(words)
    # one changed word at the header, early, in the middle, and near the end
    for at in [3, 8 + 5, int(rng.integers(9, words)), words // 2, words - 1 - int(rng.integers(0, 64))]:
        bad = proof.copy().view(np.uint64)
        bad[at] = (int(bad[at]) + 1) % p.q if at >= 8 else int(bad[at]) ^ 1
        bad = bad.view(np.uint8)
        want = oracle.verify(p, 5, 9, bad)
        got = ctx.verify(9, bad)
        assert want != 0 and got == want, (at, got, want)
    assert ctx.verify(10, proof) == oracle.verify(p, 5, 10, proof) != 0
    assert ctx.verify(9, proof[:-8]) != 0


@pytest.mark.slow
def test_verify_full_size_a0(api, oracle):
    p = P.preset("A0")
    ctx = api.Context(p, crs_seed=1)
    proof = ctx.prove(2)
    assert ctx.verify(2, proof) == 0
    bad = proof.copy()
    bad[-8 * 1000] ^= 2
    assert ctx.verify(2, bad) == oracle.verify(p, 1, 2, bad) != 0
