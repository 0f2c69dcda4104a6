"""Whole-protocol properties of the oracle: the reference's inline verifier
checks accept honest proofs, reject tampered ones, and proofs are a
deterministic function of (params, crs_seed, seed).  CPU only."""
import numpy as np
import pytest

from salsaa_b200 import params as P

CASES = {
    "snark2": P.small_snark(d=16, log_len=13, rounds=2),
    "snark3_d32": P.small_snark(d=32, q=P.Q1, module_size=2, log_len=14, rounds=3),
    "fold": P.small_folding(d=16, log_len=11),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_prove_verify(oracle, name):
    p = CASES[name]
    rc, proof, _ = oracle.prove(p, 7, 11)
    assert rc == 0
    assert proof.size == oracle.proof_size(p)
    assert oracle.verify(p, 7, 11, proof) == 0
    # another proof of the same statement shape with another seed differs and verifies
    rc2, proof2, _ = oracle.prove(p, 7, 12)
    assert rc2 == 0 and not np.array_equal(proof, proof2)
    assert oracle.verify(p, 7, 12, proof2) == 0
    # verifier bound to the seed: the other transcript is rejected
    assert oracle.verify(p, 7, 12, proof) != 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_deterministic(oracle, name):
    p = CASES[name]
    a = oracle.prove(p, 1, 2)[1]
    b = oracle.prove(p, 1, 2)[1]
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", sorted(CASES))
def test_tamper_rejected(oracle, name):
    p = CASES[name]
    _, proof, _ = oracle.prove(p, 3, 4)
    words = proof.size // 8
    rng = np.random.default_rng(0)
    for w in rng.choice(np.arange(8, words), size=12, replace=False):
        bad = proof.copy()
        bad[8 * w] ^= 1
        assert oracle.verify(p, 3, 4, bad) != 0, "flip at word %d accepted" % w


def test_explicit_witness_equals_sampled(oracle):
    p = CASES["snark2"]
    w = oracle.sample_witness(p, 11)
    assert set(np.unique(w).tolist()) <= {0, 1, p.q - 1}
    a = oracle.prove(p, 7, 11)[1]
    b = oracle.prove(p, 7, 11, witness=w)[1]
    assert np.array_equal(a, b)


def test_witness_distribution(oracle):
    """random_bounded(2): P(0) = 1/2, P(+1) = P(-1) = 1/4 (src/cyclotomic_ring.rs:293-317)."""
    p = P.make_params(128, P.Q0, 1, 4096, 1)
    w = oracle.sample_witness(p, 5).ravel()
    n = w.size
    assert abs((w == 0).sum() / n - 0.5) < 0.01
    assert abs((w == 1).sum() / n - 0.25) < 0.01
    assert abs((w == p.q - 1).sum() / n - 0.25) < 0.01


def test_bad_params_rejected(oracle):
    p = P.small_snark(log_len=9, rounds=2)  # projection chunk wider than the witness
    rc, _, _ = oracle.prove(p, 1, 1)
    assert rc != 0
