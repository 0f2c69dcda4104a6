"""Whole proofs: the device-resident prover's bytes equal the oracle's, and
the oracle's verifier accepts full-size proofs of the reference parameter
sets."""
import numpy as np
import pytest

from helpers import rand_mod
from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu

SMALL = {
    "snark2_d16": P.small_snark(d=16, log_len=13, rounds=2),
    "snark3_d32_q1": P.small_snark(d=32, q=P.Q1, module_size=2, log_len=14, rounds=3),
    "snark2_d128": P.make_params(128, P.Q0, 4, 1 << 13, 2, False),
    "snark2_d512_q2": P.make_params(512, P.Q2, 3, 1 << 13, 2, False),
    "fold_d16": P.small_folding(d=16, log_len=11),
    "fold_d128": P.make_params(128, P.Q0, 5, 1 << 12, 1, True),
    # a round without decomposition after a decomposed one: the joined witness
    # is then read in slot form by the next round
    "snark3_d128_parts121": P.make_params(128, P.Q0, 3, 1 << 14, 3, False, decomp_parts=[1, 2, 1]),
    "snark3_d128_parts112": P.make_params(128, P.Q0, 3, 1 << 14, 3, False, decomp_parts=[1, 1, 2]),
    # two initial witness rows; more key rows than the tcgen05 key tiles hold
    # (mma.sync commitment)
    "snark2_d128_rep2": P.make_params(128, P.Q0, 3, 1 << 13, 2, False, init_wit_rep=2),
    "snark2_d128_ms20": P.make_params(128, P.Q0, 20, 1 << 13, 2, False),
}


@pytest.fixture(scope="module")
def api(gpu_lib, cuda):
    from salsaa_b200 import api as A
    return A


@pytest.mark.parametrize("name", sorted(SMALL))
def test_proof_bytes_equal_oracle(api, oracle, name):
    p = SMALL[name]
    rc, want, _ = oracle.prove(p, 7, 11)
    assert rc == 0
    ctx = api.Context(p, crs_seed=7)
    got = ctx.prove(11)
    if not np.array_equal(got, want):
        w = np.flatnonzero(got.view(np.uint64) != want.view(np.uint64))
        pytest.fail("first differing word %d of %d" % (w[0], want.size // 8))
    assert oracle.verify(p, 7, 11, got) == 0


def test_explicit_witness(api, oracle):
    p = SMALL["snark2_d16"]
    rng = np.random.default_rng(0)
    w = rng.integers(-3, 4, size=(1, p.wit_len, p.d))
    w = np.where(w < 0, p.q + w, w).astype(np.uint64)
    rc, want, _ = oracle.prove(p, 1, 2, witness=w)
    assert rc == 0
    got = api.Context(p, crs_seed=1).prove(2, witness=w)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name,lo,hi", [("snark2_d16", -1, 2), ("snark2_d128_rep2", -128, 128),
                                        ("fold_d16", -128, 128)])
def test_int8_witness_upload(api, oracle, name, lo, hi):
    """salsaa_prover_enqueue_host_i8: the witness as centred signed bytes gives
    the oracle's proof of the same residues."""
    p = SMALL[name]
    rng = np.random.default_rng(5)
    w8 = rng.integers(lo, hi, size=(p.init_wit_rep, p.wit_len, p.d)).astype(np.int8)
    w = np.where(w8 < 0, p.q + w8.astype(np.int64), w8).astype(np.uint64)
    rc, want, _ = oracle.prove(p, 3, 4, witness=w)
    assert rc == 0
    ctx = api.Context(p, crs_seed=3)
    pr = api.Prover(ctx)
    got = np.zeros(ctx.proof_bytes, dtype=np.uint8)
    pr.enqueue_host_i8(4, got, np.ascontiguousarray(w8.reshape(-1)))
    pr.sync()
    assert np.array_equal(got, want)
    pr.close()


@pytest.mark.parametrize("bound", [0, 1 << 22, 1 << 30])
def test_large_witness_d128(api, oracle, bound):
    """Witness values beyond the tensor-core paths' byte limbs (uniform mod q,
    around 2^22, around 2^30) must still give the oracle's proof bytes: the
    projection and scalar-row passes fall back to their exact kernels."""
    p = P.make_params(128, P.Q0, 4, 1 << 13, 2, False)
    rng = np.random.default_rng(bound + 1)
    if bound:
        w = rng.integers(-bound, bound + 1, size=(1, p.wit_len, p.d))
        w = np.where(w < 0, p.q + w, w).astype(np.uint64)
    else:
        w = rand_mod(rng, (1, p.wit_len, p.d), p.q)
    rc, want, _ = oracle.prove(p, 3, 4, witness=w)
    assert rc == 0
    got = api.Context(p, crs_seed=3).prove(4, witness=w)
    assert np.array_equal(got, want)


def test_async_slots_match_blocking(api, oracle):
    """Several proofs in flight on separate slots give the same bytes as one at a time."""
    import torch
    p = SMALL["snark3_d32_q1"]
    ctx = api.Context(p, crs_seed=3)
    seeds = [10, 11, 12, 13]
    slots = [api.Prover(ctx) for _ in seeds]
    bufs = [torch.empty(ctx.proof_bytes // 8, dtype=torch.int64, device="cuda") for _ in seeds]
    torch.cuda.synchronize()
    for s, pr, b in zip(seeds, slots, bufs):
        pr.enqueue(s, b)
    for pr in slots:
        pr.sync()
    for s, b in zip(seeds, bufs):
        assert np.array_equal(api.to_host(b).view(np.uint8), ctx.prove(s))
        assert np.array_equal(api.to_host(b).view(np.uint8), oracle.prove(p, 3, s)[1])


@pytest.mark.slow
@pytest.mark.parametrize("name", ["F0", "A2", "A0"])
def test_full_size_proof_verifies(api, oracle, name):
    """Reference parameter sets at full size: the oracle's verifier (the
    reference's own checks) accepts the GPU proof, and a flipped word is caught."""
    p = P.preset(name)
    ctx = api.Context(p, crs_seed=1)
    proof = ctx.prove(2)
    assert oracle.verify(p, 1, 2, proof) == 0
    bad = proof.copy()
    bad[8 * 100] ^= 4
    assert oracle.verify(p, 1, 2, bad) != 0


@pytest.mark.parametrize("name", ["snark2_d128", "snark3_d128_parts121", "fold_d128"])
def test_overlap_slot_matches_oracle(api, oracle, name):
    """A slot running the projection beside the norm check makes the same bytes."""
    import torch
    p = SMALL[name]
    ctx = api.Context(p, crs_seed=7)
    pr = api.Prover(ctx)
    pr.set_overlap(True)
    buf = torch.empty(ctx.proof_bytes // 8, dtype=torch.int64, device="cuda")
    for seed in (11, 12):
        pr.enqueue(seed, buf)
        pr.sync()
        assert np.array_equal(api.to_host(buf).view(np.uint8), oracle.prove(p, 7, seed)[1])
    pr.close()


@pytest.mark.parametrize("overlap", [False, True])
def test_graph_replay_matches_oracle(api, oracle, cuda, overlap):
    """A slot replaying its captured CUDA graph (the seed changed per proof,
    queued back to back, the graph captured again for a new buffer pair and
    for the int8 upload path) gives the oracle's proof bytes every time."""
    torch = cuda
    p = P.make_params(128, P.Q0, 4, 1 << 13, 2, False)
    ctx = api.Context(p, crs_seed=7)
    pr = api.Prover(ctx)
    pr.set_overlap(overlap)
    pr.set_graph(True)
    bufs = [torch.empty(ctx.proof_bytes // 8, dtype=torch.int64, device="cuda") for _ in range(4)]
    seeds = [21, 22, 23, 24]
    plan = [(seeds[0], bufs[0]), (seeds[1], bufs[0]), (seeds[2], bufs[0]), (seeds[3], bufs[1])]
    outs = []
    for sd, b in plan:
        pr.enqueue(sd, b)
        pr.sync()
        outs.append(api.to_host(b).view(np.uint8).copy())
    for (sd, _), got in zip(plan, outs):
        rc, want, _ = oracle.prove(p, 7, sd)
        assert rc == 0 and np.array_equal(got, want), sd
    # back to back without waiting: a replay queued behind a proof still running keeps its own seed
    pr.enqueue(31, bufs[2])  # captures for bufs[2]
    pr.enqueue(32, bufs[3])  # captures for bufs[3]
    pr.enqueue(33, bufs[3])  # replays with a new seed while the previous proof may still run
    pr.sync()
    assert np.array_equal(api.to_host(bufs[2]).view(np.uint8), oracle.prove(p, 7, 31)[1])
    assert np.array_equal(api.to_host(bufs[3]).view(np.uint8), oracle.prove(p, 7, 33)[1])
    # the int8 upload path through the graph
    rng = np.random.default_rng(8)
    w8 = rng.integers(-1, 2, size=(p.init_wit_rep, p.wit_len, p.d)).astype(np.int8)
    w = np.where(w8 < 0, p.q + w8.astype(np.int64), w8).astype(np.uint64)
    for sd in (41, 42):
        got = np.zeros(ctx.proof_bytes, dtype=np.uint8)
        pr.enqueue_host_i8(sd, got, np.ascontiguousarray(w8.reshape(-1)))
        pr.sync()
        rc, want, _ = oracle.prove(p, 7, sd, witness=w)
        assert rc == 0 and np.array_equal(got, want), sd
    pr.close()
