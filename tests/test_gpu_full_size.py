"""Full-size proofs of the reference parameter sets (src/protocol.rs:28-123),
byte for byte: the SHA-256 of every GPU proof must equal the digest of the
oracle's proof of the same (preset, crs_seed, seed), committed in
tests/golden/proof_digests.json by tests/golden/make_proof_digests.py (the
oracle needs minutes per proof, so it does not run here).

Each preset is proved three ways: the blocking path (one proof at a time),
the batched path (the digest's statement among other proofs in flight on
separate slots) and the serving loop (admitted among other requests)."""
import hashlib
import json
import os

import numpy as np
import pytest

from salsaa_b200 import params as P

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "proof_digests.json")) as f:
    DIGESTS = json.load(f)
NAMES = [n for n in ("F0", "A2", "A1", "A0", "F1", "F2") if n in DIGESTS]
# proofs in flight in the batched test (workspace: 2.3 GiB F0 ... 36 GiB F2)
BATCH = {"A0": 8, "A1": 8, "A2": 8, "F0": 8, "F1": 4, "F2": 2}


def sha(buf):
    return hashlib.sha256(np.ascontiguousarray(buf).view(np.uint8).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def api(gpu_lib, cuda):
    from salsaa_b200 import api as A
    return A


def _params(name):
    g = DIGESTS[name]
    p = P.preset(name)
    assert p.as_dict() == g["params"], "preset changed since the digests were made"
    return p, g


@pytest.mark.parametrize("name", NAMES)
def test_full_size_proof_digest(api, name):
    p, g = _params(name)
    ctx = api.Context(p, crs_seed=g["crs_seed"])
    proof = ctx.prove(g["seed"])
    assert proof.size == g["bytes"]
    assert sha(proof) == g["sha256"]
    ctx.close()


@pytest.mark.parametrize("name", NAMES)
def test_full_size_batched_digest(api, cuda, name):
    """The digest's statement proved in slot 1 of a batch of proofs in flight."""
    torch = cuda
    p, g = _params(name)
    ctx = api.Context(p, crs_seed=g["crs_seed"])
    n = BATCH[name]
    slots = [api.Prover(ctx) for _ in range(n)]
    seeds = [g["seed"] + 1000 + i for i in range(n)]
    seeds[1] = g["seed"]
    bufs = [torch.empty(ctx.proof_bytes // 8, dtype=torch.int64, device="cuda") for _ in range(n)]
    torch.cuda.synchronize()
    for s, pr, b in zip(seeds, slots, bufs):
        pr.enqueue(s, b)
    for pr in slots:
        pr.sync()
    assert sha(api.to_host(bufs[1])) == g["sha256"]
    for pr in slots:
        pr.close()
    ctx.close()


def test_full_size_served_digests(api, cuda):
    """Every preset's digest statement submitted to one serving loop among
    other requests, admitted as slots free up."""
    torch = cuda
    names = [n for n in NAMES if n != "F2"]  # F2's 36 GiB slot is proved alone above
    srv = api.Server(hbm_budget_bytes=120 << 30)
    srv.limit(4)
    sets = {}
    for nm in names:
        p, g = _params(nm)
        sets[nm] = srv.register(p, crs_seed=g["crs_seed"], slots=2)
    jobs = []
    for k, nm in enumerate(names):
        p, g = _params(nm)
        for seed in (g["seed"] + 77, g["seed"]):
            buf = torch.empty(api.proof_size(p) // 8, dtype=torch.int64, device="cuda")
            jobs.append((nm, seed, buf, srv.submit(sets[nm], seed, buf)))
        srv.progress()
    pending = {t for *_, t in jobs}
    while pending:
        srv.progress()
        for t in list(pending):
            if srv.poll(t) is not None:
                pending.discard(t)
    torch.cuda.synchronize()
    for nm, seed, buf, _ in jobs:
        if seed == DIGESTS[nm]["seed"]:
            assert sha(api.to_host(buf)) == DIGESTS[nm]["sha256"], nm
    srv.close()
