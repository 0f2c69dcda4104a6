"""Continuous-batching service: requests of several parameter sets admitted
onto slots as they free up, running concurrently; every proof must equal the
proof of the same statement proved alone (and verify on the CPU)."""
import numpy as np
import pytest

from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu

MIX = {
    "snark2_d16": P.small_snark(d=16, log_len=13, rounds=2),
    "snark3_d32_q1": P.small_snark(d=32, q=P.Q1, module_size=2, log_len=14, rounds=3),
    "fold_d16": P.small_folding(d=16, log_len=11),
    "snark2_d128": P.make_params(128, P.Q0, 4, 1 << 13, 2, False),
}


@pytest.fixture(scope="module")
def api(gpu_lib, cuda):
    from salsaa_b200 import api as A
    return A


@pytest.mark.parametrize("max_inflight", [0, 1, 2])
def test_mixed_stream_equals_alone(api, oracle, cuda, max_inflight):
    torch = cuda
    srv = api.Server(hbm_budget_bytes=16 << 30)
    srv.limit(max_inflight)
    names = sorted(MIX)
    sets = {nm: srv.register(MIX[nm], crs_seed=7, slots=2) for nm in names}
    jobs = []
    rng = np.random.default_rng(3)
    for i in range(20):
        nm = names[rng.integers(len(names))]
        buf = torch.empty(api.proof_size(MIX[nm]) // 8, dtype=torch.int64, device="cuda")
        seed = 1000 + i
        jobs.append((nm, seed, buf, None))
    # submit in waves while earlier proofs run (continuous admission)
    tickets = []
    for k, (nm, seed, buf, _) in enumerate(jobs):
        tickets.append(srv.submit(sets[nm], seed, buf))
        if k % 3 == 2:
            srv.progress()
    lat = {}
    while len(lat) < len(tickets):
        srv.progress()
        for t in tickets:
            if t not in lat:
                r = srv.poll(t)
                if r is not None:
                    lat[t] = r
    torch.cuda.synchronize()
    alone = {nm: api.Context(MIX[nm], crs_seed=7) for nm in names}
    for (nm, seed, buf, _), t in zip(jobs, tickets):
        got = api.to_host(buf).view(np.uint8)
        assert np.array_equal(got, alone[nm].prove(seed)), (nm, seed)
        assert lat[t][0] >= lat[t][1] >= 0
    # one of each verifies with the reference checks and equals the oracle's proof byte for byte
    for nm in names:
        nm_jobs = [(s, b) for (n2, s, b, _) in jobs if n2 == nm]
        if nm_jobs:
            s, b = nm_jobs[0]
            got = api.to_host(b).view(np.uint8)
            assert oracle.verify(MIX[nm], 7, s, got) == 0
            rc, want, _ = oracle.prove(MIX[nm], 7, s)
            assert rc == 0 and np.array_equal(got, want), nm
    srv.close()


def test_budget_enforced(api):
    from salsaa_b200.api import SalsaaError
    srv = api.Server(hbm_budget_bytes=1 << 20)
    with pytest.raises(SalsaaError):
        srv.register(MIX["snark2_d16"], slots=1)
    srv.close()


def test_cancel_queued_request(api, cuda):
    from salsaa_b200.api import SalsaaError
    torch = cuda
    p = MIX["snark2_d16"]
    srv = api.Server(hbm_budget_bytes=16 << 30)
    srv.limit(1)
    sid = srv.register(p, crs_seed=7, slots=1)
    bufs = [torch.zeros(api.proof_size(p) // 8, dtype=torch.int64, device="cuda") for _ in range(4)]
    tickets = [srv.submit(sid, 2000 + i, b) for i, b in enumerate(bufs)]
    assert srv.progress() == 4  # one admitted, three queued
    assert srv.cancel(tickets[0]) is False  # admitted: runs to completion
    assert srv.cancel(tickets[2]) is True  # queued: withdrawn and forgotten
    with pytest.raises(SalsaaError):
        srv.poll(tickets[2])
    with pytest.raises(SalsaaError):
        srv.cancel(tickets[2])
    left = [t for t in tickets if t != tickets[2]]
    done = set()
    while len(done) < len(left):
        srv.progress()
        for t in left:
            if t not in done and srv.poll(t) is not None:
                done.add(t)
    torch.cuda.synchronize()
    alone = api.Context(p, crs_seed=7)
    for i, b in enumerate(bufs):
        got = api.to_host(b).view(np.uint8)
        if i == 2:
            assert not got.any()  # never written
        else:
            assert np.array_equal(got, alone.prove(2000 + i)), i
    srv.close()
