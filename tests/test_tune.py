"""NTT kernel schedules (salsaa_tune_load / salsaa_ntt_tune_set / get /
salsaa_tune_reset).  The table API is host-only, so it is checked on the CPU;
the GPU tests check that every schedule gives the default schedule's outputs
bit for bit, on transform sizes with partial last tiles and on whole proofs."""
import ctypes

import numpy as np
import pytest

from helpers import rand_mod
from salsaa_b200 import params as P

CANDIDATES = [(0, 0), (1, 0), (2, 0), (2, 1), (3, 0), (4, 0), (5, 0), (6, 0), (7, 1)]  # 1, 5-7: FP64 when q < 2^50


def _get(L, key):
    v, c = ctypes.c_int(), ctypes.c_int()
    assert L.salsaa_ntt_tune_get(*key, ctypes.byref(v), ctypes.byref(c)) == 0
    return v.value, c.value


def _set_all(L, variant, cps):
    for lg in range(1, 14):
        for inc in (0, 1):
            for inv in (0, 1):
                for wide in (0, 1):
                    for large in (0, 1):
                        assert L.salsaa_ntt_tune_set(lg, inc, inv, wide, large, variant, cps) == 0


def test_tune_table_roundtrip(gpu_lib, tmp_path):
    L = gpu_lib
    assert L.salsaa_tune_reset() == 0
    assert _get(L, (6, 1, 0, 0, 1)) == (0, 0)
    table = tmp_path / "t.txt"
    table.write_text("# comment\n"
                     "ntt 6 1 0 0 1 3 0   # incomplete d=128 forward, large\n"
                     "ntt 10 0 1 1 0 2 1\n"
                     "ntt 6 1 1 0 1 9 0   # variant 9 does not exist: ignored\n"
                     "ntt 7 1 0 0 1 1 0   # FP64 butterflies\n"
                     "fold 1\n"
                     "garbage line\n")
    assert L.salsaa_tune_load(str(table).encode()) == 4
    assert L.salsaa_fold_tune_get() == 1
    assert _get(L, (6, 1, 0, 0, 1)) == (3, 0)
    assert _get(L, (10, 0, 1, 1, 0)) == (2, 1)
    assert _get(L, (6, 1, 1, 0, 1)) == (0, 0)
    assert _get(L, (7, 1, 0, 0, 1)) == (1, 0)
    assert L.salsaa_tune_load(str(tmp_path / "missing.txt").encode()) < 0
    assert L.salsaa_ntt_tune_set(6, 1, 0, 0, 1, 8, 0) < 0  # no variant 8
    assert L.salsaa_ntt_tune_set(6, 1, 0, 0, 1, -1, 0) < 0
    assert L.salsaa_ntt_tune_set(14, 1, 0, 0, 1, 2, 0) < 0  # log n out of range
    assert L.salsaa_fold_tune_set(2) < 0
    assert L.salsaa_tune_reset() == 0
    assert _get(L, (6, 1, 0, 0, 1)) == (0, 0)
    assert L.salsaa_fold_tune_get() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n_arg,incomplete,q,count", [
    (128, True, P.Q0, 3 * 32 + 5),       # incomplete d = 128, partial last tile
    (256, True, P.Q1, 1000),
    (512, True, P.Q2, 17),
    (64, False, P.Q62, 64 * 300 + 1),    # more tiles than resident CTAs
    (1024, False, P.Q62, 77),
    (16, False, P.Q0, 4096),             # one exchange-free phase
    (4096, False, P.Q0, 3),              # one unit per tile
])
def test_schedules_equal_default(gpu_lib, cuda, oracle, n_arg, incomplete, q, count):
    from salsaa_b200 import api
    torch = cuda
    L = gpu_lib
    rng = np.random.default_rng(count)
    x = rand_mod(rng, (count, n_arg), q)
    xd = api.to_dev(x)
    outs = {}
    try:
        for var, cps in CANDIDATES:
            _set_all(L, var, cps)
            fwd = api.ntt(xd, n_arg, q, incomplete=incomplete, out=api.dev_empty(xd.shape))
            back = api.ntt(fwd, n_arg, q, inverse=True, incomplete=incomplete, out=api.dev_empty(xd.shape))
            torch.cuda.synchronize()
            outs[(var, cps)] = (api.to_host(fwd), api.to_host(back))
    finally:
        L.salsaa_tune_reset()
    ref_fwd, ref_back = outs[(0, 0)]
    assert np.array_equal(ref_back, x)
    want = oracle.ring_to_slot(x[:4], q) if incomplete else oracle.ntt_forward(x[:4], q)
    assert np.array_equal(ref_fwd[:4], want)
    for k, (f, b) in outs.items():
        assert np.array_equal(f, ref_fwd), k
        assert np.array_equal(b, ref_back), k


@pytest.mark.gpu
@pytest.mark.parametrize("var,cps", [(1, 0), (2, 0), (3, 0), (4, 0), (2, 1), (5, 0), (7, 0)])
def test_proofs_under_each_schedule(gpu_lib, oracle, var, cps):
    """Whole proofs with every transform on a pipelined schedule equal the oracle's."""
    from salsaa_b200 import api
    L = gpu_lib
    p = P.make_params(128, P.Q0, 4, 1 << 13, 2, False)
    rc, want, _ = oracle.prove(p, 7, 11)
    assert rc == 0
    try:
        _set_all(L, var, cps)
        assert L.salsaa_fold_tune_set(1 if var in (1, 5, 6, 7) else 0) == 0
        got = api.Context(p, crs_seed=7).prove(11)
    finally:
        L.salsaa_tune_reset()
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("rows,width,d,q", [(2, 1 << 12, 128, P.Q0), (5, 300, 256, P.Q1), (16, 64, 512, P.Q2),
                                            (3, 100, 64, P.Q62)])
def test_fold_variants(gpu_lib, oracle, rows, width, d, q):
    """The fold with integer and with FP64 products (q < 2^50; wider moduli
    keep the integer products) equals the oracle's fold."""
    from helpers import fold_challenge
    from salsaa_b200 import api
    L = gpu_lib
    rng = np.random.default_rng(rows * width)
    w = rand_mod(rng, (rows, width, d), q)
    c = fold_challenge(3, 1, rows, d, q)
    want = oracle.fold(w, q, c)
    try:
        for var in (0, 1):
            assert L.salsaa_fold_tune_set(var) == 0
            assert L.salsaa_fold_tune_get() == var
            got = api.to_host(api.fold(api.to_dev(w), q, api.to_dev(c)))
            assert np.array_equal(got, want), var
    finally:
        L.salsaa_tune_reset()
