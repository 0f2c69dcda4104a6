"""salsaa_project_noalloc: the projection for callers that must not allocate
device memory on the call path (for example a serving loop that has already
divided HBM among in-flight proofs).  Its output must equal the allocating
entry point's, bit for bit, on consecutive calls that reuse the library's
fixed scratch array, and the oracle's projection.  Collected last so a run that stops at the first failure
has already run every other test."""
import ctypes

import numpy as np
import pytest

from helpers import small_signed
from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu


def _call(fn, w, rows, width, d, q, seed, rnd, out, stream):
    return fn(ctypes.c_void_p(w.data_ptr()), rows, width, d, q, seed, rnd, ctypes.c_void_p(out.data_ptr()), stream)


def test_noalloc_matches_allocating_entry(gpu_lib, cuda, oracle):
    from helpers import proj_challenge
    from salsaa_b200 import api
    torch = cuda
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = [(2, 2048, 128, 60, 3, 1), (8, 4096, 128, 1, 4, 2), (4, 2048, 256, 200, 5, 3)]
    for rows, width, d, bound, seed, rnd in cases:  # consecutive calls share the scratch
        q = P.Q0
        rng = np.random.default_rng(seed)
        w = api.to_dev(small_signed(rng, (rows, width, d), bound, q))
        ref = api.dev_empty((width, d))
        got = api.dev_empty((width, d))
        got.fill_(-1)
        assert _call(gpu_lib.salsaa_project, w, rows, width, d, q, seed, rnd, ref, stream) == 0
        assert _call(gpu_lib.salsaa_project_noalloc, w, rows, width, d, q, seed, rnd, got, stream) == 0, \
            gpu_lib.salsaa_last_error()
        torch.cuda.synchronize()
        assert torch.equal(ref, got)
        iz, sg = proj_challenge(seed, rnd, rows * 256)  # and the oracle's projection, word for word
        want = oracle.project(small_signed(np.random.default_rng(seed), (rows, width, d), bound, q), q, iz, sg)
        assert np.array_equal(api.to_host(got), want)


@pytest.mark.parametrize("rows,width,d,msg", [
    (16, 4096, 16, b"2048-column scratch"),          # more rows than the scratch covers
    (1 << 56, 4096, 16, b"2048-column scratch"),     # rows * 256 would wrap to 0
    ((1 << 56) + 1, 4096, 16, b"2048-column scratch"),  # rows * 256 would wrap to 256
    (8, 1024, 16, b"exceeds the witness width"),     # chunk wider than the witness
    (3, 2048, 16, b"exceeds the witness width"),     # width not a multiple of the chunk
])
def test_noalloc_rejects_bad_shapes(gpu_lib, cuda, rows, width, d, msg):
    """Shapes outside the fixed scratch return -3 before any launch: the
    output buffer keeps its contents."""
    from salsaa_b200 import api
    torch = cuda
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    w = api.to_dev(np.zeros((min(rows, 16), width, d), dtype=np.uint64))
    out = api.dev_empty((width, d))
    out.fill_(7)
    torch.cuda.synchronize()
    rc = _call(gpu_lib.salsaa_project_noalloc, w, rows, width, d, P.Q0, 1, 0, out, stream)
    assert rc == -3
    assert msg in gpu_lib.salsaa_last_error()
    torch.cuda.synchronize()
    assert bool((out == 7).all())
