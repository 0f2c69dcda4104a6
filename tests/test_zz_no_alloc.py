"""salsaa_project_noalloc: the projection for callers that must not allocate
device memory on the call path (for example a serving loop that has already
divided HBM among in-flight proofs).  Its output must equal the allocating
entry point's, bit for bit, on consecutive calls that reuse the library's
fixed scratch array.  Collected last so a run that stops at the first failure
has already run every other test."""
import ctypes

import numpy as np
import pytest

from helpers import small_signed
from salsaa_b200 import params as P

pytestmark = pytest.mark.gpu


def _call(fn, w, rows, width, d, q, seed, rnd, out, stream):
    return fn(ctypes.c_void_p(w.data_ptr()), rows, width, d, q, seed, rnd, ctypes.c_void_p(out.data_ptr()), stream)


def test_noalloc_matches_allocating_entry(gpu_lib, cuda):
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


def test_noalloc_rejects_oversize(gpu_lib, cuda):
    from salsaa_b200 import api
    torch = cuda
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    w = api.to_dev(np.zeros((16, 4096, 16), dtype=np.uint64))
    out = api.dev_empty((4096, 16))
    rc = _call(gpu_lib.salsaa_project_noalloc, w, 16, 4096, 16, P.Q0, 1, 0, out, stream)
    assert rc == -3
    assert b"2048-column scratch" in gpu_lib.salsaa_last_error()
