"""The C-ABI library loads and exports every symbol include/salsaa_gpu.h
declares; host-only entry points agree with the oracle.  No GPU needed."""
import ctypes
import os
import re

import pytest

from salsaa_b200 import params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "salsaa_gpu.h")

# extern "C" block of the reference's Rust crate (src/hexl/bindings.rs:1-74)
REFERENCE_FFI = {
    "multiply_mod", "power_mod", "add_mod", "sub_mod", "eltwise_mult_mod", "get_roots", "inv_mod",
    "get_inv_roots", "sum_sq", "sum_sq_fast", "sum", "sum_fast", "eltwise_fma_mod", "eltwise_add_mod",
    "eltwise_sub_mod", "multiply_poly", "eltwise_reduce_mod", "eltwise_reduce_mod_naive",
    "polynomial_multiply_cyclotomic_mod", "ntt_forward_in_place", "ntt_inverse_in_place",
}


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[a-z_ ]*?(?:uint64_t|void|int|const char|const uint64_t)\s*\*?\s*([a-z_0-9]+)\s*\(",
                       text, flags=re.M)
    return set(names)


def test_header_declares_reference_ffi():
    assert REFERENCE_FFI <= header_functions()


def test_library_exports_header(gpu_lib):
    missing = [n for n in sorted(header_functions()) if not hasattr(gpu_lib, n)]
    assert not missing


def test_abi_table_covers_header():
    from salsaa_b200 import _abi
    assert header_functions() == set(_abi.ALL_SYMBOLS)


@pytest.mark.parametrize("name", sorted(P.PRESETS))
def test_presets_and_proof_size(gpu_lib, oracle, name):
    p = P.SalsaaParams()
    assert gpu_lib.salsaa_params_preset(name.encode(), ctypes.byref(p)) == 0
    ref = P.preset(name)
    assert p.as_dict() == ref.as_dict()
    assert gpu_lib.salsaa_proof_size(ctypes.byref(p)) == oracle.proof_size(ref)
    assert gpu_lib.salsaa_workspace_bytes(ctypes.byref(p)) > 0


def test_unknown_preset(gpu_lib):
    p = P.SalsaaParams()
    assert gpu_lib.salsaa_params_preset(b"Z9", ctypes.byref(p)) != 0
    assert b"unknown" in gpu_lib.salsaa_last_error()


def test_invalid_params_have_no_proof_size(gpu_lib):
    p = P.small_snark(log_len=9, rounds=2)
    assert gpu_lib.salsaa_proof_size(ctypes.byref(p)) == 0


def test_wide_decomposition_rejected(gpu_lib, oracle):
    """More than two decomposition parts give projection chunks wider than
    2048 (16 rows x 256 after the split): the library refuses the shape up
    front (no proof size, no workspace), although the oracle proves it."""
    p = P.make_params(128, P.Q0, 3, 1 << 15, 2, False, decomp_parts=[1, 4])
    assert gpu_lib.salsaa_proof_size(ctypes.byref(p)) == 0
    assert gpu_lib.salsaa_workspace_bytes(ctypes.byref(p)) == 0
    ok = P.make_params(128, P.Q0, 3, 1 << 15, 2, False)
    assert gpu_lib.salsaa_proof_size(ctypes.byref(ok)) == oracle.proof_size(ok)


def test_host_scalar_symbols(gpu_lib, oracle):
    q = P.Q62
    for a, b in [(12345, 67890), (q - 1, q - 2), (2 ** 61, 3)]:
        assert gpu_lib.multiply_mod(a, b, q) == oracle.mul_mod(a, b, q)
        assert gpu_lib.add_mod(a % q, b % q, q) == oracle.add_mod(a, b, q)
        assert gpu_lib.sub_mod(a % q, b % q, q) == oracle.sub_mod(a, b, q)
        assert gpu_lib.power_mod(a, b, q) == oracle.pow_mod(a, b, q)
        assert gpu_lib.inv_mod(a, q) == oracle.inv_mod(a, q)
    assert gpu_lib.multiply_mod(12345, 67890, 1000000007) == 838102050


def test_root_tables_match_oracle(gpu_lib, oracle):
    for n, q in [(8, 65537), (64, P.Q0), (1024, P.Q62)]:
        r = gpu_lib.get_roots(n, q)
        ri = gpu_lib.get_inv_roots(n, q)
        assert [r[i] for i in range(n)] == oracle.get_roots(n, q).tolist()
        assert [ri[i] for i in range(n)] == oracle.get_roots(n, q, inverse=True).tolist()
    assert not gpu_lib.get_roots(12, 65537)  # not a power of two
