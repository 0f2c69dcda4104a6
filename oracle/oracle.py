"""ctypes wrapper of the CPU oracle (libsalsaa_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the salsaa_b200 package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsalsaa_oracle.so")

U64 = ctypes.c_uint64
U64P = ctypes.POINTER(ctypes.c_uint64)
U8P = ctypes.POINTER(ctypes.c_uint8)


class SoTiming(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("commit", "norm1", "norm2", "norm3", "split", "projection", "fold", "decomp", "total")]

    def as_dict(self):
        return {n: float(getattr(self, n)) for n, _ in self._fields_}


def build():
    """Compile the oracle in place (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        for name in ("so_mul_mod", "so_add_mod", "so_sub_mod", "so_pow_mod"):
            getattr(L, name).restype = U64
            getattr(L, name).argtypes = [U64, U64, U64]
        L.so_inv_mod.restype = U64
        L.so_inv_mod.argtypes = [U64, U64]
        L.so_minimal_root.restype = U64
        L.so_minimal_root.argtypes = [U64, U64]
        L.so_prf.restype = U64
        L.so_prf.argtypes = [U64, U64, U64]
        for name in ("so_ntt_forward", "so_ntt_inverse"):
            getattr(L, name).restype = ctypes.c_int
            getattr(L, name).argtypes = [U64P, U64, U64]
        for name in ("so_get_roots", "so_get_inv_roots"):
            getattr(L, name).restype = ctypes.c_int
            getattr(L, name).argtypes = [U64, U64, U64P]
        L.so_multiply_poly.restype = ctypes.c_int
        L.so_multiply_poly.argtypes = [U64P, U64P, U64P, U64, U64]
        for name in ("so_eltwise_mult_mod", "so_eltwise_add_mod", "so_eltwise_sub_mod"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [U64P, U64P, U64P, U64, U64]
        L.so_eltwise_fma_mod.restype = None
        L.so_eltwise_fma_mod.argtypes = [U64P, U64P, U64, U64P, U64, U64]
        L.so_eltwise_reduce_mod.restype = None
        L.so_eltwise_reduce_mod.argtypes = [U64P, U64P, U64, U64]
        for name in ("so_sum", "so_sum_sq"):
            getattr(L, name).restype = U64
            getattr(L, name).argtypes = [U64P, U64, U64]
        for name in ("so_ring_to_slot", "so_ring_from_slot"):
            getattr(L, name).restype = ctypes.c_int
            getattr(L, name).argtypes = [U64P, U64P, U64, U64]
        L.so_ring_mul.restype = ctypes.c_int
        L.so_ring_mul.argtypes = [U64P, U64P, U64P, U64, U64]
        L.so_dense_commit.restype = ctypes.c_int
        L.so_dense_commit.argtypes = [U64P, U64P, U64P, U64, U64, U64, U64, U64]
        L.so_conjugate.restype = None
        L.so_conjugate.argtypes = [U64P, U64P, U64, U64]
        L.so_shift_factors.restype = ctypes.c_int
        L.so_shift_factors.argtypes = [U64P, U64, U64]
        L.so_tensor.restype = None
        L.so_tensor.argtypes = [U64P, U64P, U64, U64]
        L.so_sumcheck.restype = ctypes.c_int
        L.so_sumcheck.argtypes = [U64P, U64, U64, U64P, U64P, U64P, U64P]
        L.so_qnr.restype = U64
        L.so_qnr.argtypes = [U64]
        L.so_sumcheck_fq2.restype = ctypes.c_int
        L.so_sumcheck_fq2.argtypes = [U64P, U64, U64, U64, U64P, U64P, U64P, U64P]
        L.so_decompose.restype = ctypes.c_int
        L.so_decompose.argtypes = [U64P, U64, U64, U64, U64, U64, U64P, U64P]
        L.so_project.restype = ctypes.c_int
        L.so_project.argtypes = [U64P, U64, U64, U64, U64, U8P, U8P, U64P]
        L.so_commit_ck.restype = ctypes.c_int
        L.so_commit_ck.argtypes = [ctypes.c_void_p, U64, U64P, U64, U64, U64P]
        L.so_fold.restype = ctypes.c_int
        L.so_fold.argtypes = [U64P, U64, U64, U64, U64, U64P, U64P]
        L.so_sample_crs.restype = None
        L.so_sample_crs.argtypes = [ctypes.c_void_p, U64, U64P]
        L.so_sample_witness.restype = None
        L.so_sample_witness.argtypes = [ctypes.c_void_p, U64, U64P]
        L.so_proof_size.restype = U64
        L.so_proof_size.argtypes = [ctypes.c_void_p]
        L.so_prove.restype = ctypes.c_int
        L.so_prove.argtypes = [ctypes.c_void_p, U64, U64, U64P, U8P, U64, ctypes.POINTER(SoTiming),
                               ctypes.c_int]
        L.so_verify.restype = ctypes.c_int
        L.so_verify.argtypes = [ctypes.c_void_p, U64, U64, U8P, U64]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(U64P)


def _b(a):
    return a.ctypes.data_as(U8P)


def u64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


# ---- scalar / element-wise -------------------------------------------------
def mul_mod(a, b, q):
    return lib().so_mul_mod(a, b, q)


def add_mod(a, b, q):
    return lib().so_add_mod(a, b, q)


def sub_mod(a, b, q):
    return lib().so_sub_mod(a, b, q)


def pow_mod(a, e, q):
    return lib().so_pow_mod(a, e, q)


def inv_mod(a, q):
    return lib().so_inv_mod(a, q)


def minimal_root(order, q):
    return lib().so_minimal_root(order, q)


def prf(seed, domain, index):
    return lib().so_prf(seed, domain, index)


def eltwise(op, a, b, q):
    a, b = u64(a), u64(b)
    r = np.zeros_like(a)
    getattr(lib(), "so_eltwise_%s_mod" % op)(_p(r), _p(a), _p(b), a.size, q)
    return r


def eltwise_fma(a, s, b, q):
    a, b = u64(a), u64(b)
    r = np.zeros_like(a)
    lib().so_eltwise_fma_mod(_p(r), _p(a), s, _p(b), a.size, q)
    return r


def eltwise_reduce(a, q):
    a = u64(a)
    r = np.zeros_like(a)
    lib().so_eltwise_reduce_mod(_p(r), _p(a), a.size, q)
    return r


def sum_mod(a, q):
    a = u64(a)
    return lib().so_sum(_p(a), a.size, q)


def sum_sq(a, q):
    a = u64(a)
    return lib().so_sum_sq(_p(a), a.size, q)


# ---- NTT / ring ------------------------------------------------------------
def ntt_forward(a, q):
    """Batched: last axis is the polynomial."""
    a = u64(a).copy()
    n = a.shape[-1]
    flat = a.reshape(-1, n)
    for row in flat:
        assert lib().so_ntt_forward(_p(row), n, q) == 0
    return flat.reshape(a.shape)


def ntt_inverse(a, q):
    a = u64(a).copy()
    n = a.shape[-1]
    flat = a.reshape(-1, n)
    for row in flat:
        assert lib().so_ntt_inverse(_p(row), n, q) == 0
    return flat.reshape(a.shape)


def get_roots(n, q, inverse=False):
    out = np.zeros(n, dtype=np.uint64)
    fn = lib().so_get_inv_roots if inverse else lib().so_get_roots
    assert fn(n, q, _p(out)) == 0
    return out


def multiply_poly(a, b, q):
    a, b = u64(a), u64(b)
    r = np.zeros_like(a)
    assert lib().so_multiply_poly(_p(r), _p(a), _p(b), a.size, q) == 0
    return r


def ring_to_slot(a, q):
    a = u64(a)
    d = a.shape[-1]
    flat = a.reshape(-1, d)
    out = np.zeros_like(flat)
    for i in range(flat.shape[0]):
        assert lib().so_ring_to_slot(_p(out[i]), _p(np.ascontiguousarray(flat[i])), d, q) == 0
    return out.reshape(a.shape)


def ring_from_slot(a, q):
    a = u64(a)
    d = a.shape[-1]
    flat = a.reshape(-1, d)
    out = np.zeros_like(flat)
    for i in range(flat.shape[0]):
        assert lib().so_ring_from_slot(_p(out[i]), _p(np.ascontiguousarray(flat[i])), d, q) == 0
    return out.reshape(a.shape)


def ring_mul(a, b, q):
    a, b = u64(a), u64(b)
    r = np.zeros_like(a)
    assert lib().so_ring_mul(_p(r), _p(a), _p(b), a.size, q) == 0
    return r


def dense_commit(A, W, q):
    """C = A * W (src/arithmetic.rs:429-457): A n x m x d, W r x m x d -> n x r x d."""
    A, W = u64(A), u64(W)
    n, m, d = A.shape
    r = W.shape[0]
    C = np.zeros((n, r, d), dtype=np.uint64)
    assert lib().so_dense_commit(_p(C), _p(A), _p(W), n, m, r, d, q) == 0
    return C


def conjugate(a, q):
    a = u64(a)
    r = np.zeros_like(a)
    lib().so_conjugate(_p(r), _p(a), a.size, q)
    return r


def shift_factors(d, q):
    out = np.zeros(d // 2, dtype=np.uint64)
    assert lib().so_shift_factors(_p(out), d, q) == 0
    return out


def tensor(cs, q):
    cs = u64(cs)
    out = np.zeros(1 << cs.size, dtype=np.uint64)
    lib().so_tensor(_p(out), _p(cs), cs.size, q)
    return out


# ---- subroutines -------------------------------------------------------------
def sumcheck(w, q, cs):
    w, cs = u64(w), u64(cs)
    n = w.size
    nr = n.bit_length() - 1
    claim = U64(0)
    final = U64(0)
    polys = np.zeros((max(nr, 1), 3), dtype=np.uint64)
    assert lib().so_sumcheck(_p(w), n, q, _p(cs), ctypes.byref(claim), _p(polys), ctypes.byref(final)) == 0
    return int(claim.value), polys[:nr], int(final.value)


def qnr(q):
    return lib().so_qnr(q)


def sumcheck_fq2(w, q, shift, cs):
    """cs: log2(n) x 2 challenges (re, im) -> (claim, polys log2(n) x 3 x 2, final (re, im))."""
    w, cs = u64(w), u64(cs)
    n = w.size
    nr = n.bit_length() - 1
    claim = U64(0)
    final = np.zeros(2, dtype=np.uint64)
    polys = np.zeros((max(nr, 1), 3, 2), dtype=np.uint64)
    assert lib().so_sumcheck_fq2(_p(w), n, q, shift, _p(cs), ctypes.byref(claim), _p(polys), _p(final)) == 0
    return int(claim.value), polys[:nr], (int(final[0]), int(final[1]))


def decompose(w, q, parts):
    """w: rows x width x d (coefficient form)."""
    w = u64(w)
    rows, width, d = w.shape
    out = np.zeros((rows * parts, width, d), dtype=np.uint64)
    radix = U64(0)
    assert lib().so_decompose(_p(w), rows, width, d, q, parts, _p(out), ctypes.byref(radix)) == 0
    return out, int(radix.value)


def project(w, q, is_zero, sign):
    w = u64(w)
    rows, width, d = w.shape
    iz = np.ascontiguousarray(is_zero, dtype=np.uint8)
    sg = np.ascontiguousarray(sign, dtype=np.uint8)
    out = np.zeros((width, d), dtype=np.uint64)
    assert lib().so_project(_p(w), rows, width, d, q, _b(iz), _b(sg), _p(out)) == 0
    return out


def commit_ck(params, crs_seed, w):
    w = u64(w)
    rows, width, d = w.shape
    out = np.zeros((params.module_size, rows, d), dtype=np.uint64)
    assert lib().so_commit_ck(ctypes.byref(params), crs_seed, _p(w), rows, width, _p(out)) == 0
    return out


def fold(w, q, c):
    w, c = u64(w), u64(c)
    rows, width, d = w.shape
    out = np.zeros((width, d), dtype=np.uint64)
    assert lib().so_fold(_p(w), rows, width, d, q, _p(c), _p(out)) == 0
    return out


def sample_crs(params, crs_seed):
    out = np.zeros((params.module_size, params.d), dtype=np.uint64)
    lib().so_sample_crs(ctypes.byref(params), crs_seed, _p(out))
    return out


def sample_witness(params, seed):
    out = np.zeros((params.init_wit_rep, params.wit_len, params.d), dtype=np.uint64)
    lib().so_sample_witness(ctypes.byref(params), seed, _p(out))
    return out


def proof_size(params):
    return lib().so_proof_size(ctypes.byref(params))


def prove(params, crs_seed, seed, witness=None, nthreads=0):
    """Returns (rc, proof bytes as uint8 array, timing dict)."""
    n = proof_size(params)
    proof = np.zeros(n, dtype=np.uint8)
    t = SoTiming()
    wp = None
    if witness is not None:
        witness = u64(witness)
        wp = _p(witness)
    rc = lib().so_prove(ctypes.byref(params), crs_seed, seed, wp, _b(proof), n, ctypes.byref(t), nthreads)
    return rc, proof, t.as_dict()


def verify(params, crs_seed, seed, proof):
    proof = np.ascontiguousarray(proof, dtype=np.uint8)
    return lib().so_verify(ctypes.byref(params), crs_seed, seed, _b(proof), proof.size)
