"""Host-side mirror of the reference's prover interface over the C ABI.

Function names follow the reference (src/protocol.rs, src/subroutines/*,
src/arithmetic.rs) so that tests read like its own; the arguments are device
tensors (torch, int64 storage holding the u64 residues bit-for-bit) or numpy
uint64 arrays for the host-buffer entry points.  Every call goes to
libsalsaa_gpu.so; there is no CPU path here.
"""
import ctypes

import numpy as np

from . import lib
from ._abi import SalsaaTiming
from .params import SalsaaParams


class SalsaaError(RuntimeError):
    pass


def _check(rc, what):
    if rc:
        msg = lib().salsaa_last_error()
        raise SalsaaError("%s failed (%d): %s" % (what, rc, msg.decode() if msg else ""))


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise SalsaaError("no CUDA device visible: the SALSAA prover runs on the GPU only")
    return torch


# ---- device buffers ---------------------------------------------------------
def to_dev(a):
    """numpy uint64 array -> CUDA int64 tensor with identical bits."""
    torch = _torch()
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
    return torch.from_numpy(a.view(np.int64)).cuda()


def to_host(t):
    """CUDA int64 tensor -> numpy uint64 array with identical bits."""
    return t.detach().cpu().contiguous().numpy().view(np.uint64)


def dev_empty(shape):
    torch = _torch()
    return torch.empty(shape, dtype=torch.int64, device="cuda")


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# ---- parameter sets -----------------------------------------------------------
def params_preset(name):
    p = SalsaaParams()
    _check(lib().salsaa_params_preset(name.encode(), ctypes.byref(p)), "params_preset")
    return p


def proof_size(params):
    return int(lib().salsaa_proof_size(ctypes.byref(params)))


def workspace_bytes(params):
    return int(lib().salsaa_workspace_bytes(ctypes.byref(params)))


# ---- context / prover -----------------------------------------------------------
class Context:
    """CRS::gen_crs + compute_commitment_keys on one GPU (src/subroutines/crs.rs:23-72)."""

    def __init__(self, params, crs_seed=0, device=0):
        self.params = params
        self.crs_seed = crs_seed
        self.device = device
        h = ctypes.c_void_p()
        _check(lib().salsaa_ctx_create(ctypes.byref(params), crs_seed, device, ctypes.byref(h)), "ctx_create")
        self.h = h
        self.proof_bytes = proof_size(params)

    def close(self):
        if self.h:
            lib().salsaa_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prove(self, seed, witness=None):
        """protocol() through host buffers: returns the proof bytes (numpy uint8)."""
        out = np.zeros(self.proof_bytes, dtype=np.uint8)
        wp = None
        if witness is not None:
            witness = np.ascontiguousarray(witness, dtype=np.uint64)
            p = self.params
            assert witness.size == p.init_wit_rep * p.wit_len * p.d
            wp = witness.ctypes.data_as(ctypes.c_void_p)
        _check(lib().salsaa_prove(self.h, seed, wp, out.ctypes.data_as(ctypes.c_void_p), out.size), "prove")
        return out

    def verify(self, seed, proof):
        """The reference verifier's checks on proof bytes (GPU-checked final
        statement); returns 0 for accept, else the code of the failed check."""
        proof = np.ascontiguousarray(proof, dtype=np.uint8)
        verdict = ctypes.c_int(0)
        _check(lib().salsaa_verify(self.h, seed, proof.ctypes.data_as(ctypes.c_void_p), proof.size,
                                   ctypes.byref(verdict)), "verify")
        return verdict.value

    def parallel_dot_series_matrix(self, w):
        """Commitment-key rows times the witness rows (src/arithmetic.rs:459-505).
        w: CUDA tensor rows x width x d (coefficients) -> module_size x rows x d."""
        rows, width, d = w.shape
        out = dev_empty((self.params.module_size, rows, d))
        _check(lib().salsaa_commit(self.h, _p(w), rows, width, _p(out), _stream()), "commit")
        return out

    def parallel_dot_series_matrix_multi(self, ws):
        """The same for several witnesses of uneven shapes in one launch of
        each step (salsaa_commit_multi); returns one output per witness."""
        k = len(ws)
        outs = [dev_empty((self.params.module_size, w.shape[0], w.shape[2])) for w in ws]
        wp = (ctypes.c_void_p * k)(*[w.data_ptr() for w in ws])
        op = (ctypes.c_void_p * k)(*[o.data_ptr() for o in outs])
        rows = (ctypes.c_uint64 * k)(*[w.shape[0] for w in ws])
        widths = (ctypes.c_uint64 * k)(*[w.shape[1] for w in ws])
        _check(lib().salsaa_commit_multi(self.h, wp, rows, widths, k, op, _stream()), "commit_multi")
        return outs


class Prover:
    """One proof slot (device workspace + private stream) of a Context."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = ctypes.c_void_p()
        _check(lib().salsaa_prover_create(ctx.h, ctypes.byref(h)), "prover_create")
        self.h = h

    def close(self):
        if self.h:
            lib().salsaa_prover_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return lib().salsaa_prover_stream(self.h)

    def enqueue(self, seed, d_proof, d_witness=None):
        _check(lib().salsaa_prover_enqueue(self.h, seed, _p(d_witness), _p(d_proof)), "prover_enqueue")

    def enqueue_host(self, seed, h_proof, h_witness=None):
        """Asynchronous prove through (preferably page-locked) host buffers."""
        wp = None if h_witness is None else ctypes.c_void_p(h_witness.ctypes.data)
        _check(lib().salsaa_prover_enqueue_host(self.h, seed, wp, ctypes.c_void_p(h_proof.ctypes.data)),
               "prover_enqueue_host")

    def enqueue_host_i8(self, seed, h_proof, h_witness):
        """As enqueue_host, with the short witness as centred int8
        coefficients (one byte each on the bus instead of eight)."""
        if h_witness.dtype != np.int8:
            raise TypeError("enqueue_host_i8: witness must be int8")
        _check(lib().salsaa_prover_enqueue_host_i8(self.h, seed, ctypes.c_void_p(h_witness.ctypes.data),
                                                   ctypes.c_void_p(h_proof.ctypes.data)),
               "prover_enqueue_host_i8")

    def set_overlap(self, on=True):
        """Run each round's projection beside the norm check (lower latency
        for a proof alone on the GPU; off by default)."""
        _check(lib().salsaa_prover_set_overlap(self.h, 1 if on else 0), "prover_set_overlap")

    def set_graph(self, on=True):
        """Replay a captured CUDA graph of the proof for later proofs into
        the same buffers (fewer launch gaps; off by default)."""
        _check(lib().salsaa_prover_set_graph(self.h, 1 if on else 0), "prover_set_graph")

    def query(self):
        rc = lib().salsaa_prover_query(self.h)
        if rc < 0:
            _check(rc, "prover_query")
        return rc

    def sync(self):
        _check(lib().salsaa_prover_sync(self.h), "prover_sync")

    def timing(self):
        t = SalsaaTiming()
        _check(lib().salsaa_prover_timing(self.h, ctypes.byref(t)), "prover_timing")
        return t.as_dict()


# ---- subroutine-level entry points -------------------------------------------------
def ntt(x, n, q, inverse=False, incomplete=False, out=None):
    """Batched negacyclic NTT of a CUDA tensor whose last axis has n (or d) words."""
    count = x.numel() // n
    out = x if out is None else out
    _check(lib().salsaa_ntt(_p(x), _p(out), n, count, q, int(inverse), int(incomplete), _stream()), "ntt")
    return out


def ntt_multi(xs, n, q, inverse=False, incomplete=False, outs=None):
    """Several uneven batches (CUDA tensors whose last axis has n, or d,
    words) transformed in one launch; in place unless outs is given."""
    outs = list(xs) if outs is None else list(outs)
    k = len(xs)
    ins = (ctypes.c_void_p * k)(*[x.data_ptr() for x in xs])
    ous = (ctypes.c_void_p * k)(*[o.data_ptr() for o in outs])
    counts = (ctypes.c_uint64 * k)(*[x.numel() // n for x in xs])
    _check(lib().salsaa_ntt_multi(ins, ous, counts, k, n, q, int(inverse), int(incomplete), _stream()), "ntt_multi")
    return outs


def poly_mul(a, b, n, q, out=None):
    """Batched negacyclic product of CUDA tensors whose last axis has n words
    (multiply_poly, hexl-bindings/hexl_wrapper.cpp, for many pairs at once)."""
    count = a.numel() // n
    out = dev_empty(a.shape) if out is None else out
    _check(lib().salsaa_poly_mul(_p(a), _p(b), _p(out), n, count, q, _stream()), "poly_mul")
    return out


def sum_check_batch(vecs, q, seed, round_):
    """Independent sumchecks of a list of CUDA vectors (power-of-two lengths,
    one repetition each, instance i on the challenge stream (round, i)) ->
    (claims[count], [polys_i of shape (log2 len_i, 3)])."""
    count = len(vecs)
    ptrs = (ctypes.c_void_p * count)(*[v.data_ptr() for v in vecs])
    lens = (ctypes.c_uint64 * count)(*[v.numel() for v in vecs])
    nrs = [v.numel().bit_length() - 1 for v in vecs]
    claims = dev_empty((count,))
    polys = dev_empty((max(sum(nrs), 1), 3))
    _check(lib().salsaa_sumcheck_batch(ptrs, lens, count, q, seed, round_, _p(claims), _p(polys), _stream()),
           "sumcheck_batch")
    out, o = [], 0
    for nr in nrs:
        out.append(polys[o:o + nr])
        o += nr
    return claims, out



def fq2_shift(q):
    """The non-residue s of F_{q^2} = F_q[X]/(X^2 - s) used by sum_check_fq2_batch."""
    return int(lib().salsaa_fq2_shift(q))


def sum_check_fq2_batch(vecs, q, seed, round_):
    """The sumcheck over F_{q^2} of a list of CUDA vectors (F_q entries,
    power-of-two lengths) -> (claims[count], [polys_i of shape (log2 len_i, 3, 2)])."""
    count = len(vecs)
    ptrs = (ctypes.c_void_p * count)(*[v.data_ptr() for v in vecs])
    lens = (ctypes.c_uint64 * count)(*[v.numel() for v in vecs])
    nrs = [v.numel().bit_length() - 1 for v in vecs]
    claims = dev_empty((count,))
    polys = dev_empty((max(sum(nrs), 1), 3, 2))
    _check(lib().salsaa_sumcheck_fq2_batch(ptrs, lens, count, q, seed, round_, _p(claims), _p(polys), _stream()),
           "sumcheck_fq2_batch")
    out, o = [], 0
    for nr in nrs:
        out.append(polys[o:o + nr])
        o += nr
    return claims, out


class DenseKey:
    """Ajtai commitment key A (n x m ring elements, coefficient form) for
    C = A * W (parallel_dot_matrix_matrix, src/arithmetic.rs:429-457)."""

    def __init__(self, a, q):
        n, m, d = a.shape
        self.n, self.m, self.d, self.q = n, m, d, q
        self._h = ctypes.c_void_p()
        _check(lib().salsaa_dense_key_create(_p(a), n, m, d, q, _stream(), ctypes.byref(self._h)),
               "dense_key_create")

    def commit(self, w, out=None, w_slot=None):
        """w: r x m x d CUDA tensor (columns of W) -> n x r x d commitment."""
        r = w.shape[0]
        out = dev_empty((self.n, r, self.d)) if out is None else out
        _check(lib().salsaa_dense_commit(self._h, _p(w), r, _p(out), _p(w_slot) if w_slot is not None else None,
                                         _stream()), "dense_commit")
        return out

    def close(self):
        if self._h:
            lib().salsaa_dense_key_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def selftest_umma_i8(a, b):
    """Exact u8 product on the tensor cores: a (128 x k), b (n x k) uint8 numpy
    arrays -> int32 numpy (128 x n) = a @ b.T."""
    torch = _torch()
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    n, k = b.shape
    ta = torch.from_numpy(a).cuda()
    tb = torch.from_numpy(b).cuda()
    out = torch.empty((128, n), dtype=torch.int32, device="cuda")
    _check(lib().salsaa_selftest_umma_i8(_p(ta), _p(tb), n, k, _p(out), _stream()), "selftest_umma_i8")
    return out.cpu().numpy()


def sum_check(w, d, q, seed, round_):
    """norm_check_1 + both sum_check repetitions (src/subroutines/fast_norm_check.rs:135-320).
    w: CUDA tensor rows x n -> (claims[rows], polys[2, log2 n, rows, 3])."""
    rows = w.shape[0]
    n = w.numel() // rows
    nr = n.bit_length() - 1
    claims = dev_empty((rows,))
    polys = dev_empty((2, nr, rows, 3))
    _check(lib().salsaa_sumcheck(_p(w), rows, n, d, q, seed, round_, _p(claims), _p(polys), _stream()), "sumcheck")
    return claims, polys


def decompose_matrix_by_chunks(w, q, parts):
    """src/arithmetic.rs:1572-1593: rows x width x d -> ((rows*parts) x width x d, radix)."""
    rows, width, d = w.shape
    out = dev_empty((rows * parts, width, d))
    radix = dev_empty((1,))
    _check(lib().salsaa_decompose(_p(w), rows, width, d, q, parts, _p(out), _p(radix), _stream()), "decompose")
    return out, radix


def project(w, q, seed, round_):
    """src/subroutines/project.rs:50-103: rows x width x d -> width x d."""
    rows, width, d = w.shape
    out = dev_empty((width, d))
    _check(lib().salsaa_project(_p(w), rows, width, d, q, seed, round_, _p(out), _stream()), "project")
    return out


def fold(w, q, c):
    """src/subroutines/fold.rs:22-27: rows x width x d with rows ring challenges -> width x d."""
    rows, width, d = w.shape
    out = dev_empty((width, d))
    _check(lib().salsaa_fold(_p(w), rows, width, d, q, _p(c), _p(out), _stream()), "fold")
    return out


# ---- HEXL-compatible tier (host buffers) -------------------------------------------
def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def hexl_call(name, *args):
    """Call a HEXL-compatible symbol; numpy arrays are passed as uint64*."""
    conv = [(_u64p(a) if isinstance(a, np.ndarray) else a) for a in args]
    return getattr(lib(), name)(*conv)


# ---- serving --------------------------------------------------------------------
class Server:
    """Continuous-batching proof service on one GPU (salsaa_server_* in the C ABI)."""

    def __init__(self, hbm_budget_bytes, device=0):
        h = ctypes.c_void_p()
        _check(lib().salsaa_server_create(device, hbm_budget_bytes, ctypes.byref(h)), "server_create")
        self.h = h
        self.sets = []

    def register(self, params, crs_seed=0, slots=1):
        sid = ctypes.c_int()
        _check(lib().salsaa_server_register(self.h, ctypes.byref(params), crs_seed, slots, ctypes.byref(sid)),
               "server_register")
        self.sets.append(params)
        return sid.value

    def submit(self, set_id, seed, d_proof, d_witness=None):
        t = ctypes.c_uint64()
        _check(lib().salsaa_server_submit(self.h, set_id, seed, _p(d_witness), _p(d_proof), ctypes.byref(t)),
               "server_submit")
        return t.value

    def limit(self, max_inflight):
        """Cap the proofs running at once (0 = only the slots limit)."""
        _check(lib().salsaa_server_limit(self.h, max_inflight), "server_limit")

    def progress(self):
        rc = lib().salsaa_server_progress(self.h)
        if rc < 0:
            _check(rc, "server_progress")
        return rc

    def poll(self, ticket):
        """None while pending, else (latency_ms, run_ms)."""
        lat, run = ctypes.c_double(), ctypes.c_double()
        rc = lib().salsaa_server_poll(self.h, ticket, ctypes.byref(lat), ctypes.byref(run))
        if rc == 1:
            return None
        _check(rc, "server_poll")
        return lat.value, run.value

    def cancel(self, ticket):
        """True if the queued request was withdrawn, False if it already runs."""
        rc = lib().salsaa_server_cancel(self.h, ticket)
        if rc < 0:
            _check(rc, "server_cancel")
        return rc == 0

    def close(self):
        if self.h:
            lib().salsaa_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
