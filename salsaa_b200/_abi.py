"""ctypes signatures of include/salsaa_gpu.h."""
import ctypes

from .params import SalsaaParams

U64 = ctypes.c_uint64
U64P = ctypes.POINTER(ctypes.c_uint64)
U8P = ctypes.POINTER(ctypes.c_uint8)
VP = ctypes.c_void_p
INT = ctypes.c_int
SIZE = ctypes.c_size_t


class SalsaaTiming(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("commit", "norm1", "norm2", "norm3", "split", "projection", "fold", "decomp", "total")]

    def as_dict(self):
        return {n: float(getattr(self, n)) for n, _ in self._fields_}


# name -> (restype, argtypes); the twenty HEXL-compatible symbols first
HEXL_SYMBOLS = {
    "multiply_mod": (U64, [U64, U64, U64]),
    "add_mod": (U64, [U64, U64, U64]),
    "sub_mod": (U64, [U64, U64, U64]),
    "power_mod": (U64, [U64, U64, U64]),
    "inv_mod": (U64, [U64, U64]),
    "get_roots": (U64P, [SIZE, U64]),
    "get_inv_roots": (U64P, [SIZE, U64]),
    "eltwise_mult_mod": (None, [U64P, U64P, U64P, U64, U64]),
    "eltwise_fma_mod": (None, [U64P, U64P, U64, U64P, U64, U64]),
    "eltwise_add_mod": (None, [U64P, U64P, U64P, SIZE, U64]),
    "eltwise_sub_mod": (None, [U64P, U64P, U64P, SIZE, U64]),
    "eltwise_reduce_mod": (None, [U64P, U64P, SIZE, U64]),
    "eltwise_reduce_mod_naive": (None, [U64P, U64P, SIZE, U64]),
    "multiply_poly": (None, [U64P, U64P, U64P, U64, U64]),
    "polynomial_multiply_cyclotomic_mod": (None, [U64P, U64P, U64P, SIZE, U64]),
    "ntt_forward_in_place": (None, [U64P, SIZE, U64]),
    "ntt_inverse_in_place": (None, [U64P, SIZE, U64]),
    "sum": (U64, [U64P, U64, U64]),
    "sum_fast": (U64, [U64P, U64, U64]),
    "sum_sq": (U64, [U64P, U64, U64]),
    "sum_sq_fast": (U64, [U64P, U64, U64]),
}

PP = ctypes.POINTER(SalsaaParams)
DEVICE_SYMBOLS = {
    "salsaa_last_error": (ctypes.c_char_p, []),
    "salsaa_kernel_launches": (U64, []),
    "salsaa_device_status": (INT, []),
    "salsaa_trace_enable": (None, [INT]),
    "salsaa_trace_read": (INT, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(U64)]),
    "salsaa_params_preset": (INT, [ctypes.c_char_p, PP]),
    "salsaa_proof_size": (U64, [PP]),
    "salsaa_workspace_bytes": (U64, [PP]),
    "salsaa_ctx_create": (INT, [PP, U64, INT, ctypes.POINTER(VP)]),
    "salsaa_ctx_destroy": (None, [VP]),
    "salsaa_prover_create": (INT, [VP, ctypes.POINTER(VP)]),
    "salsaa_prover_destroy": (None, [VP]),
    "salsaa_prover_stream": (VP, [VP]),
    "salsaa_prover_enqueue": (INT, [VP, U64, VP, VP]),
    "salsaa_prover_enqueue_host": (INT, [VP, U64, VP, VP]),
    "salsaa_prover_enqueue_host_i8": (INT, [VP, U64, VP, VP]),
    "salsaa_prover_query": (INT, [VP]),
    "salsaa_prover_sync": (INT, [VP]),
    "salsaa_prover_timing": (INT, [VP, ctypes.POINTER(SalsaaTiming)]),
    "salsaa_prove": (INT, [VP, U64, VP, VP, U64]),
    "salsaa_verify": (INT, [VP, U64, VP, U64, VP]),
    "salsaa_prover_set_overlap": (INT, [VP, INT]),
    "salsaa_prover_set_graph": (INT, [VP, INT]),
    "salsaa_ntt": (INT, [VP, VP, U64, U64, U64, INT, INT, VP]),
    "salsaa_poly_mul": (INT, [VP, VP, VP, U64, U64, U64, VP]),
    "salsaa_ntt_multi": (INT, [ctypes.POINTER(VP), ctypes.POINTER(VP), ctypes.POINTER(U64), ctypes.c_uint32, U64,
                               U64, INT, INT, VP]),
    "salsaa_sumcheck_batch": (INT, [ctypes.POINTER(VP), ctypes.POINTER(U64), ctypes.c_uint32, U64, U64, U64, VP,
                                    VP, VP]),
    "salsaa_fq2_shift": (U64, [U64]),
    "salsaa_sumcheck_fq2_batch": (INT, [ctypes.POINTER(VP), ctypes.POINTER(U64), ctypes.c_uint32, U64, U64, U64,
                                        VP, VP, VP]),
    "salsaa_dense_key_create": (INT, [VP, U64, U64, U64, U64, VP, ctypes.POINTER(VP)]),
    "salsaa_dense_key_destroy": (None, [VP]),
    "salsaa_dense_commit": (INT, [VP, VP, U64, VP, VP, VP]),
    "salsaa_selftest_umma_i8": (INT, [VP, VP, ctypes.c_uint32, ctypes.c_uint32, VP, VP]),
    "salsaa_commit": (INT, [VP, VP, U64, U64, VP, VP]),
    "salsaa_commit_multi": (INT, [VP, ctypes.POINTER(VP), ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.c_uint32,
                                  ctypes.POINTER(VP), VP]),
    "salsaa_sumcheck": (INT, [VP, U64, U64, U64, U64, U64, U64, VP, VP, VP]),
    "salsaa_decompose": (INT, [VP, U64, U64, U64, U64, U64, VP, VP, VP]),
    "salsaa_project": (INT, [VP, U64, U64, U64, U64, U64, U64, VP, VP]),
    "salsaa_fold": (INT, [VP, U64, U64, U64, U64, VP, VP, VP]),
    "salsaa_project_noalloc": (INT, [VP, U64, U64, U64, U64, U64, U64, VP, VP]),
    "salsaa_server_create": (INT, [INT, U64, ctypes.POINTER(VP)]),
    "salsaa_server_register": (INT, [VP, PP, U64, ctypes.c_uint32, ctypes.POINTER(INT)]),
    "salsaa_server_submit": (INT, [VP, INT, U64, VP, VP, ctypes.POINTER(U64)]),
    "salsaa_server_limit": (INT, [VP, ctypes.c_uint32]),
    "salsaa_server_progress": (INT, [VP]),
    "salsaa_server_poll": (INT, [VP, U64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "salsaa_server_cancel": (INT, [VP, U64]),
    "salsaa_server_destroy": (None, [VP]),
    "salsaa_tune_load": (INT, [ctypes.c_char_p]),
    "salsaa_tune_reset": (INT, []),
    "salsaa_fold_tune_set": (INT, [INT]),
    "salsaa_fold_tune_get": (INT, []),
    "salsaa_ntt_tune_set": (INT, [ctypes.c_uint32, INT, INT, INT, INT, INT, INT]),
    "salsaa_ntt_tune_get": (INT, [ctypes.c_uint32, INT, INT, INT, INT, ctypes.POINTER(INT), ctypes.POINTER(INT)]),
}

ALL_SYMBOLS = {**HEXL_SYMBOLS, **DEVICE_SYMBOLS}


def bind(L):
    for name, (res, args) in ALL_SYMBOLS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L
