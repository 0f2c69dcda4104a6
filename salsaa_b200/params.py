"""SALSAA parameter sets and the ctypes mirror of ``salsaa_params``.

The twelve presets are the cargo features of the reference
(src/protocol.rs:28-123): ring degree ``d`` (N), modulus ``q`` (MOD_Q),
commitment-key rows (MODULE_SIZE), witness width (WIT_LEN), rounds
(NOF_ROUNDS) and the SNARK / folding switch (FOLDING_SCHEME, which also sets
INIT_WIT_REP to 4).  DECOMP_PARTS is src/protocol.rs:26.
"""
import ctypes

Q0 = 1125899904679937
Q1 = 1125899906840833
Q2 = 1125899906822657
Q62 = 4546383823830515713  # the reference's unit-test / NTT-microbench prime

DECOMP_PARTS = [1] + [2] * 11


class SalsaaParams(ctypes.Structure):
    """Same layout as ``salsaa_params`` in include/salsaa_gpu.h."""

    _fields_ = [
        ("d", ctypes.c_uint64),
        ("q", ctypes.c_uint64),
        ("module_size", ctypes.c_uint64),
        ("wit_len", ctypes.c_uint64),
        ("init_wit_rep", ctypes.c_uint64),
        ("nof_rounds", ctypes.c_uint64),
        ("folding", ctypes.c_uint64),
        ("decomp_parts", ctypes.c_uint64 * 12),
    ]

    def as_dict(self):
        return {f: (list(getattr(self, f)) if f == "decomp_parts" else int(getattr(self, f)))
                for f, _ in self._fields_}


def make_params(d, q, module_size, wit_len, nof_rounds, folding=False, init_wit_rep=None,
                decomp_parts=None):
    p = SalsaaParams()
    p.d, p.q, p.module_size, p.wit_len = d, q, module_size, wit_len
    p.nof_rounds = nof_rounds
    p.folding = 1 if folding else 0
    p.init_wit_rep = init_wit_rep if init_wit_rep is not None else (4 if folding else 1)
    parts = decomp_parts if decomp_parts is not None else DECOMP_PARTS
    for i in range(12):
        p.decomp_parts[i] = parts[i] if i < len(parts) else parts[-1]
    return p


# name -> (d, q, MODULE_SIZE, WIT_LEN, NOF_ROUNDS, FOLDING_SCHEME)
PRESETS = {
    "A0": (128, Q0, 12, 1 << 19, 8, False),
    "A1": (256, Q1, 7, 1 << 18, 7, False),
    "A2": (512, Q2, 4, 1 << 17, 6, False),
    "B0": (128, Q0, 12, 1 << 21, 10, False),
    "B1": (256, Q1, 7, 1 << 20, 9, False),
    "B2": (512, Q2, 4, 1 << 19, 8, False),
    "C0": (128, Q0, 12, 1 << 23, 12, False),
    "C1": (256, Q1, 7, 1 << 22, 11, False),
    "C2": (512, Q2, 4, 1 << 21, 10, False),
    "F0": (128, Q0, 12, 1 << 17, 1, True),
    "F1": (128, Q0, 13, 1 << 19, 1, True),
    "F2": (128, Q0, 13, 1 << 21, 1, True),
}


def preset(name):
    d, q, ms, wl, nr, fold = PRESETS[name]
    return make_params(d, q, ms, wl, nr, fold)


def small_snark(d=16, q=Q0, module_size=3, log_len=13, rounds=2):
    """A SNARK instance small enough for the oracle to prove in well under a second."""
    return make_params(d, q, module_size, 1 << log_len, rounds, False)


def small_folding(d=16, q=Q0, module_size=3, log_len=11):
    return make_params(d, q, module_size, 1 << log_len, 1, True)
