"""Shared helpers for the tests (test code only)."""
import numpy as np

DOM_CRS, DOM_WIT, DOM_NC, DOM_PROJ, DOM_FOLD = 1, 2, 3, 4, 5


def domain(kind, a, b):
    return (kind << 56) | (a << 24) | b


def rand_mod(rng, shape, q):
    """Uniform residues in [0, q) (q < 2^62) from a seeded numpy generator."""
    hi = rng.integers(0, 1 << 31, size=shape, dtype=np.uint64)
    lo = rng.integers(0, 1 << 31, size=shape, dtype=np.uint64)
    return ((hi << np.uint64(31)) | lo) % np.uint64(q)


def small_signed(rng, shape, bound, q):
    """Values in [-bound, bound] as residues mod q."""
    v = rng.integers(-bound, bound + 1, size=shape)
    return np.where(v < 0, q + v, v).astype(np.uint64)


M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15


def _mix64_int(z):
    z &= M64
    z ^= z >> 30
    z = (z * 0xBF58476D1CE4E5B9) & M64
    z ^= z >> 27
    z = (z * 0x94D049BB133111EB) & M64
    z ^= z >> 31
    return z


def _mix64_np(z):
    with np.errstate(over="ignore"):
        z = z ^ (z >> np.uint64(30))
        z = z * np.uint64(0xBF58476D1CE4E5B9)
        z = z ^ (z >> np.uint64(27))
        z = z * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def prf_np(seed, dom, idx):
    """Vectorised copy of the PRF (so_prf) for building test inputs."""
    key = _mix64_int(seed ^ _mix64_int(dom + GOLDEN))
    idx = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _mix64_np(np.uint64(key) + idx * np.uint64(GOLDEN))


def proj_challenge(seed, round_, cw):
    """The projection challenge J of (seed, round) as is_zero / sign bytes (256 x cw)."""
    r = prf_np(seed, domain(DOM_PROJ, round_, 0), np.arange(256 * cw, dtype=np.uint64)).reshape(256, cw)
    return (r & np.uint64(1)).astype(np.uint8), ((r >> np.uint64(1)) & np.uint64(1)).astype(np.uint8)


def fold_challenge(seed, round_, rows, d, q):
    r = prf_np(seed, domain(DOM_FOLD, round_, 0), np.arange(rows * d, dtype=np.uint64))
    t = np.array([(int(x) * 3) >> 64 for x in r], dtype=np.uint64)
    out = np.where(t == 0, np.uint64(q - 1), np.where(t == 1, np.uint64(0), np.uint64(1)))
    return out.reshape(rows, d).astype(np.uint64)


def nc_challenges(seed, round_, rep, nr, q):
    r = prf_np(seed, domain(DOM_NC, round_, rep), np.arange(nr, dtype=np.uint64))
    return np.array([(int(x) * q) >> 64 for x in r], dtype=np.uint64)
