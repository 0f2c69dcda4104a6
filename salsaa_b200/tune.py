"""Autotuner for the NTT kernel schedules of libsalsaa_gpu.so.

The register-path negacyclic NTT (salsaa_ntt and every transform inside the
prover) has several kernel schedules that give identical outputs: one
4096-coefficient tile per CTA with integer (64-bit Shoup) butterflies, the
same with FP64 butterflies (for the protocol's primes below 2^50), or
persistent CTAs that stage tiles through shared memory with bulk copies 2, 3
or 4 tiles ahead, optionally capped at one CTA per SM.  Which is fastest
depends on the transform size, the direction, the modulus width and the batch
size, so this script times every candidate on the GPU for each key (log2 n,
incomplete, inverse, q >= 2^50, large batch), checks that each candidate's
output equals the default schedule's bit for bit, and writes the winners to a
table the library loads at its first transform (tune_table.txt beside the
library, or $SALSAA_TUNE_FILE).  It also times the fold with integer and with
FP64 products.

Usage: python -m salsaa_b200.tune [--out PATH] [--reps K] [--quick]
"""
import argparse
import ctypes
import json
import os
import sys

from . import lib
from .params import Q0, Q1, Q2, Q62

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tune_table.txt")

# (variant, ctas_per_sm): 0 = one tile per CTA, integer butterflies; 1 = the
# same with FP64 butterflies (q < 2^50 only); 2..4 = bulk-copy stages ahead;
# 5..7 = bulk-copy stages 2..4 with FP64 butterflies (q < 2^50 only)
CANDIDATES = [(0, 0), (1, 0), (2, 0), (2, 1), (3, 0), (4, 0), (5, 0), (6, 0), (7, 0)]
SMALL_COEFFS = 1 << 20  # a "small" call (below the library's 2^22 large-batch class)
LARGE_COEFFS = 1 << 27  # a "large" call: 1 GiB of coefficients, far above L2


def targets(quick=False):
    """(label, n_arg, incomplete, q) of the transforms to tune: the prover's
    incomplete transforms at the protocol moduli (d = 128, 256, 512) and the
    microbench's full transforms at the 62-bit prime."""
    t = [("incomplete_d%d" % d, d, True, q) for d, q in ((128, Q0), (256, Q1), (512, Q2))]
    t += [("full_n%d" % n, n, False, Q62) for n in (64, 128, 256, 1024)]
    return t[:2] if quick else t


def _key(n_arg, incomplete, q, inverse, large):
    n = n_arg // 2 if incomplete else n_arg
    return (n.bit_length() - 1, int(incomplete), int(inverse), int(q >= (1 << 50)), int(large))


def _check(rc, what):
    if rc < 0:
        raise RuntimeError("%s failed: %s" % (what, lib().salsaa_last_error().decode()))
    return rc


def time_schedule(torch, x, out, n_arg, incomplete, q, inverse, reps):
    """Mean device milliseconds of one salsaa_ntt call (CUDA events, current stream)."""
    L = lib()
    count = x.numel() // n_arg
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        _check(L.salsaa_ntt(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), n_arg, count, q,
                            int(inverse), int(incomplete), st), "salsaa_ntt")

    call()
    call()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        call()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / reps


def tune(reps=10, quick=False, verbose=True):
    """Times every candidate for every target; returns the result records.
    Leaves the library with the winning schedules set."""
    import torch
    L = lib()
    torch.cuda.init()
    results = []
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    for label, n_arg, incomplete, q in targets(quick):
        for large in (False, True):
            coeffs = LARGE_COEFFS if large else SMALL_COEFFS
            x = torch.randint(0, 1 << 62, (coeffs // n_arg, n_arg), dtype=torch.int64, device="cuda",
                              generator=gen) % q
            out = torch.empty_like(x)
            ref = torch.empty_like(x)
            for inverse in (False, True):
                key = _key(n_arg, incomplete, q, inverse, large)
                times = {}
                for var, cps in CANDIDATES:
                    if var in (1, 5, 6, 7) and q >= (1 << 50):
                        continue
                    _check(L.salsaa_ntt_tune_set(key[0], key[1], key[2], key[3], key[4], var, cps), "tune_set")
                    ms = time_schedule(torch, x, out, n_arg, incomplete, q, inverse, reps)
                    if (var, cps) == (0, 0):
                        ref.copy_(out)
                    elif not torch.equal(out, ref):
                        raise RuntimeError("schedule %s of %s differs from the default schedule" % ((var, cps), label))
                    times[(var, cps)] = ms
                best = min(times, key=times.get)
                _check(L.salsaa_ntt_tune_set(key[0], key[1], key[2], key[3], key[4], best[0], best[1]), "tune_set")
                gbs = 16.0 * coeffs / (times[best] * 1e6)
                rec = {"target": label, "inverse": inverse, "large": large, "key": list(key),
                       "coefficients": coeffs, "best": list(best), "ms": {"%d/%d" % k: v for k, v in times.items()},
                       "default_ms": times[(0, 0)], "best_ms": times[best], "best_GB/s": gbs}
                results.append(rec)
                if verbose:
                    print("%-16s %s %s  default %.3f ms  best %s %.3f ms (%.0f GB/s)"
                          % (label, "inv" if inverse else "fwd", "large" if large else "small",
                             times[(0, 0)], best, times[best], gbs), flush=True)
            del x, out, ref
            torch.cuda.empty_cache()
    return results


def tune_fold(reps=10, verbose=True):
    """Times the fold (salsaa_fold: two rows of 2^18 ring elements, d = 128,
    the 50-bit prime) with integer and FP64 products, checks that both give
    the same words, and leaves the faster set.  Returns the timing record."""
    import torch
    L = lib()
    q, d, rows, width = Q0, 128, 2, 1 << 18
    gen = torch.Generator(device="cuda")
    gen.manual_seed(12)
    w = torch.randint(0, 1 << 62, (rows, width, d), dtype=torch.int64, device="cuda", generator=gen) % q
    c = torch.randint(0, 1 << 62, (rows, d), dtype=torch.int64, device="cuda", generator=gen) % q
    out = torch.empty((width, d), dtype=torch.int64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        _check(L.salsaa_fold(ctypes.c_void_p(w.data_ptr()), rows, width, d, q, ctypes.c_void_p(c.data_ptr()),
                             ctypes.c_void_p(out.data_ptr()), st), "salsaa_fold")

    times, ref = {}, None
    for var in (0, 1):
        _check(L.salsaa_fold_tune_set(var), "fold_tune_set")
        call()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            call()
        b.record()
        b.synchronize()
        times[var] = a.elapsed_time(b) / reps
        if ref is None:
            ref = out.clone()
        elif not torch.equal(out, ref):
            raise RuntimeError("fold variant %d differs from the integer products" % var)
    best = min(times, key=times.get)
    _check(L.salsaa_fold_tune_set(best), "fold_tune_set")
    if verbose:
        print("fold (salsaa_fold, 2 x 2^18 x 128)  int %.3f ms  fp64 %.3f ms  best %d" % (times[0], times[1], best),
              flush=True)
    return {"target": "fold", "ms": {str(k): v for k, v in times.items()}, "best": best}


def write_table(results, path, fold=None):
    with open(path, "w") as f:
        f.write("# NTT kernel schedules chosen by salsaa_b200/tune.py on %s\n" % _device_name())
        f.write("# ntt <log_n> <incomplete> <inverse> <wide_modulus> <large_batch> <variant> <ctas_per_sm>\n")
        if fold is not None:
            f.write("fold %d   # fold products: int %.4f ms, fp64 %.4f ms\n"
                    % (fold["best"], fold["ms"]["0"], fold["ms"]["1"]))
        for r in results:
            k, b = r["key"], r["best"]
            f.write("ntt %d %d %d %d %d %d %d   # %s %s %s: default %.4f ms, best %.4f ms\n"
                    % (k[0], k[1], k[2], k[3], k[4], b[0], b[1], r["target"], "inv" if r["inverse"] else "fwd",
                       "large" if r["large"] else "small", r["default_ms"], r["best_ms"]))


def _device_name():
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown device"


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--json", default=None, help="also write the timing records here")
    a = ap.parse_args(argv)
    res = tune(a.reps, a.quick)
    fold = tune_fold(a.reps)
    write_table(res, a.out, fold)
    if a.json:
        with open(a.json, "w") as f:
            json.dump({"ntt": res, "fold": fold}, f, indent=1)
    print("wrote", a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
