#!/usr/bin/env python
"""SALSAA prover benchmark on B200: proofs/s and p50/p99 prove latency of the
A0 SNARK parameter set (d=128, q=1125899904679937, 12 commitment-key rows,
WIT_LEN=2^19, 8 rounds; src/protocol.rs:28-35), batched prover vs the plain
one-proof-at-a-time GPU path, plus the negacyclic NTT's HBM throughput.

One JSON line on rank 0.  A step is one batch of `--slots` proofs proved
concurrently (one CUDA stream and workspace per slot), each over its own
synthetic ternary witness resident in HBM (P(0)=1/2, P(+-1)=1/4, the
reference's random_bounded(2)) and its own seed.  Witnesses are 512 MiB each,
larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (under torchrun) every rank proves its own batches: proofs
are independent, so this is replicas with no collective on the data path;
the timed region is bracketed by barriers and the max over ranks is used.

--impl reference times the CPU implementation of the same workload on this
host's cores (the C restatement under oracle/, since the Rust + Intel HEXL
reference cannot be built here) on a bounded sample: the A0 shape with
WIT_LEN=2^15 and 4 rounds, scaled by 16 (prover work is linear in WIT_LEN).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PRESET = "A0"
CPU_SAMPLE_LOG_LEN = 15
CPU_SAMPLE_ROUNDS = 4
CPU_SCALE = 1 << (19 - CPU_SAMPLE_LOG_LEN)
WORKLOAD = ("A0 SNARK prove: d=128, q=1125899904679937, module_size=12, wit_len=2^19, 8 rounds, "
            "ternary witness")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slots", type=int, default=8, help="proofs in flight per GPU (batch)")
    ap.add_argument("--plain-proofs", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ntt", action="store_true")
    ap.add_argument("--preset", default=PRESET, help="parameter set (profiling; the metric is quoted on A0)")
    ap.add_argument("--wit-log", type=int, default=0,
                    help="profiling: shrink WIT_LEN to 2^L (SNARK rounds L-11), keeping d, q and the rows")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU leg: the oracle port on a bounded sample
# ---------------------------------------------------------------------------
def cpu_sample_seconds(threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from salsaa_b200 import params as P
    p = P.make_params(128, P.Q0, 12, 1 << CPU_SAMPLE_LOG_LEN, CPU_SAMPLE_ROUNDS, False)
    t0 = time.perf_counter()
    rc, _, _ = O.prove(p, 1, 2, nthreads=threads)
    el = time.perf_counter() - t0
    if rc:
        raise RuntimeError("oracle prove failed: %d" % rc)
    return el


def cpu_baseline(threads):
    el = cpu_sample_seconds(threads)
    return {"value": 1.0 / (el * CPU_SCALE), "unit": "proofs/s", "cores": threads, "kind": "port",
            "sample": "A0 shape with wit_len=2^%d and %d rounds (1/%d of the witness), %.2f s, scaled x%d"
                      % (CPU_SAMPLE_LOG_LEN, CPU_SAMPLE_ROUNDS, CPU_SCALE, el, CPU_SCALE)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample_seconds(threads)
    times = [cpu_sample_seconds(threads) for _ in range(args.steps)]
    tot = sum(times) * CPU_SCALE
    value = args.steps / tot
    line = {
        "impl": "reference", "metric": "proofs/s", "value": value, "unit": "proofs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64 mod q", "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch": 1, "parallelism": "cpu threads %d" % threads},
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "port",
                         "sample": "A0 shape with wit_len=2^%d and %d rounds per step, scaled x%d"
                                   % (CPU_SAMPLE_LOG_LEN, CPU_SAMPLE_ROUNDS, CPU_SCALE)},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1000.0 * statistics.median(times) * CPU_SCALE,
        "p99_ms": 1000.0 * max(times) * CPU_SCALE,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or parts[0] != str(self.gpu):
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
def ternary_witness(torch, shape, q, gen):
    r = torch.randint(0, 4, shape, dtype=torch.int64, device="cuda", generator=gen)
    w = torch.zeros(shape, dtype=torch.int64, device="cuda")
    w[r == 2] = 1
    w[r == 3] = np.int64(q - 1)
    return w


def run_ours(args):
    import torch
    import torch.distributed as dist
    from salsaa_b200 import api, lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    params = api.params_preset(args.preset)
    if args.wit_log:
        params.wit_len = 1 << args.wit_log
        if not params.folding:
            params.nof_rounds = args.wit_log - 11
    q = params.q
    ctx = api.Context(params, crs_seed=1, device=local)
    S = args.slots
    slots = [api.Prover(ctx) for _ in range(S)]
    words = ctx.proof_bytes // 8
    proofs = [torch.empty(words, dtype=torch.int64, device="cuda") for _ in range(S)]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    wshape = (params.init_wit_rep, params.wit_len, params.d)
    witnesses = [ternary_witness(torch, wshape, q, gen) for _ in range(S)]
    ext = [torch.cuda.ExternalStream(pr.stream) for pr in slots]
    main = torch.cuda.current_stream()
    torch.cuda.synchronize()

    def batch(step, start_ev):
        done = []
        for i in range(S):
            ext[i].wait_event(start_ev)
            slots[i].enqueue(seed=(rank << 40) + step * S + i + 1, d_proof=proofs[i], d_witness=witnesses[i])
            e = torch.cuda.Event(enable_timing=True)
            e.record(ext[i])
            main.wait_event(e)
            done.append(e)
        return done

    # warm-up
    for w in range(args.warmup):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(main)
        batch(-1 - w, ev)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = lib().salsaa_kernel_launches()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(main)
    lat = []
    step_events = []
    for s in range(args.steps):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(main)
        step_events.append((ev, batch(s, ev)))
    t_end.record(main)
    t_end.synchronize()
    launches = lib().salsaa_kernel_launches() - launches0
    elapsed_ms = t_start.elapsed_time(t_end)
    for ev, done in step_events:
        lat += [ev.elapsed_time(e) for e in done]
    clk = clocks.stop()
    barrier()
    elapsed_ms = max_over_ranks(elapsed_ms)
    total = S * args.steps * world
    value = total / (elapsed_ms / 1000.0)
    timing = slots[0].timing()

    # correctness spot check of the last batch: first proof verifies on the CPU
    check = None
    if rank == 0 and args.steps > 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        try:
            import oracle as O
            pb = api.to_host(proofs[0]).view(np.uint8)
            check = O.verify(params, 1, (rank << 40) + (args.steps - 1) * S + 1, pb) == 0
        except Exception as e:  # the checker is optional here; tests own parity
            check = "not run: %s" % e

    # plain path: one proof at a time on one slot
    plain = []
    for i in range(args.plain_proofs):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(ext[0])
        slots[0].enqueue(seed=10 ** 6 + i, d_proof=proofs[0], d_witness=witnesses[0])
        b.record(ext[0])
        b.synchronize()
        if i > 0:
            plain.append(a.elapsed_time(b))
    plain_value = 1000.0 / statistics.mean(plain) if plain else None

    # e2e: the same batches through host buffers (pinned), copies inside the timing
    e2e = None
    if not args.no_e2e:
        wbytes = params.init_wit_rep * params.wit_len * params.d * 8
        h_w = [torch.empty(wbytes // 8, dtype=torch.int64, pin_memory=True) for _ in range(S)]
        h_p = [torch.empty(words, dtype=torch.int64, pin_memory=True) for _ in range(S)]
        for i in range(S):
            h_w[i].copy_(witnesses[i].view(-1))
        hw = [x.numpy() for x in h_w]
        hp = [x.numpy() for x in h_p]
        torch.cuda.synchronize()

        def ebatch(step, start_ev):
            for i in range(S):
                ext[i].wait_event(start_ev)
                slots[i].enqueue_host((rank << 40) + 5 * 10 ** 6 + step * S + i, hp[i], hw[i])
                e = torch.cuda.Event()
                e.record(ext[i])
                main.wait_event(e)

        ev = torch.cuda.Event()
        ev.record(main)
        ebatch(-1, ev)
        torch.cuda.synchronize()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(main)
        for s in range(args.steps):
            ev = torch.cuda.Event()
            ev.record(main)
            ebatch(s, ev)
        b.record(main)
        b.synchronize()
        e_ms = max_over_ranks(a.elapsed_time(b))
        e2e = {"value": S * args.steps * world / (e_ms / 1000.0), "unit": "proofs/s",
               "h2d_bytes_per_step": S * wbytes, "d2h_bytes_per_step": S * words * 8}

    ntt = ntt_bench(torch, api) if rank == 0 and not args.no_ntt else None
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(os.cpu_count() or 1)
    if rank == 0:
        peak, kind = measured_peaks()
        line = {
            "metric": "proofs/s", "value": value, "unit": "proofs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 mod q", "data": "synthetic",
            "config": {"workload": WORKLOAD if (args.preset == PRESET and not args.wit_log)
                       else "%s wit_len=2^%d" % (args.preset, params.wit_len.bit_length() - 1), "batch": S,
                       "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (512 MiB witness per proof)"},
            "p50_ms": statistics.median(lat), "p99_ms": float(np.percentile(lat, 99)),
            "plain": {"proofs_per_s": plain_value, "latency_ms": statistics.mean(plain) if plain else None},
            "batched_over_plain": (value / world) / plain_value if plain_value else None,
            "phase_ms_last_proof": timing,
            "gpu_launches": int(launches),
            "e2e": e2e,
            "ntt": ntt,
            "roofline": roofline_from(ntt, peak, kind),
            "cpu_baseline": cpu,
            "clocks": clk,
            "verified": check,
        }
        print(json.dumps(line), flush=True)
    for pr in slots:
        pr.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def ntt_bench(torch, api):
    """forward -> pointwise -> inverse, n=1024, the 62-bit prime,
    2^18 polynomials (2 GiB, larger than L2); forward/inverse timed alone."""
    from salsaa_b200 import params as P
    q, n, count = P.Q62, 1024, 1 << 18
    x = torch.randint(0, 1 << 62, (count, n), dtype=torch.int64, device="cuda") % q
    reps = 5
    res = {}
    for inv in (False, True):
        for _ in range(2):
            api.ntt(x, n, q, inverse=inv)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            api.ntt(x, n, q, inverse=inv)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b) / reps
        res["inverse" if inv else "forward"] = {"ms": ms, "GB/s": 16.0 * n * count / (ms * 1e6)}
    # protocol-shaped incomplete NTT: d=128 (two n=64 halves), 2^19 ring elements
    y = torch.randint(0, 1 << 50, (1 << 19, 128), dtype=torch.int64, device="cuda") % P.Q0
    out = torch.empty_like(y)
    api.ntt(y, 128, P.Q0, incomplete=True, out=out)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        api.ntt(y, 128, P.Q0, incomplete=True, out=out)
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b) / reps
    res["incomplete_d128"] = {"ms": ms, "GB/s": 16.0 * 128 * (1 << 19) / (ms * 1e6)}
    res["config"] = "n=1024 q=4546383823830515713 2^18 polys; incomplete d=128 q=1125899904679937 2^19 elements"
    return res


def roofline_from(ntt, peak, kind):
    if not ntt:
        return None
    f = ntt["forward"]
    return {"kernel": "ntt_kernel (forward, n=1024, 62-bit q)", "bound": "hbm", "achieved": f["GB/s"],
            "peak": peak, "unit": "GB/s", "frac": f["GB/s"] / peak, "peak_kind": kind,
            "traffic": None, "algorithmic_bytes_per_launch": 16 * 1024 * (1 << 18)}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
