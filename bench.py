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
host's cores: the C restatement under oracle/ (the Rust + Intel HEXL reference
cannot be built here).  Every timed step is one full A0 proof with all host
threads; the warm-up steps prove a small instance of the same shape
(WIT_LEN=2^13, 2 rounds) so the warm-up does not double the run.
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
WORKLOAD = ("A0 SNARK prove: d=128, q=1125899904679937, module_size=12, wit_len=2^19, 8 rounds, "
            "ternary witness")
# The statement every arm proves once and compares with the committed oracle
# digest (tests/golden/proof_digests.json): A0 with CRS seed 1 and seed 2.
DIGEST_CRS_SEED, DIGEST_SEED = 1, 2


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
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-only", action="store_true", help="run only the serving sweep and print its JSON")
    ap.add_argument("--serve-requests", type=int, default=96)
    ap.add_argument("--preset", default=PRESET, help="parameter set (profiling; the metric is quoted on A0)")
    ap.add_argument("--wit-log", type=int, default=0,
                    help="profiling: shrink WIT_LEN to 2^L (SNARK rounds L-11), keeping d, q and the rows")
    ap.add_argument("--no-dense", action="store_true",
                    help="skip the dense commitment and batched sumcheck microbenches")
    ap.add_argument("--dense-only", action="store_true",
                    help="profiling: run only the dense commitment and batched sumcheck microbenches")
    ap.add_argument("--ntt-only", action="store_true",
                    help="profiling: run only the NTT microbench and print its JSON")
    ap.add_argument("--ntt-log-coeffs", type=int, default=28,
                    help="log2 of the coefficients per NTT batch (28 = 2 GiB per buffer)")
    ap.add_argument("--no-tune-compare", action="store_true",
                    help="skip the runs with the untuned (default) kernel schedules")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch every proof's kernels directly (no CUDA-graph replay)")
    return ap.parse_args()


def measured_peaks(tensor=False):
    """HBM copy GB/s, or (tensor=True) the sustained dense bf16 TFLOP/s, which
    applies to a kernel timed inside a long step."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        if tensor:
            return float(d["bf16_tflops_sustained"]), "measured (cuBLAS bf16 dense, sustained)"
        return float(d["hbm_gbs"]), "measured (copy)"
    except Exception:
        return (1400.0, "fallback") if tensor else (6650.0, "fallback")


# ---------------------------------------------------------------------------
# CPU legs: the oracle port
# ---------------------------------------------------------------------------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def committed_digest(name=PRESET):
    """(crs_seed, seed, sha256) of the committed oracle proof of preset `name`."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "proof_digests.json")) as f:
            g = json.load(f)[name]
        return g["crs_seed"], g["seed"], g["sha256"]
    except Exception:
        return None


def cpu_prove_seconds(params, seed, threads):
    """Wall time of one oracle proof (with all `threads`) and its SHA-256."""
    import hashlib
    O = _oracle()
    t0 = time.perf_counter()
    rc, proof, _ = O.prove(params, DIGEST_CRS_SEED, seed, nthreads=threads)
    el = time.perf_counter() - t0
    if rc:
        raise RuntimeError("oracle prove failed: %d" % rc)
    return el, hashlib.sha256(proof.tobytes()).hexdigest()


def cpu_baseline(threads):
    """One full A0 proof on the host cores (the same statement as the digest)."""
    from salsaa_b200 import params as P
    el, _ = cpu_prove_seconds(P.preset(PRESET), DIGEST_SEED, threads)
    return {"value": 1.0 / el, "unit": "proofs/s", "cores": threads, "kind": "port",
            "sample": "one full A0 proof (wit_len=2^19, 8 rounds), %.2f s wall, oracle port with %d threads"
                      % (el, threads)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from salsaa_b200 import params as P
    threads = os.cpu_count() or 1
    small = P.make_params(128, P.Q0, 12, 1 << 13, 2, False)
    for w in range(args.warmup):
        cpu_prove_seconds(small, 100 + w, threads)
    full = P.preset(PRESET)
    times, first_sha = [], None
    for s in range(args.steps):
        el, h = cpu_prove_seconds(full, DIGEST_SEED + s, threads)
        times.append(el)
        if s == 0:
            first_sha = h
    tot = sum(times)
    value = args.steps / tot if tot else None
    dg = committed_digest()
    line = {
        "impl": "reference", "metric": "proofs/s", "value": value, "unit": "proofs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * tot / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64 mod q", "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch": 1, "parallelism": "cpu threads %d" % threads,
                   "warmup_workload": "A0 shape at wit_len=2^13, 2 rounds"},
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "port",
                         "sample": "each step one full A0 proof (wit_len=2^19, 8 rounds), oracle port, "
                                   "%d threads" % threads},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1000.0 * statistics.median(times) if times else None,
        "p99_ms": 1000.0 * float(np.percentile(times, 99)) if times else None,
        "proof_digest": {"crs_seed": DIGEST_CRS_SEED, "seed": DIGEST_SEED, "sha256": first_sha,
                         "equals_committed": (dg is not None and first_sha == dg[2]) if first_sha else None},
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
    from salsaa_b200 import api, lib, replicas

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
    # each slot replays a captured CUDA graph of its proof (the seed changed per
    # proof) unless --no-graph; the graphs are captured again after a schedule
    # change, so the default-vs-tuned comparison below compares like with like
    for pr in slots:
        pr.set_graph(not args.no_graph)
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
            slots[i].enqueue(seed=replicas.proof_seed(rank, step, i, S), d_proof=proofs[i], d_witness=witnesses[i])
            e = torch.cuda.Event(enable_timing=True)
            e.record(ext[i])
            main.wait_event(e)
            done.append(e)
        return done

    # untuned kernel schedules first (the library's defaults), for the
    # tuned-vs-default comparison; the timed region below runs the tuned table
    default_value = None
    if not args.no_tune_compare:
        set_schedules("default")
        for w in range(args.warmup):
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(main)
            batch(-100 - w, ev)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(main)
        nd = max(1, min(args.steps, 3))
        for sidx in range(nd):
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(main)
            batch(-200 - sidx, ev)
        b.record(main)
        b.synchronize()
        default_value = S * nd / (a.elapsed_time(b) / 1000.0)
    tuned_entries = set_schedules("tuned")
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
    # correctness spot checks after the timed region: the last batch's first
    # proof verifies on the CPU, and the committed oracle digest's statement
    # (witness sampled from its seed) gives the same proof bytes here
    check = digest_check = None
    if rank == 0 and args.steps > 0:
        try:
            O = _oracle()
            pb = api.to_host(proofs[0]).view(np.uint8)
            check = O.verify(params, 1, replicas.proof_seed(rank, args.steps - 1, 0, S), pb) == 0
        except Exception as e:  # the checker is optional here; tests own parity
            check = "not run: %s" % e
        dg = committed_digest()
        if dg and args.preset == PRESET and not args.wit_log:
            import hashlib
            slots[0].enqueue(seed=dg[1], d_proof=proofs[0])
            slots[0].sync()
            got = hashlib.sha256(api.to_host(proofs[0]).tobytes()).hexdigest()
            digest_check = {"crs_seed": dg[0], "seed": dg[1], "sha256": got, "equals_committed": got == dg[2]}

    # the same batches with direct launches, for the graph-replay comparison
    direct_value = None
    if not args.no_graph and args.steps > 0:
        for pr in slots:
            pr.set_graph(False)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(main)
        batch(-300, ev)  # warm
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(main)
        nd = max(1, min(args.steps, 3))
        for sidx in range(nd):
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(main)
            batch(-400 - sidx, ev)
        b.record(main)
        b.synchronize()
        direct_value = S * nd / (a.elapsed_time(b) / 1000.0)
    # per-phase times come from a proof launched directly (replays keep none)
    slots[0].set_graph(False)
    slots[0].enqueue(seed=replicas.proof_seed(rank, 0, 0, S), d_proof=proofs[0], d_witness=witnesses[0])
    slots[0].sync()
    timing = slots[0].timing()
    for pr in slots:
        pr.set_graph(not args.no_graph)


    # plain path: one proof at a time on one slot.  First with every kernel on
    # the slot's stream: the per-kernel trace runs there, where nothing else
    # shares the GPU, so each launch's events bracket that launch alone.
    def plain_run(overlap, trace):
        slots[0].set_overlap(overlap)
        out = []
        for i in range(args.plain_proofs):
            if trace and i == 1:
                torch.cuda.synchronize()
                lib().salsaa_trace_enable(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(ext[0])
            slots[0].enqueue(seed=10 ** 6 + i, d_proof=proofs[0], d_witness=witnesses[0])
            b.record(ext[0])
            b.synchronize()
            if i > 0:
                out.append(a.elapsed_time(b))
        torch.cuda.synchronize()
        return out

    serial = plain_run(False, True)
    traced = None
    if args.plain_proofs > 1:
        traced = {k: trace_read("ck_umma_kernel" + k) for k in ("", ":int8", ":mac")}
    lib().salsaa_trace_enable(0)
    # then latency mode: each round's projection and each commitment's
    # statement rows run on a second stream beside the main chain
    plain = plain_run(True, False) if args.plain_proofs else []
    plain_ms_graph = plain_ms_direct = None
    if plain and not args.no_graph:
        plain_ms_graph = statistics.mean(plain)
        slots[0].set_graph(False)
        plain_ms_direct = statistics.mean(plain_run(True, False))
        slots[0].set_graph(True)
    slots[0].set_overlap(False)
    plain_value = 1000.0 / statistics.mean(plain) if plain else None

    # e2e: the same batches through host buffers (pinned), copies inside the
    # timing.  The witness is short (ternary), so the headline path uploads it
    # as centred int8 coefficients (salsaa_prover_enqueue_host_i8, one byte
    # each); the same run through the u64 entry point is reported beside it.
    e2e = e2e_u64 = None
    if not args.no_e2e:
        n_coef = params.init_wit_rep * params.wit_len * params.d
        h_p = [torch.empty(words, dtype=torch.int64, pin_memory=True) for _ in range(S)]
        h_w = [torch.empty(n_coef, dtype=torch.int64, pin_memory=True) for _ in range(S)]
        h_w8 = [torch.empty(n_coef, dtype=torch.int8, pin_memory=True) for _ in range(S)]
        for i in range(S):
            wv = witnesses[i].view(-1)
            h_w[i].copy_(wv)
            h_w8[i].copy_(torch.where(wv > params.q // 2, wv - params.q, wv).to(torch.int8))
        hp = [x.numpy() for x in h_p]
        torch.cuda.synchronize()

        # Each slot's stream carries its proofs back to back (stream order is
        # the only dependency: a slot's next host->device copy follows its
        # previous proof), so the copies of one slot overlap the proofs of
        # the others, as in a serving loop; the timed region brackets all
        # steps' copies, proofs and result reads.
        def e2e_run(call, hw, wbytes):
            def ebatch(step):
                for i in range(S):
                    call(slots[i], (rank << 40) + 5 * 10 ** 6 + step * S + i, hp[i], hw[i])

            ebatch(-1)
            torch.cuda.synchronize()
            barrier()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(main)
            for i in range(S):
                ext[i].wait_event(a)
            for s in range(args.steps):
                ebatch(s)
            for i in range(S):
                e = torch.cuda.Event()
                e.record(ext[i])
                main.wait_event(e)
            b.record(main)
            b.synchronize()
            e_ms = max_over_ranks(a.elapsed_time(b))
            return {"value": S * args.steps * world / (e_ms / 1000.0), "unit": "proofs/s",
                    "h2d_bytes_per_step": S * wbytes, "d2h_bytes_per_step": S * words * 8}

        e2e = e2e_run(lambda pr, sd, p_, w: pr.enqueue_host_i8(sd, p_, w), [x.numpy() for x in h_w8], n_coef)
        e2e["witness"] = "int8 centred coefficients (salsaa_prover_enqueue_host_i8)"
        last_i8 = [x.copy() for x in hp]
        e2e_u64 = e2e_run(lambda pr, sd, p_, w: pr.enqueue_host(sd, p_, w), [x.numpy() for x in h_w], 8 * n_coef)
        e2e_u64["witness"] = "u64 canonical coefficients (salsaa_prover_enqueue_host)"
        # both runs prove the same seeds and witnesses: the last proofs agree
        e2e["same_proofs_as_u64"] = all(np.array_equal(x, y) for x, y in zip(last_i8, hp))

    for pr in slots:
        pr.close()
    slots = []
    del witnesses, proofs
    torch.cuda.empty_cache()
    ntt = ntt_default = None
    if rank == 0 and not args.no_ntt:
        if not args.no_tune_compare:
            set_schedules("default")
            ntt_default = ntt_bench(torch, api, forward_only=True)
            set_schedules("tuned")
        ntt = ntt_bench(torch, api)
    dense = dense_bench(torch, api) if rank == 0 and not args.no_dense else None
    scb = sumcheck_batch_bench(torch, api) if rank == 0 and not args.no_dense else None
    multi = batched_launch_bench(torch, api) if rank == 0 and not args.no_dense else None
    serving = serving_bench(torch, api, args.serve_requests, rank) if not args.no_serve else None
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
            "plain": {"proofs_per_s": plain_value, "latency_ms": statistics.mean(plain) if plain else None,
                      "overlap": True,
                      "latency_ms_single_stream": statistics.mean(serial) if serial else None},
            "batched_over_plain": (value / world) / plain_value if plain_value else None,
            "phase_ms_last_proof": timing,
            "gpu_launches": int(launches),
            "e2e": e2e,
            "e2e_u64_witness": e2e_u64,
            "ntt": ntt,
            "commit_dense": dense,
            "sumcheck_batch": scb,
            "batched_launches": multi,
            "serving": serving,
            "roofline": roofline_ck(traced, sum(serial) if serial else None,
                                    args.preset == "A0" and not args.wit_log),
            "ntt_roofline": roofline_ntt(ntt, peak, kind),
            "graphs": {"value_graph_replay": None if args.no_graph else value / world,
                       "value_direct_launches": (value / world) if args.no_graph else direct_value,
                       "graph_over_direct": (value / world) / direct_value if direct_value else None,
                       "plain_ms_graph_replay": plain_ms_graph,
                       "plain_ms_direct_launches": plain_ms_direct,
                       "note": "each slot captures its proof's launch sequence once and replays it with "
                               "the seed changed (salsaa_prover_set_graph); same proof bytes"},
            "tuning": {"table_entries": tuned_entries,
                       "value_default_schedules": default_value,
                       "value_tuned_schedules": value / world,
                       "tuned_over_default": (value / world) / default_value if default_value else None,
                       "ntt_default": ntt_default},
            "cpu_baseline": cpu,
            "clocks": clk,
            "verified": check,
            "proof_digest": digest_check,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


SERVE_SLOTS = {"A0": 4, "A1": 4, "A2": 4, "F0": 4, "F1": 2, "F2": 1}
SERVE_BUDGET = 140 << 30
SERVE_MAX_INFLIGHT = 4  # proofs running at once in the served path
SERVE_LOADS = (0.5, 1.0, 1.5, 2.0, 3.0)  # offered load as multiples of the plain path's capacity
SERVE_SLO_MS = (100.0, 200.0, 400.0, 800.0)  # p99 targets for the equal-p99 comparison


def serving_bench(torch, api, nreq, rank):
    """Serving stream: Poisson arrivals of A0/A1/A2 SNARK proves and F0/F1/F2
    folding steps (size classes 0/1/2 drawn 40/30/30, SNARK or folding 50/50),
    each with its own seed and a witness sampled on the GPU.  The same request
    stream (names, seeds, arrival pattern) is offered at several loads, as
    multiples of the plain path's capacity (1 / mean service time), through
    the plain path (one proof at a time, in arrival order) and through the
    continuous-batching server; latency counts from arrival.  At each p99
    target the throughput each path sustains within it is compared (the
    highest completed rate over the loads whose p99 meets the target)."""
    import time as _t
    rng = np.random.default_rng(4242 + rank)
    cls = rng.choice(3, size=nreq, p=[0.4, 0.3, 0.3])
    kind = rng.integers(0, 2, size=nreq)
    names = [("A%d" if k == 0 else "F%d") % c for c, k in zip(cls, kind)]
    gaps = rng.exponential(1.0, size=nreq)  # unit-rate gaps, scaled per load
    seeds = [10 ** 7 + rank * 10 ** 5 + i for i in range(nreq)]
    params = {nm: api.params_preset(nm) for nm in SERVE_SLOTS}

    def stats(lat, span):
        return {"proofs_per_s": nreq / span, "p50_ms": 1e3 * float(np.median(lat)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99))}

    # plain path: one slot per set, proofs strictly one after another
    ctxs = {nm: api.Context(params[nm], crs_seed=3) for nm in SERVE_SLOTS}
    provers = {nm: api.Prover(ctxs[nm]) for nm in SERVE_SLOTS}
    bufs = {nm: torch.empty(ctxs[nm].proof_bytes // 8, dtype=torch.int64, device="cuda") for nm in SERVE_SLOTS}
    service = {}
    for nm in SERVE_SLOTS:  # warm-up and per-set service time
        provers[nm].enqueue(1, bufs[nm])
        provers[nm].sync()
        t0 = _t.perf_counter()
        provers[nm].enqueue(2, bufs[nm])
        provers[nm].sync()
        service[nm] = _t.perf_counter() - t0
    capacity = 1.0 / float(np.mean([service[nm] for nm in names]))
    plain_runs = {}
    for load in SERVE_LOADS:
        arrivals = np.cumsum(gaps) / (load * capacity)
        lat = []
        t0 = _t.perf_counter()
        for i, nm in enumerate(names):
            while _t.perf_counter() - t0 < arrivals[i]:
                pass
            provers[nm].enqueue(seeds[i], bufs[nm])
            provers[nm].sync()
            lat.append(_t.perf_counter() - t0 - arrivals[i])
        plain_runs[load] = stats(lat, _t.perf_counter() - t0)
    for nm in SERVE_SLOTS:
        provers[nm].close()
        ctxs[nm].close()
    del bufs
    torch.cuda.empty_cache()
    # served path
    srv = api.Server(SERVE_BUDGET)
    srv.limit(SERVE_MAX_INFLIGHT)
    sets = {nm: srv.register(params[nm], crs_seed=3, slots=SERVE_SLOTS[nm]) for nm in SERVE_SLOTS}
    outs = [torch.empty(api.proof_size(params[nm]) // 8, dtype=torch.int64, device="cuda") for nm in names]
    warm = [srv.submit(sets[nm], 1, torch.empty(api.proof_size(params[nm]) // 8, dtype=torch.int64,
                                                device="cuda")) for nm in SERVE_SLOTS]
    while srv.progress() > 0:
        pass
    for t in warm:
        srv.poll(t)
    served_runs = {}
    for load in SERVE_LOADS:
        arrivals = np.cumsum(gaps) / (load * capacity)
        tickets = [None] * nreq
        done = {}
        nsub = 0
        t0 = _t.perf_counter()
        while len(done) < nreq:
            now = _t.perf_counter() - t0
            while nsub < nreq and arrivals[nsub] <= now:
                tickets[nsub] = srv.submit(sets[names[nsub]], seeds[nsub], outs[nsub])
                nsub += 1
            srv.progress()
            for i in range(nsub):
                if i not in done:
                    r = srv.poll(tickets[i])
                    if r is not None:
                        done[i] = _t.perf_counter() - t0 - arrivals[i]
        served_runs[load] = stats([done[i] for i in range(nreq)], _t.perf_counter() - t0)
    srv.close()
    sweep = [{"offered_x_plain_capacity": load, "offered_per_s": load * capacity, "plain": plain_runs[load],
              "served": served_runs[load]} for load in SERVE_LOADS]

    def best_within(runs, slo):
        ok = [r["proofs_per_s"] for r in runs.values() if r["p99_ms"] <= slo]
        return max(ok) if ok else None

    equal_p99 = []
    for slo in SERVE_SLO_MS:
        a, b = best_within(plain_runs, slo), best_within(served_runs, slo)
        equal_p99.append({"p99_target_ms": slo, "plain_proofs_per_s": a, "served_proofs_per_s": b,
                          "served_over_plain": (b / a) if (a and b) else None})
    return {"requests": nreq, "mix": {nm: names.count(nm) for nm in SERVE_SLOTS}, "slots": SERVE_SLOTS,
            "max_in_flight": SERVE_MAX_INFLIGHT, "plain_capacity_per_s": capacity,
            "service_ms_alone": {nm: 1e3 * v for nm, v in service.items()}, "sweep": sweep,
            "at_equal_p99": equal_p99,
            "served_over_plain_peak": max(r["proofs_per_s"] for r in served_runs.values())
            / max(r["proofs_per_s"] for r in plain_runs.values())}


def dense_bench(torch, api):
    """Ajtai commitment microbench: C = A W over R_q (d = 128, the 50-bit
    prime), A n x m uniform, W m x r base-b digits uniform in [-b/2, b/2)
    (seeded), for n in {8, 16}, m in {2^12, 2^16}, r in {1, 8, 32},
    b in {2, 16}.  A is prepared once (its byte image for the tensor cores);
    each timed call includes W's NTT, the product and C's inverse NTT, and
    W's NTT is also timed alone."""
    from salsaa_b200 import params as P
    q, d, reps = P.Q0, 128, 5
    gen = torch.Generator(device="cuda")
    gen.manual_seed(77)
    out = []
    for n in (8, 16):
        for mlog in (12, 16):
            m = 1 << mlog
            A = torch.randint(0, 1 << 62, (n, m, d), dtype=torch.int64, device="cuda", generator=gen) % q
            key = api.DenseKey(A, q)
            del A
            for r in (1, 8, 32):
                ws = api.dev_empty((r, m, d))
                C = api.dev_empty((n, r, d))
                for b in (2, 16):
                    W = torch.randint(-(b // 2), b // 2, (r, m, d), dtype=torch.int64, device="cuda",
                                      generator=gen) % q
                    key.commit(W, out=C, w_slot=ws)
                    a = torch.cuda.Event(enable_timing=True)
                    e = torch.cuda.Event(enable_timing=True)
                    a.record()
                    for _ in range(reps):
                        key.commit(W, out=C, w_slot=ws)
                    e.record()
                    e.synchronize()
                    ms = a.elapsed_time(e) / reps
                    a.record()
                    for _ in range(reps):
                        api.ntt(W, d, q, incomplete=True, out=ws)
                    e.record()
                    e.synchronize()
                    ntt_ms = a.elapsed_time(e) / reps
                    nbytes = 8 * d * (n * m + m * r + n * r)
                    out.append({"n": n, "m": m, "r": r, "b": b, "ms": ms, "w_ntt_ms": ntt_ms,
                                "GB/s": nbytes / (ms * 1e6),
                                "Gmulmod/s": n * m * r * 2 * d / (ms * 1e6)})
                    del W
                del ws, C
            key.close()
            torch.cuda.empty_cache()
    return {"q": q, "d": d, "bytes": "8 d (n m + m r + n r) per call", "mulmods": "n m r 2d per call",
            "runs": out}


def sumcheck_batch_bench(torch, api):
    """Norm-check sumcheck microbench: 64 instances with lengths log-uniform in
    2^16..2^22 (seeded), ternary coefficients, the 50-bit prime; all rounds of
    all instances in one batched call, against the same instances one call
    each.  Bytes: 8 per coefficient (each vector is read once)."""
    from salsaa_b200 import params as P
    q, reps = P.Q0, 5
    rng = np.random.default_rng(2024)
    logs = np.sort(rng.integers(16, 23, size=64))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    vecs = [(torch.randint(-1, 2, (1 << int(k),), dtype=torch.int64, device="cuda", generator=gen) % q)
            for k in logs]
    total = sum(v.numel() for v in vecs)

    def timed(fn):
        fn()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        e.record()
        e.synchronize()
        return a.elapsed_time(e) / reps

    batched = timed(lambda: api.sum_check_batch(vecs, q, 1, 0))
    single = timed(lambda: [api.sum_check_batch([v], q, 1, 0) for v in vecs])
    res = {"instances": len(vecs), "lengths_log2": [int(k) for k in logs], "coefficients": int(total),
           "batched_ms": batched, "one_call_each_ms": single, "batched_GB/s": 8.0 * total / (batched * 1e6),
           "speedup": single / batched}
    del vecs
    torch.cuda.empty_cache()
    return res


def batched_launch_bench(torch, api):
    """Uneven instances in one launch against one launch each: 64 batches of
    incomplete d = 128 transforms (log-uniform 2^8..2^14 ring elements, the
    50-bit prime, salsaa_ntt_multi) and the A0 commitment-key rows over 8
    witnesses of uneven shapes (salsaa_commit_multi).  CUDA events around 5
    repetitions of each form on the current stream."""
    from salsaa_b200 import params as P
    reps = 5
    rng = np.random.default_rng(99)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(9)

    def timed(fn):
        fn()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        e.record()
        e.synchronize()
        return a.elapsed_time(e) / reps

    q, d = P.Q0, 128
    logs = np.sort(rng.integers(8, 15, size=64))
    xs = [torch.randint(0, 1 << 50, (1 << int(k), d), dtype=torch.int64, device="cuda", generator=gen) % q
          for k in logs]
    outs = [torch.empty_like(x) for x in xs]
    one = timed(lambda: api.ntt_multi(xs, d, q, incomplete=True, outs=outs))
    each = timed(lambda: [api.ntt(x, d, q, incomplete=True, out=o) for x, o in zip(xs, outs)])
    coeffs = sum(x.numel() for x in xs)
    ntt = {"instances": len(xs), "elements_log2": [int(k) for k in logs], "one_launch_ms": one,
           "one_launch_each_ms": each, "speedup": each / one, "one_launch_GB/s": 16.0 * coeffs / (one * 1e6)}
    del xs, outs
    params = api.params_preset("A0")
    ctx = api.Context(params, crs_seed=1)
    shapes = [(1, 1 << 19), (3, 1 << 16), (9, 1 << 12), (2, 1 << 18), (1, 1 << 14), (5, 1 << 15), (4, 1 << 11),
              (2, 1 << 17)]
    ws = [torch.randint(-1, 2, (r, w, params.d), dtype=torch.int64, device="cuda", generator=gen) % params.q
          for r, w in shapes]
    one = timed(lambda: ctx.parallel_dot_series_matrix_multi(ws))
    each = timed(lambda: [ctx.parallel_dot_series_matrix(w) for w in ws])
    commit = {"witnesses": [list(sh) for sh in shapes], "one_launch_ms": one, "one_launch_each_ms": each,
              "speedup": each / one}
    del ws
    ctx.close()
    torch.cuda.empty_cache()
    return {"ntt": ntt, "commit": commit}


def trace_read(name):
    """(launches, total device ms, total algorithmic work) of a traced kernel."""
    import ctypes
    from salsaa_b200 import lib
    ms, work, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_uint64()
    rc = lib().salsaa_trace_read(name.encode(), ctypes.byref(ms), ctypes.byref(work), ctypes.byref(n))
    if rc:
        raise RuntimeError("trace_read failed for %s" % name)
    return {"launches": int(n.value), "ms": ms.value, "work": work.value}


def timed_launches(torch, fn, name, reps):
    """Run fn reps times with the trace on; per-launch device time of `name`."""
    from salsaa_b200 import lib
    torch.cuda.synchronize()
    lib().salsaa_trace_enable(1)
    for _ in range(reps):
        fn()
    torch.cuda.synchronize()
    t = trace_read(name)
    lib().salsaa_trace_enable(0)
    return t


def flush_l2(torch, buf):
    buf.add_(1)


def set_schedules(mode):
    """'default': the library's untuned kernel schedules; 'tuned': reload the
    tuner's table (tune_table.txt beside the library).  Returns the number of
    table entries loaded (tuned), or None."""
    from salsaa_b200 import lib
    if mode == "default":
        lib().salsaa_tune_reset()
        return None
    n = lib().salsaa_tune_load(None)
    return n if n >= 0 else 0


def ntt_bench(torch, api, log_coeffs=28, forward_only=False):
    """Batched negacyclic NTT microbench (62-bit prime, coefficients uniform in
    [0, q)): forward, inverse and the fused forward-product-inverse for
    n in {64, 128, 256, 1024}, plus the protocol-shaped incomplete transform
    (d = 128, 50-bit prime).  Every batch is >= 512 MiB (larger than L2) and
    each launch is timed by CUDA events on its own stream."""
    from salsaa_b200 import params as P
    q = P.Q62
    res = {}
    reps = 5
    for n in (64, 128, 256, 1024):
        count = min(1 << 20, (1 << log_coeffs) // n)
        x = torch.randint(0, 1 << 62, (count, n), dtype=torch.int64, device="cuda") % q
        y = torch.randint(0, 1 << 62, (count, n), dtype=torch.int64, device="cuda") % q
        r = torch.empty_like(x)
        row = {"polys": count}
        for inv in ((False,) if forward_only else (False, True)):
            api.ntt(x, n, q, inverse=inv)
            t = timed_launches(torch, lambda: api.ntt(x, n, q, inverse=inv), "ntt_kernel", reps)
            ms = t["ms"] / t["launches"]
            row["inverse" if inv else "forward"] = {"ms": ms, "GB/s": t["work"] / t["launches"] / (ms * 1e6)}
        if forward_only:
            res["n%d" % n] = row
            del x, y, r
            continue
        api.poly_mul(x, y, n, q, out=r)
        t = timed_launches(torch, lambda: api.poly_mul(x, y, n, q, out=r), "ntt_mul_kernel", reps)
        ms = t["ms"] / t["launches"]
        row["fused_product"] = {"ms": ms, "GB/s": t["work"] / t["launches"] / (ms * 1e6)}
        res["n%d" % n] = row
        del x, y, r
    ne = min(1 << 19, (1 << log_coeffs) // 128)
    z = torch.randint(0, 1 << 50, (ne, 128), dtype=torch.int64, device="cuda") % P.Q0
    out = torch.empty_like(z)
    api.ntt(z, 128, P.Q0, incomplete=True, out=out)
    t = timed_launches(torch, lambda: api.ntt(z, 128, P.Q0, incomplete=True, out=out), "ntt_kernel", reps)
    ms = t["ms"] / t["launches"]
    res["incomplete_d128"] = {"ms": ms, "GB/s": t["work"] / t["launches"] / (ms * 1e6), "elements": ne}
    res["q"] = q
    res["bytes"] = "forward/inverse 16 B per coefficient, fused product 24 B per coefficient (read a, b; write r)"
    return res


def roofline_ntt(ntt, peak, kind):
    """The NTT microbench against the measured copy bandwidth: the protocol's
    incomplete d = 128 transform (50-bit prime) as the headline, every size's
    forward and inverse fraction beside it."""
    if not ntt:
        return None
    f = ntt["incomplete_d128"]
    per = {}
    for k, row in ntt.items():
        if isinstance(row, dict):
            for direction in ("forward", "inverse"):
                if direction in row:
                    per["%s_%s" % (k, direction)] = row[direction]["GB/s"] / peak
            if "GB/s" in row:
                per[k] = row["GB/s"] / peak
    return {"kernel": "register NTT, incomplete d=128 (two 64-point transforms), q=1125899904679937, "
                      "2^19 ring elements", "bound": "hbm",
            "achieved": f["GB/s"], "peak": peak, "unit": "GB/s", "frac": f["GB/s"] / peak, "peak_kind": kind,
            "algorithmic_bytes_per_launch": 16 * 128 * f["elements"], "frac_per_size": per}


# DRAM bytes (read + write) of ck_umma_kernel per launch, mean over the eight
# launches of one A0 proof (dram__bytes_read.sum + dram__bytes_write.sum), from
# one ncu capture made by CK_TRAFFIC_CMD; ncu cannot run inside this process,
# so the figure is carried with the command that measured it.
CK_TRAFFIC_A0 = 653.8e6
CK_TRAFFIC_CMD = ("ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum "
                  "--clock-control none -k regex:ck_umma -c 8 --csv python bench.py --steps 1 --warmup 1 "
                  "--slots 1 --plain-proofs 1 --no-e2e --no-ntt --no-serve --no-cpu-baseline --no-dense")


def roofline_ck(traced, elapsed_ms, a0):
    """Dominant kernel of the prove: the commitment-key rows on the tensor
    cores.  Its bound is HBM: the algorithmic bytes are the slot-form witness
    read once and the accumulators written once, against the measured copy
    bandwidth.  Beside it, the tensor-pipe fraction (int8 operations the
    tensor cores execute, against NVIDIA's dense int8 rate, which is twice
    the dense bf16 rate; the bf16 rate is measured here) and the exact mod-q
    multiply-accumulates per second.  elapsed_ms: summed device time of the
    traced plain proofs; a0: the default A0 workload, the one the traffic
    capture covers."""
    if not traced or not traced[""]["launches"]:
        return None
    t, t8, tm = traced[""], traced[":int8"], traced[":mac"]
    per_ms = t["ms"] / t["launches"]
    nbytes = t["work"] / t["launches"]
    achieved = nbytes / (per_ms * 1e6)
    hbm, hbm_kind = measured_peaks()
    bf16, bf16_kind = measured_peaks(tensor=True)
    int8_peak = 2.0 * bf16
    ops = t8["work"] / t8["launches"]
    tops = ops / (per_ms * 1e-3) / 1e12
    macs = tm["work"] / tm["launches"]
    return {"kernel": "ck_umma_kernel (exact int8 limb-split commitment, tcgen05.mma kind::i8, TMEM)",
            "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_kind": hbm_kind + " copy bandwidth",
            "traffic": CK_TRAFFIC_A0 if a0 else None,
            "traffic_note": ("DRAM read+write bytes per launch, mean over the 8 launches of one A0 proof, "
                             "from one ncu capture (command in traffic_cmd)") if a0
            else "no capture for this workload",
            "traffic_cmd": CK_TRAFFIC_CMD if a0 else None,
            "algorithmic_bytes_per_launch": nbytes,
            "launches": t["launches"], "ms_per_launch": per_ms,
            "tensor": {"achieved": tops, "unit": "TOP/s int8", "peak": int8_peak,
                       "peak_kind": "2 x %s bf16 (dense int8 = 2 x dense bf16 on B200)" % bf16_kind,
                       "frac": tops / int8_peak, "int8_ops_per_launch": ops},
            "mac_per_s": macs / (per_ms * 1e-3), "mac_per_launch": macs,
            "share_of_plain_prove": t["ms"] / elapsed_ms if elapsed_ms else None,
            "measured_on": "plain path (one proof at a time, one stream), CUDA events around each launch"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.dense_only:
        import torch
        from salsaa_b200 import api
        print(json.dumps({"commit_dense": dense_bench(torch, api),
                          "sumcheck_batch": sumcheck_batch_bench(torch, api),
                          "batched_launches": batched_launch_bench(torch, api)}), flush=True)
        return 0
    if args.serve_only:
        import torch
        from salsaa_b200 import api
        print(json.dumps({"serving": serving_bench(torch, api, args.serve_requests, 0)}), flush=True)
        return 0
    if args.ntt_only:
        import torch
        from salsaa_b200 import api
        print(json.dumps({"ntt": ntt_bench(torch, api, args.ntt_log_coeffs)}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
