#!/usr/bin/env python
"""Benchmark of the hera read-alignment hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config2] [--chunk 1000000] [--write-bam 1]

A step is one pass of the hot path over one chunk of read pairs (default
1M pairs of the transcriptome-scale workload).  `value` is device-timed
throughput with the chunk already resident in HBM; `e2e` is the same metric
through the public C ABI with host buffers (H2D of the reads and D2H of the
Candidate records inside the timed region).  Under torchrun each rank runs a
replica of the index on its own GPU over its own chunks (weak scaling, no
data-path collective); the reported time is the max over ranks.

Besides the headline, the default run checks the last timed step's records
against the oracle on a sample (`bit_exact`, outside the timed region) and
adds legs: the drop-in Candidate call, the -w tail's BAM records, FASTQ
chunk text -> records, add_class and the EM, config 3 (mixed lengths,
batched vs plain, single-end reads), config 4 (high divergence, mate-rescue
roofline) and the config-5 serving loop with each sample's EM checked bit for
bit against the oracle's.

`--impl reference` times the reference program's own CPU implementation of
the same path (oracle/_ref/libhera_ref.so: check_in_transcriptome +
intersect2 per pair) on all host cores, on steps of the same size.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "aligned read pairs/s"
STAGES = ("seed_ms", "position_ms", "build_ms", "dp_ms", "resolve_ms", "rescue_ms", "pack_ms")
COUNTS = ("probes", "seed_hits", "sw_cells", "ssw_cells")
UNIT = "pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2")
    ap.add_argument("--chunk", type=int, default=1_000_000)
    ap.add_argument("--distinct", type=int, default=3, help="distinct chunks generated per rank")
    ap.add_argument("--write-bam", type=int, default=1, help="hera WRITE_BAM (1 = no -w)")
    ap.add_argument("--cpu-sample", type=int, default=200_000,
                    help="pairs per slice of the in-run CPU baseline (the reference arm times whole "
                         "--chunk steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--paths", default="plain,batched", help="execution forms to time (batched last)")
    ap.add_argument("--lanes", type=int, default=0, help="concurrent sub-batches (0 = library default)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop leg")
    ap.add_argument("--no-fastq", action="store_true", help="skip the FASTQ-chunk leg")
    ap.add_argument("--fastq-only", action="store_true",
                    help="time only the FASTQ-chunk leg (one JSON line with the leg's numbers)")
    ap.add_argument("--bam-only", action="store_true",
                    help="time only the BAM-record leg (the -w tail's records on the device; one JSON line)")
    ap.add_argument("--pin-tuning", default="", help="BUILD_BLOCKS_PER_SM,RESCUE_WARPS_PER_BLOCK: "
                    "fixed launch shapes instead of the autotuner (reproducible profiles)")
    ap.add_argument("--serve-scale", type=float, default=1.0,
                    help="sample sizes of the serving leg as a fraction of 0.5M-8M pairs")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle checks of the timed records")
    ap.add_argument("--parity-pairs", type=int, default=20_000,
                    help="pairs of the last timed step checked against the oracle")
    ap.add_argument("--no-config-legs", action="store_true", help="skip the config-3 and config-4 legs")
    ap.add_argument("--no-bam", action="store_true", help="skip the BAM-record leg")
    ap.add_argument("--no-hera-quant", action="store_true",
                    help="skip the leg that times hera quant against hera quant with the library inside")
    ap.add_argument("--quant-pairs", type=int, default=2_000_000, help="read pairs of the hera quant leg")
    ap.add_argument("--leg-pairs", type=int, default=500_000, help="pairs per step of the config-3/4 legs")
    ap.add_argument("--leg-steps", type=int, default=5, help="timed steps of the config-3/4 legs")
    return ap.parse_args()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


_T0 = [time.perf_counter()]


def phase(name: str) -> None:
    """Log the wall seconds since the previous phase mark (stderr)."""
    t = time.perf_counter()
    log(f"[phase] {name}: {t - _T0[0]:.1f}s")
    _T0[0] = t


class ClockSampler:
    """nvidia-smi SM clock / throttle samples while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_chunks(name, ann, tx, chunk, distinct, seed0):
    from hera_b200 import workloads
    out = []
    for k in range(distinct):
        t = time.time()
        r1, r2 = workloads.pairs(name, ann, tx, chunk, seed0 + k)
        out.append((r1, r2))
        log(f"chunk {k}: {chunk} pairs in {time.time() - t:.1f}s")
    return out


def cpu_baseline(ix, chunks, sample: int, write_bam: int, target_s: float = 10.0):
    """The reference's own code on all host cores over a bounded sample."""
    import oracle
    if not oracle.reference_available():
        return None
    ref = oracle.Reference(ix)
    threads = os.cpu_count() or 1
    done, elapsed = 0, 0.0
    k = 0
    while elapsed < target_s and k < 4 * len(chunks):
        r1, r2 = chunks[k % len(chunks)]
        lo = (k // len(chunks)) * sample
        if lo + sample > r1.n:
            break
        idx = np.arange(lo, lo + sample)
        a, b = r1.subset(idx), r2.subset(idx)
        t = time.perf_counter()
        ref.align_pairs_mt(a, b, write_bam, threads)
        elapsed += time.perf_counter() - t
        done += sample
        k += 1
    return {"value": done / elapsed, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{done} pairs of the workload in slices of {sample} "
                      f"(reference check_in_transcriptome+intersect2, {threads} threads, "
                      f"{elapsed:.1f} s)"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from hera_b200 import workloads
    import oracle
    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhera_ref.so not built"}))
        return
    t = time.time()
    ann, tx, ix = workloads.build(args.workload, device=None if args.workload != "config2" else _maybe_cuda())
    log(f"index {time.time() - t:.1f}s")
    ref = oracle.Reference(ix)
    threads = os.cpu_count() or 1
    sample = args.chunk   # the same pairs per step as the device arm
    chunks = make_chunks(args.workload, ann, tx, sample, min(args.distinct, args.steps + args.warmup), 1000)
    times = []
    for s in range(args.warmup + args.steps):
        r1, r2 = chunks[s % len(chunks)]
        a, b = r1.copy(), r2.copy()
        t0 = time.perf_counter()
        ref.align_pairs_mt(a, b, args.write_bam, threads)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = sample * len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": f"{args.workload}: {workloads.DESCRIPTION[args.workload]}",
                   "pairs_per_step": sample, "write_bam": args.write_bam,
                   "parallelism": f"replicas x{args.gpus}"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{sample} pairs per step, reference code on {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _maybe_cuda():
    try:
        import torch
        return "cuda" if torch.cuda.is_available() else None
    except Exception:
        return None


def to_device(chunks):
    """Device-resident copies of the chunks (mates interleaved), the layout
    of the device-resident entry point."""
    import torch
    from hera_b200 import workloads
    dev, max_len = [], 0
    for r1, r2 in chunks:
        seq, off, lens = workloads.interleave(r1, r2)
        max_len = max(max_len, int(lens.max()))
        dev.append((torch.from_numpy(seq).cuda(), torch.from_numpy(off).cuda(), torch.from_numpy(lens).cuda()))
    torch.cuda.synchronize()
    return dev, max_len


def measure(ix, dev, max_len, chunk, path, args, local, world, steps=None, warmup=None):
    """`steps` device-resident calls of `chunk` pairs on one context, timed
    with CUDA events on the context's stream (max over ranks).  Returns the
    context (its last call's records still on the device) and the numbers."""
    import torch
    import torch.distributed as dist
    from hera_b200 import api, shard
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    # the plain form is one pass per chunk: one lane
    lanes = 1 if path == "plain" else args.lanes
    ctx = api.Context(ix, device=local, path=path, lanes=lanes, max_batch=chunk if path == "plain" else 0)
    if args.pin_tuning:
        ctx.set_tuning(*[int(x) for x in args.pin_tuning.split(",")])
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step(i):
        s, o, ln = dev[i % len(dev)]
        ctx.align_pairs_device(s.data_ptr(), o.data_ptr(), ln.data_ptr(), chunk, max_len, args.write_bam,
                               ctx.stream)

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    stage = {k: 0.0 for k in STAGES}
    counts = {k: 0 for k in COUNTS}
    launches, jobs, calls, lookups, wide = 0, 0, 0, 0, 0
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    torch.cuda.synchronize()
    evs[0].record(stream)
    for i in range(steps):
        step(i)
        evs[i + 1].record(stream)
        tm = ctx.timing()
        launches += int(tm["launches"])
        jobs += int(tm["dp_jobs"])
        calls += int(tm["dp_calls"])
        lookups += int(tm["lookups"])
        wide += int(tm["wide_items"])
        for k in stage:
            stage[k] += float(tm[k])
        for k in counts:
            counts[k] += int(tm[k])
    torch.cuda.synchronize()
    clocks = sampler.stop()
    per = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
    ms = evs[0].elapsed_time(evs[-1])
    ms = shard.max_over_ranks(ms, device="cuda")
    if world > 1:
        dist.barrier()
    out = {"path": path, "ms": ms, "per_step_ms": per, "stage": stage, "launches": launches,
           "dp_jobs": jobs, "dp_calls": calls, "lookups": lookups, "counts": counts, "wide_items": wide,
           "clocks": clocks, "last": (steps - 1) % len(dev), "steps": steps,
           "value": chunk * steps * world / (ms / 1000.0)}
    return ctx, out


def bit_exact(ctx, orc, chunk_pairs, n_pairs, k, write_bam):
    """The records of the context's last device-resident call against the
    oracle (the reference's algorithm restated in C), on the first k pairs
    of that call's chunk: checked outside the timed region."""
    r1, r2 = chunk_pairs
    k = min(k, r1.n)
    res = ctx.fetch(2 * n_pairs)
    idx = np.arange(k)
    want = orc.align_pairs(r1.subset(idx), r2.subset(idx), write_bam)
    got = res.canonical(0, 2 * k)
    exp = want.canonical()
    bad = sum(1 for a, b in zip(got, exp) if a != b)
    return {"bit_exact": bad == 0 and len(got) == len(exp), "pairs_checked": k, "records_differing": bad}


def leg_summary(m):
    per = sorted(m["per_step_ms"])
    return {"value": m["value"], "ms_per_step": m["ms"] / m["steps"], "gpu_launches": m["launches"],
            "wide_pass_pairs": m["wide_items"],
            "stage_ms_per_step": {k: round(v / m["steps"], 4) for k, v in m["stage"].items()},
            "p50_ms": per[len(per) // 2]}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    import torch
    import torch.distributed as dist
    from hera_b200 import api, workloads
    if not torch.cuda.is_available():
        print(json.dumps({"metric": METRIC, "error": "no CUDA device"}))
        sys.exit(1)
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    from hera_b200 import shard
    t = time.time()
    ann, tx, ix = workloads.build(args.workload, device=f"cuda:{local}")
    log(f"[{rank}] index: {ix.n_trans} transcripts, {int(ix.length.sum())} bases, {ix.buckets.shape[0]} k-mers, "
        f"{ix.n_pos} occurrences in {time.time() - t:.1f}s")
    if args.fastq_only:
        r1, r2 = workloads.pairs(args.workload, ann, tx, args.chunk, seed=100 + 1000 * rank)
        print(json.dumps({"fastq": fastq_bench(args, ix, (r1, r2), local),
                          "config": {"workload": args.workload, "pairs_per_step": args.chunk}}), flush=True)
        return
    if args.bam_only:
        r1, r2 = workloads.pairs(args.workload, ann, tx, args.chunk, seed=100 + 1000 * rank)
        print(json.dumps({"bam": bam_bench(args, ix, ann, (r1, r2), local),
                          "config": {"workload": args.workload, "pairs_per_step": args.chunk}}), flush=True)
        return
    chunks = make_chunks(args.workload, ann, tx, args.chunk, args.distinct, 100 + 1000 * rank)
    dev, max_len = to_device(chunks)
    solo = rank == 0 and world == 1
    phase("index and chunks")
    orc = None
    if solo and not args.no_parity:
        try:
            import oracle   # the checker: outside every timed region
            orc = oracle.Oracle(ix)
        except Exception as e:
            log(f"oracle unavailable: {e}")

    phase("oracle")
    paths = [p for p in args.paths.split(",") if p]
    plain = parity_plain = None
    if "plain" in paths:
        ctx_p, plain = measure(ix, dev, max_len, args.chunk, "plain", args, local, world)
        if orc is not None:
            parity_plain = bit_exact(ctx_p, orc, chunks[plain["last"]], args.chunk, args.parity_pairs,
                                     args.write_bam)
        ctx_p.close()
    main_path = "batched" if "batched" in paths else "plain"
    ctx, batched = measure(ix, dev, max_len, args.chunk, main_path, args, local, world)
    value = batched["value"]
    parity = None
    if orc is not None:
        parity = bit_exact(ctx, orc, chunks[batched["last"]], args.chunk, args.parity_pairs, args.write_bam)
        log(f"parity ({main_path}, last step, first {parity['pairs_checked']} pairs): {parity}")

    phase("plain and batched steps, parity")
    # end to end through the public C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        r1, r2 = chunks[0]
        out = ctx.align_pairs(r1, r2, args.write_bam)   # warm staging and result buffers
        caps = [int(x * 1.3) + 4096 for x in (out.c.list_used, out.c.op_used, out.c.miss_used)]
        outs = [api.Result(2 * args.chunk, *caps) for _ in range(2)]
        # inputs and results in page-locked host memory, registered once
        pinned = [a for c in chunks for rs in c for a in (rs.seq,)] + outs[0].arrays() + outs[1].arrays()
        for a in pinned:
            api.host_register(a)
        # both lane groups warm
        tk = [ctx.submit_pairs(r1, r2, args.write_bam, outs[0]), ctx.submit_pairs(r1, r2, args.write_bam, outs[1])]
        for t in tk:
            ctx.complete_pairs(t)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

        def bytes_of(res, r1, r2):
            return (int(r1.len.sum() + r2.len.sum()) + 12 * 2 * r1.n,
                    res.recs.nbytes + 8 * int(res.c.list_used) + 4 * int(res.c.op_used) + int(res.c.miss_used))

        # pipelined: step i+1's reads go to the device while step i computes
        t0 = time.perf_counter()
        h2d = d2h = 0
        pending = []
        for i in range(args.steps):
            r1, r2 = chunks[i % len(chunks)]
            pending.append((ctx.submit_pairs(r1, r2, args.write_bam, outs[i % 2]), r1, r2))
            if len(pending) == 2 or i == args.steps - 1:
                while pending and (len(pending) == 2 or i == args.steps - 1):
                    t, a, b = pending.pop(0)
                    hb, db = bytes_of(ctx.complete_pairs(t), a, b)
                    h2d += hb
                    d2h += db
        torch.cuda.synchronize()
        e2e_s = shard.max_over_ranks(time.perf_counter() - t0, device="cuda")
        # one call at a time, for comparison
        t0 = time.perf_counter()
        for i in range(args.steps):
            r1, r2 = chunks[i % len(chunks)]
            ctx.align_pairs(r1, r2, args.write_bam, out=outs[0])
        torch.cuda.synchronize()
        sync_s = shard.max_over_ranks(time.perf_counter() - t0, device="cuda")
        e2e = {"value": args.chunk * args.steps * world / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
               "api": "hera_gpu_align_pairs_submit / _complete, two calls in flight",
               "one_call_at_a_time": args.chunk * args.steps * world / sync_s,
               "host_memory": "reads and result pools page-locked (registered once before timing)"}
        for a in pinned:
            api.host_unregister(a)
        if solo:
            try:
                e2e["dropin"] = dropin_bench(ctx, chunks[0], args)
            except Exception as e:
                e2e["dropin"] = {"error": str(e)}

    phase("end to end and drop-in")
    cpu = None
    if solo and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(ix, chunks, args.cpu_sample, args.write_bam)
        except Exception as e:   # the checker is optional on a box without it
            log(f"cpu baseline failed: {e}")

    phase("cpu baseline")
    st = batched["stage"]
    tuning = ctx.tuning() if main_path == "batched" else None
    ctx.close()
    ktm, classes = kernel_pass(ix, dev[0], max_len, args, local, rank, world) if main_path == "batched" \
        else (None, None)
    dpx = api.dpx_peak(local)
    pair_bytes = int(chunks[0][0].len.sum() + chunks[0][1].len.sum())
    roof, roof_seed, roof_rescue = roofline(ktm, dpx, args.chunk, pair_bytes, max_len)
    phase("kernel pass and classes")
    del dev

    legs = {}
    if solo:
        for name, fn in (("bam", lambda: None if args.no_bam else bam_bench(args, ix, ann, chunks[0], local)),
                         ("fastq", lambda: None if args.no_fastq else fastq_bench(args, ix, chunks[0], local)),
                         ("hera_quant", lambda: None if args.no_hera_quant else hera_quant_bench(args, local))):
            try:
                legs[name] = fn()
            except Exception as e:
                log(f"{name} leg failed: {e}")
                legs[name] = {"error": str(e)}
            phase(f"{name} leg")
        del orc, chunks
        ix1 = None
        phase("config-1 workloads start")
        if not args.no_config_legs or not args.no_serve:
            try:
                ann1, tx1, ix1 = workloads.build("config1", device=f"cuda:{local}")
            except Exception as e:   # the line is still printed, the legs carry the error
                log(f"config1 index failed: {e}")
                for name in ("config3", "config4", "serving"):
                    legs[name] = {"error": f"config1 index: {e}"}
        if ix1 is not None:
            orc1 = None
            if not args.no_parity:
                try:
                    import oracle
                    orc1 = oracle.Oracle(ix1)
                except Exception as e:
                    log(f"oracle unavailable: {e}")
            for name, fn in (("config3", lambda: None if args.no_config_legs else
                              config3_leg(args, ann1, tx1, ix1, orc1, local)),
                             ("config4", lambda: None if args.no_config_legs else
                              config4_leg(args, ann1, tx1, ix1, orc1, local, dpx)),
                             ("serving", lambda: None if args.no_serve else
                              serve_bench(args, ann1, tx1, ix1, orc1, local))):
                try:
                    legs[name] = fn()
                except Exception as e:
                    log(f"{name} leg failed: {e}")
                    legs[name] = {"error": str(e)}
                phase(f"{name} leg")

    if rank == 0:
        per = sorted(batched["per_step_ms"])
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": batched["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {workloads.DESCRIPTION[args.workload]}",
                       "pairs_per_step": args.chunk, "write_bam": args.write_bam,
                       "parallelism": f"replicas x{world}"},
            "bit_exact": None if parity is None else parity["bit_exact"],
            "parity": {main_path: parity, "plain": parity_plain},
            "plain": None if plain is None else {
                "value": plain["value"], "ms_per_step": plain["ms"] / args.steps,
                "batched_over_plain": value / plain["value"], "gpu_launches": plain["launches"]},
            "roofline": _short_roof(roof), "roofline_seed": _short_roof(roof_seed),
            "roofline_rescue": _short_roof(roof_rescue),
            "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": batched["launches"], "clocks": batched["clocks"],
            "setup": {"path": ("batched (build / length-binned DP jobs / replay rounds)"
                               if main_path == "batched" else "plain (thread per call / pair)"),
                      "l2": "inputs larger than L2 (reads 200 MB/step, index in HBM)"},
            "latency_ms": {"p50": per[len(per) // 2], "p99": per[min(len(per) - 1, int(0.99 * len(per)))]},
            "wide_pass_pairs": batched["wide_items"],
            "kernel_ms_per_step": None if ktm is None else {
                k: round(float(ktm[k]), 4) for k in ("seed_kernel_ms", "build_ms", "dp_kernel_ms",
                                                     "rescue_kernel_ms", "resolve_ms", "pack_ms")},
            "stage_ms_per_step": {k: round(v / args.steps, 4) for k, v in st.items()},
            "plain_stage_ms_per_step": None if plain is None else
            {k: round(v / args.steps, 4) for k, v in plain["stage"].items()},
            "dp_jobs_per_step": batched["dp_jobs"] // args.steps,
            "dp_calls_per_step": batched["dp_calls"] // args.steps,
            "roofline_detail": {"dp": roof, "seed": roof_seed, "rescue": roof_rescue},
            "tuning": tuning, "classes": classes, **legs,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _short_roof(r):
    if r is None:
        return None
    return {k: r.get(k) for k in ("bound", "achieved", "peak", "unit", "frac", "traffic", "kernel")}


def kernel_pass(ix, dv, max_len, args, local, rank, world):
    """One step on a single-lane context, so each kernel's CUDA-event
    duration is its own (the timed run overlaps several lanes)."""
    import torch
    from hera_b200 import api
    kctx = api.Context(ix, device=local, path="batched", lanes=1)
    if args.pin_tuning:
        kctx.set_tuning(*[int(x) for x in args.pin_tuning.split(",")])
    s, o, ln = dv
    for _ in range(2):
        kctx.align_pairs_device(s.data_ptr(), o.data_ptr(), ln.data_ptr(), args.chunk, max_len,
                                args.write_bam, kctx.stream)
    torch.cuda.synchronize()
    tm = kctx.timing()
    cls = None
    if rank == 0 and world == 1:
        try:
            cls = classes_leg(kctx, args.chunk, ix.length)
        except Exception as e:
            log(f"classes leg failed: {e}")
            cls = {"error": str(e)}
    kctx.close()
    return tm, cls


def dropin_bench(ctx, chunk, args, k: int = 200_000):
    """hera's own call shape: reads as struct read_inf, results as
    heap-allocated Candidate pairs for the unchanged host tail
    (hera_gpu_align_pairs), on the first k pairs of a chunk; the Candidates
    are freed afterwards as hera's destroy_candidate would."""
    r1, r2 = chunk
    idx = np.arange(min(k, r1.n))
    a, b = r1.subset(idx), r2.subset(idx)
    ctx.align_pairs_dropin(a, b, args.write_bam)   # warm
    ms = ctx.align_pairs_dropin(a, b, args.write_bam)
    return {"value": a.n / (ms / 1e3), "unit": UNIT, "pairs": a.n, "call_ms": round(ms, 3),
            "path": "hera_gpu_align_pairs: read_inf in, malloc'd Candidates out (freed after the clock)"}


def config3_leg(args, ann, tx, ix, orc, local):
    """Config 3's batching comparison: mixed 50/75/100/150 bp reads (1:1:2:1)
    on the config-1 index, half in pairs and half single-end.  Pairs: the
    batched form (length-binned persistent build, autotuned launch shapes)
    against the plain one-launch-per-chunk form, device-resident, records
    checked against the oracle on a sample.  Single-end reads: through the
    flat C ABI (host buffers; align_single_read's two get_position calls)."""
    from hera_b200 import api, workloads
    n = args.leg_pairs
    chunks = make_chunks("config3", ann, tx, n, 2, 3000)
    dev, max_len = to_device(chunks)
    out = {"workload": f"config3: {workloads.DESCRIPTION['config3']}", "pairs_per_step": n}
    for path in ("plain", "batched"):
        ctx, m = measure(ix, dev, max_len, n, path, args, local, 1, steps=args.leg_steps)
        out[path] = leg_summary(m)
        if orc is not None:
            out[path].update(bit_exact(ctx, orc, chunks[m["last"]], n, args.parity_pairs // 4, args.write_bam))
        ctx.close()
    out["batched_over_plain"] = out["batched"]["value"] / out["plain"]["value"]
    rs = workloads.singles("config3", tx, n, 3100)
    ctx = api.Context(ix, device=local)
    try:
        got = ctx.align_single(rs, args.write_bam)   # warm
        t0 = time.perf_counter()
        for _ in range(args.leg_steps):
            got = ctx.align_single(rs, args.write_bam)
        wall = time.perf_counter() - t0
        single = {"reads_per_s": n * args.leg_steps / wall, "reads_per_step": n,
                  "path": "hera_gpu_align_single_flat (host buffers)"}
        if orc is not None:
            k = min(args.parity_pairs // 4, n)
            sub = rs.subset(np.arange(k))
            single["bit_exact"] = got.canonical(0, k) == orc.align_single(sub, args.write_bam).canonical()
            single["reads_checked"] = k
        out["single"] = single
    finally:
        ctx.close()
    return out


def config4_leg(args, ann, tx, ix, orc, local, dpx):
    """Config 4, high divergence: 2x150 bp, 3% substitutions, 0.5% 1-8 bp
    indels, 5% pairs from mutated unannotated loci (they fall through
    unmapped and take the mate rescue); batched and plain, device-resident,
    with the rescue kernel's roofline from a single-lane pass."""
    import torch
    from hera_b200 import api, workloads
    n = args.leg_pairs
    chunks = make_chunks("config4", ann, tx, n, 1, 4000)
    dev, max_len = to_device(chunks)
    out = {"workload": f"config4: {workloads.DESCRIPTION['config4']}", "pairs_per_step": n}
    for path in ("plain", "batched"):
        ctx, m = measure(ix, dev, max_len, n, path, args, local, 1, steps=args.leg_steps)
        out[path] = leg_summary(m)
        if orc is not None:
            out[path].update(bit_exact(ctx, orc, chunks[m["last"]], n, args.parity_pairs // 4, args.write_bam))
        ctx.close()
    out["batched_over_plain"] = out["batched"]["value"] / out["plain"]["value"]
    kctx = api.Context(ix, device=local, path="batched", lanes=1)
    s, o, ln = dev[0]
    for _ in range(2):
        kctx.align_pairs_device(s.data_ptr(), o.data_ptr(), ln.data_ptr(), n, max_len, args.write_bam, kctx.stream)
    torch.cuda.synchronize()
    tm = kctx.timing()
    kctx.close()
    roof, _, rescue = roofline(tm, dpx, n, int(chunks[0][0].len.sum() + chunks[0][1].len.sum()), max_len)
    out["roofline"] = _short_roof(roof)
    out["roofline_rescue"] = _short_roof(rescue)
    out["kernel_ms_per_step"] = {k: round(float(tm[k]), 4) for k in ("seed_kernel_ms", "build_ms", "dp_kernel_ms",
                                                                     "rescue_kernel_ms", "resolve_ms", "pack_ms")}
    out["ssw_cells"] = int(tm["ssw_cells"])
    return out


def classes_leg(kctx, pairs: int, length) -> dict:
    """hera's add_class on the device (hera_gpu_classes_add_last) over the
    device-resident records of the step kctx just ran: kernel time with a
    fresh table (every class inserted) and with the same records again
    (every class found).  Bytes counted: each pair's two 52-byte records
    plus 4 B per list entry the tail hashes.  Then hera's EM on the device
    over the first table, against the EM restated in C (one host thread)
    on the same table: time and bit-for-bit equality."""
    from hera_b200 import api
    out = {}
    cls = api.Classes(kctx, max_classes=1 << 22, max_list=1 << 26)
    try:
        cls.add_last(kctx)
        first = cls.timing()
        t = cls.fetch()
        g, o, rounds, em_ms = cls.em(kctx)
        cls.add_last(kctx)
        again = cls.timing()
    finally:
        cls.close()
    em = {"device_ms": round(em_ms, 3), "rounds": rounds, "transcripts": len(length)}
    try:
        import oracle   # the CPU baseline of this leg: the EM restated in C
        t0 = time.perf_counter()
        g0, o0, k0 = oracle.em_port(t, length)
        cpu_s = time.perf_counter() - t0
        em.update({"cpu_port_ms": round(cpu_s * 1e3, 3), "cpu_cores": 1,
                   "bit_exact": bool(k0 == rounds and np.array_equal(g.view(np.uint64), g0.view(np.uint64))
                                     and np.array_equal(o.view(np.uint64), o0.view(np.uint64)))})
    except Exception as e:
        em["cpu_error"] = str(e)
    out["em"] = em
    hashed = int(t.ns.sum()) + int(t.tx_count.sum())
    algo = 104 * pairs + 4 * hashed
    peak = _hbm_peak()
    for tag, tm in (("insert", first), ("lookup", again)):
        ms = tm["kernel_ms"]
        gbs = algo / (ms / 1e3) / 1e9 if ms > 0 else None
        out[tag] = {"kernel_ms": round(ms, 4), "pairs_per_s": pairs / (ms / 1e3) if ms > 0 else None,
                    "launches": tm["launches"], "achieved_gbs": gbs,
                    "frac_of_hbm": None if gbs is None else gbs / peak[0]}
    out.update({"classes": t.n_classes, "paired": t.paired, "single_transcript_reads": int(t.tx_count.sum()),
                "algorithmic_bytes": algo, "hbm_peak": peak[1]})
    return out


def _read_names(n: int, mate: int) -> np.ndarray:
    """Rows "r<i, 7+ digits>/<mate>" NUL-padded to 16 bytes (more when i
    needs over 10 digits), built with digit arithmetic."""
    w = max(7, len(str(max(n - 1, 0))))
    a = np.zeros((n, max(16, w + 4)), np.uint8)
    a[:, 0] = ord("r")
    i = np.arange(n, dtype=np.int64)
    for k in range(w):
        a[:, 1 + k] = 48 + (i // 10 ** (w - 1 - k)) % 10
    a[:, 1 + w] = ord("/")
    a[:, 2 + w] = 48 + mate
    return a


def _bgzf_inflate(z: bytes) -> bytes:
    """The data of back-to-back BGZF blocks, block by block (each block's
    size from its BC extra field; each member's CRC-32 and length checked).
    Linear in the stream: Python's multi-member gzip.decompress copies the
    rest of the stream once per member."""
    import struct
    import zlib
    parts, o = [], 0
    while o < len(z):
        if z[o:o + 4] != b"\x1f\x8b\x08\x04" or z[o + 12:o + 16] != b"BC\x02\x00":
            raise ValueError(f"not a BGZF block at byte {o}")
        bsize = struct.unpack_from("<H", z, o + 16)[0] + 1
        d = zlib.decompress(z[o + 18:o + bsize - 8], wbits=-15)
        crc, isize = struct.unpack_from("<II", z, o + bsize - 8)
        if zlib.crc32(d) != crc or len(d) != isize:
            raise ValueError(f"bad CRC or size in the BGZF block at byte {o}")
        parts.append(d)
        o += bsize
    return b"".join(parts)


def _write_fastq_fast(reads, path: str, mate: int) -> None:
    """FASTQ of a read set ('?' qualities, names read<i>/<mate>), built as
    one buffer: hera's parser sees the same text synth.write_fastq writes."""
    n = reads.n
    parts = []
    step = 200_000
    for lo in range(0, n, step):
        hi = min(n, lo + step)
        buf = []
        for i in range(lo, hi):
            s = reads.seq[reads.off[i]:reads.off[i] + reads.len[i]].tobytes()
            buf.append(b"@read%d/%d\n%s\n+\n%s\n" % (i, mate, s, b"?" * len(s)))
        parts.append(b"".join(buf))
    with open(path, "wb") as f:
        for b in parts:
            f.write(b)


def hera_quant_bench(args, local):
    """hera's own program end to end on the same index directory and FASTQ
    files: the unmodified reference (oracle/_ref/hera) and the same program
    with the library in its paired-end worker loop (oracle/_ref/hera_gpu:
    hera_gpu_align_pairs per chunk, hera's own align_pair_read tail,
    add_class, EM and output), both with -t = all host cores.  Each runs on
    N/4 and on N pairs: the whole-program wall time of each run, and from
    their difference the per-pair rate with the fixed costs (index load,
    the library's context and index upload, EM, output) taken out."""
    import oracle
    from hera_b200 import index, workloads
    hera, hera_gpu = oracle.REFERENCE_BIN, os.path.join(oracle.REF_DIR, "hera_gpu")
    if not (os.path.exists(hera) and os.path.exists(hera_gpu)):
        return {"unavailable": "oracle/_ref/hera or hera_gpu not built (make -C oracle ref dropin)"}
    import tempfile
    cores = os.cpu_count() or 1
    wl = "config2s"
    ann, tx, ix = workloads.build(wl)
    n = args.quant_pairs
    n_small = n // 4
    r1, r2 = workloads.pairs("config2", ann, tx, n, seed=71)
    with tempfile.TemporaryDirectory(dir=os.environ.get("TMPDIR")) as d:
        index.write_index_dir(ann, ix, os.path.join(d, "idx"))
        fq = {}
        for tag, k in (("small", n_small), ("full", n)):
            idx = np.arange(k)
            a, b = os.path.join(d, f"{tag}_1.fq"), os.path.join(d, f"{tag}_2.fq")
            _write_fastq_fast(r1.subset(idx) if k < n else r1, a, 1)
            _write_fastq_fast(r2.subset(idx) if k < n else r2, b, 2)
            fq[tag] = (a, b)
        out = {}
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
        for name, binary in (("hera", hera), ("hera_gpu", hera_gpu)):
            walls = {}
            for tag in ("small", "full"):
                a, b = fq[tag]
                o = os.path.join(d, f"{name}_{tag}")
                t = time.perf_counter()
                p = subprocess.run([binary, "quant", "-i", os.path.join(d, "idx"), "-1", a, "-2", b, "-o", o,
                                    "-t", str(cores)], capture_output=True, text=True, timeout=1200, env=env)
                walls[tag] = time.perf_counter() - t
                if p.returncode != 0:
                    return {"error": f"{name} exited {p.returncode}: {p.stderr[-300:]}"}
            rate = (n - n_small) / max(1e-9, walls["full"] - walls["small"])
            out[name] = {"wall_s": round(walls["full"], 3), "wall_s_quarter": round(walls["small"], 3),
                         "pairs_per_s": n / walls["full"], "pairs_per_s_incremental": rate,
                         "fixed_s": round(walls["small"] - n_small / rate, 3)}
            if name == "hera_gpu":   # the worker's own account of its threads' time (full run)
                out[name]["worker"] = [ln for ln in p.stderr.splitlines() if ln.startswith("hera_gpu:")]
        same = {f: open(os.path.join(d, "hera_full", f), "rb").read()
                == open(os.path.join(d, "hera_gpu_full", f), "rb").read()
                for f in ("abundance.tsv", "abundance.gene.tsv")}
    out.update({"workload": f"{wl} index, {n_small} and {n} config-2-model pairs (2x100 bp)", "threads": cores,
                "speedup_wall": out["hera"]["wall_s"] / out["hera_gpu"]["wall_s"],
                "speedup_per_pair": out["hera_gpu"]["pairs_per_s_incremental"] / out["hera"]["pairs_per_s_incremental"],
                "files_identical": same,
                "note": "with -t > 1 hera's own add_class order follows thread timing, so the files can "
                        "differ in the last bits (-t 1 identity: tests/test_hera_dropin.py)"})
    return out


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        peaks = {}
    return float(peaks.get("hbm_gbs", 6650.0)), "measured" if "hbm_gbs" in peaks else "fallback"


def bam_bench(args, ix, ann, chunk, local, cpu_sample: int = 50_000):
    """The -w tail's BAM records for one chunk of pairs: aligned with
    traceback through the flat C ABI, then written by hera_gpu_bam_pairs
    (host buffers in and out; the reported device time covers the input
    copies and both writer passes).  The oracle's restatement on one host
    thread over a sample is the CPU baseline of this leg."""
    from hera_b200 import api, synth
    r1, r2 = chunk
    n = r1.n
    q1 = np.full(r1.seq.shape[0] + 1, ord("?"), np.uint8)
    q2 = np.full(r2.seq.shape[0] + 1, ord("?"), np.uint8)
    names = [_read_names(n, mate) for mate in (1, 2)]
    gm = synth.gene_map(ann)
    phase("bam: names and gene map")
    ctx = api.Context(ix, device=local)
    phase("bam: context")
    try:
        res = ctx.align_pairs(r1, r2, 0)
        tmb = ctx.timing()
        phase(f"bam: traceback alignment ({int(tmb.get('wide_items', 0))} pairs through the wide pass)")
        w = api.BamWriter(ctx, gm)
        try:
            w.pairs(res, r1, r2, q1, q2, names[0], names[1])   # warm
            t0 = time.perf_counter()
            out, off, ms = w.pairs(res, r1, r2, q1, q2, names[0], names[1])
            wall = time.perf_counter() - t0
        finally:
            w.close()
        phase("bam: device records")
        # the records' BGZF framing on the device (hera_gpu_bgzf, host buffers)
        bgz = None
        try:
            ctx.bgzf(out[:1 << 20])   # warm
            t0 = time.perf_counter()
            z, zms = ctx.bgzf(out)
            zwall = time.perf_counter() - t0
            bgz = {"device_ms": round(zms, 3), "call_ms": round(zwall * 1e3, 3),
                   "gbs_device": len(out) / (zms / 1e3) / 1e9, "pairs_per_s_call": n / zwall,
                   "ratio": round(len(out) / max(1, len(z)), 2),
                   "decompresses_to_records": bool(_bgzf_inflate(z.tobytes()) == out.tobytes())}
        except Exception as e:
            bgz = {"error": str(e)}
    finally:
        ctx.close()
    leg = {"pairs": n, "record_bytes": int(off[-1]), "device_ms": round(ms, 3),
           "pairs_per_s_device": n / (ms / 1e3), "pairs_per_s_call": n / wall,
           "record_gbs_device": int(off[-1]) / (ms / 1e3) / 1e9, "bgzf_device": bgz}
    # BGZF framing stays with the caller: what it costs on the host cores.
    # The records in 64 KiB blocks, each deflated at zlib's default level
    # (hera's COMPRESS_LEVEL -1) as its own raw stream, on 1 thread and on
    # all threads (zlib releases the GIL).
    try:
        import zlib
        from concurrent.futures import ThreadPoolExecutor
        data = memoryview(out)
        B = 0xff00

        def deflate(lo):
            c = zlib.compressobj(-1, zlib.DEFLATED, -15)
            return len(c.compress(data[lo:lo + B])) + len(c.flush())

        starts = list(range(0, len(data), B))
        one = starts[:max(1, min(len(starts), (64 << 20) // B))]
        t0 = time.perf_counter()
        for lo in one:
            deflate(lo)
        t1 = time.perf_counter() - t0
        cores = os.cpu_count() or 1
        with ThreadPoolExecutor(cores) as ex:
            t0 = time.perf_counter()
            zbytes = sum(ex.map(deflate, starts))
            tn = time.perf_counter() - t0
        mb1 = len(one) * B / t1 / 1e6
        leg["host_bgzf"] = {"mb_per_s_1_thread": round(mb1, 1), "mb_per_s_all": round(len(data) / tn / 1e6, 1),
                            "threads": cores, "pairs_per_s_all": n / tn, "ratio": round(len(data) / zbytes, 2),
                            "note": "deflate of the records (hera's bam_write on the host cores)"}
    except Exception as e:
        leg["host_bgzf"] = {"error": str(e)}
    try:
        import oracle   # the CPU baseline of this leg: the writer restated in C
        k = min(cpu_sample, n)
        idx = np.arange(k)
        a1, a2 = r1.subset(idx), r2.subset(idx)
        phase("bam: bgzf (device and host)")
        orc = oracle.Oracle(ix)
        ores = orc.align_pairs(a1, a2, 0)
        phase("bam: oracle traceback alignment of the sample")
        c1 = np.full(a1.seq.shape[0] + 1, ord("?"), np.uint8)
        c2 = np.full(a2.seq.shape[0] + 1, ord("?"), np.uint8)
        t0 = time.perf_counter()
        ob, ooff = oracle.bam_pairs(gm, ores, a1, a2, [c1, c2], [names[0][:k].copy(), names[1][:k].copy()])
        cpu_s = time.perf_counter() - t0
        leg["cpu_port"] = {"pairs_per_s": k / cpu_s, "cores": 1, "sample": f"first {k} pairs",
                           "bytes_equal": bool(ob.tobytes() == out[:int(off[k])].tobytes())}
    except Exception as e:
        leg["cpu_port"] = {"error": str(e)}
    return leg


def fastq_bench(args, ix, chunk, local):
    """The step's pairs as two FASTQ chunk buffers (hera's reader input):
    the device parse against HBM bandwidth (the parse kernels' CUDA-event
    time, chunk copies excluded), and chunk text -> records end to end
    through hera_gpu_align_fastq_pairs (chunk copies included)."""
    import torch
    from hera_b200 import api, synth
    r1, r2 = chunk
    left = np.frombuffer(synth.fastq_bytes(r1, 1), np.uint8).copy()
    right = np.frombuffer(synth.fastq_bytes(r2, 2), np.uint8).copy()
    for a in (left, right):
        api.host_register(a)
    ctx = api.Context(ix, device=local)
    try:
        for _ in range(args.warmup):
            recs = ctx.parse_fastq_pairs(left, right)
        parse_ms, h2d_ms = [], []
        for _ in range(args.steps):
            recs = ctx.parse_fastq_pairs(left, right)
            st = ctx.fastq_stats()
            parse_ms.append(st["parse_ms"])
            h2d_ms.append(st["h2d_ms"])
        assert recs.shape[0] == 2 * r1.n
        text = int(left.size + right.size)
        reads = int(recs.shape[0])
        # algorithmic bytes: every chunk byte read once, one 32-byte record
        # written per read
        alg = text + 32 * reads
        ms = float(np.median(parse_ms))
        peak, src = _hbm_peak()
        achieved = alg / (ms / 1000.0) / 1e9
        parse = {"kernels": "k_fq_count, k_fq_scan, k_fq_lines, k_fq_ends, k_fq_recs",
                 "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                 "frac": achieved / peak, "peak_source": src, "bytes_per_step": alg,
                 "chunk_bytes": text, "reads": reads, "parse_ms": ms, "h2d_ms": float(np.median(h2d_ms))}
        res, recs = ctx.align_fastq_pairs(left, right, args.write_bam)   # warm
        res, recs = ctx.align_fastq_pairs(left, right, args.write_bam, out=res)
        pinned = res.arrays() + [ctx._fq_recs]
        for a in pinned:
            api.host_register(a)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d2h = 0
        for _ in range(args.steps):
            res, recs = ctx.align_fastq_pairs(left, right, args.write_bam, out=res)
            d2h += (res.recs.nbytes + 8 * int(res.c.list_used) + 4 * int(res.c.op_used)
                    + int(res.c.miss_used) + recs.nbytes)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        for a in pinned:
            api.host_unregister(a)
        e2e = {"value": r1.n * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": text,
               "d2h_bytes_per_step": d2h // args.steps,
               "path": "FASTQ chunk text -> device parse -> align -> records (hera_gpu_align_fastq_pairs)"}
        return {"parse": parse, "e2e": e2e}
    finally:
        ctx.close()
        for a in (left, right):
            api.host_unregister(a)


def serve_bench(args, ann, tx, ix, orc, local):
    """The serving loop on the config-5 shape: the config-1 index resident,
    64 samples of log-uniform 0.5M-8M pairs (times --serve-scale), read
    lengths 75-150 bp, arriving as 131072-pair (256k-read) chunks by a
    Poisson process at 1.5x the plain path's measured capacity.  During the
    Poisson run each waited chunk's records go into its sample's class table
    on the device (hera's add_class, in the sample's chunk order); after it,
    every sample's EM on the device is checked bit for bit against the EM
    the oracle computes over the class table of the oracle's own records
    for the same chunks."""
    import types
    from hera_b200 import api, synth
    CH = 131072
    pool = []   # one chunk per read length; chunks of a sample reuse its pool chunk
    for k, L in enumerate((75, 100, 125, 150)):
        pool.append(synth.simulate_pairs(tx, CH, seed=500 + k, read_len=L, frag_mu=max(250.0, 2.5 * L),
                                         frag_sd=25.0, sub_rate=0.005, indel_rate=0.0001))
    # the plain path's capacity, host buffers in and out like the server's
    pctx = api.Context(ix, device=local, path="plain", lanes=1, max_batch=CH)   # one launch per chunk
    for r1, r2 in pool:   # buffers at every read length before the clock
        pctx.align_pairs(r1, r2)
    t = time.perf_counter()
    for r1, r2 in pool:
        pctx.align_pairs(r1, r2)
    plain = len(pool) * CH / (time.perf_counter() - t)
    pctx.close()
    rate = 1.5 * plain
    rng = np.random.default_rng(55)
    sizes = np.exp(rng.uniform(np.log(5e5), np.log(8e6), 64)) * args.serve_scale
    sizes = np.maximum(sizes.astype(np.int64), 1)
    rlen = rng.integers(0, 4, 64)
    plan = []   # (sample, n) in arrival order: samples interleaved
    left = sizes.copy()
    while left.sum() > 0:
        for s in rng.permutation(64):
            if left[s] > 0:
                n = int(min(CH, left[s]))
                plan.append((int(s), n))
                left[s] -= n
    gaps = rng.exponential(1.0, len(plan))
    gaps *= np.array([n for _, n in plan]) / rate   # mean gap = chunk size / rate

    def chunk_of(s, n):
        r1, r2 = pool[rlen[s]]
        if n < CH:
            r1 = types.SimpleNamespace(n=n, seq=r1.seq, off=r1.off[:n], len=r1.len[:n])
            r2 = types.SimpleNamespace(n=n, seq=r2.seq, off=r2.off[:n], len=r2.len[:n])
        return r1, r2

    ctx = api.Context(ix, device=local)
    # the pool chunks outlive every wait: submit borrows them (no copy)
    srv = api.Server(ctx, batch_pairs=CH, write_bam=args.write_bam, max_samples=64, borrow_reads=True)
    # warm the slots (buffers at the longest reads, autotuner) before the clock
    warm = [srv.submit(0, *pool[3]) for _ in range(2 * srv.stats()["slots"])]
    keep = None   # one host result reused by the waiter
    for tk in warm:
        keep = srv.wait(tk, out=keep)[0]
    # capacity: the whole plan submitted at once
    t = time.perf_counter()
    sat = [srv.submit(s, *chunk_of(s, n)) for s, n in plan]
    t_sub = time.perf_counter() - t
    for tk in sat:
        srv.wait(tk, out=keep)
    capacity = float(sizes.sum()) / (time.perf_counter() - t)
    log(f"serving capacity run: submit {t_sub:.2f}s, total {float(sizes.sum()) / capacity:.2f}s, "
        f"{srv.stats()}")
    # per-sample class tables on the device, filled as chunks are waited for
    tables = [api.Classes(ctx, max_classes=1 << 14, max_list=1 << 18) for _ in range(64)]
    tickets, infos = [], []
    lock = threading.Lock()
    done = threading.Event()

    def feed():
        t0 = time.perf_counter()
        due = 0.0
        for (s, n), g in zip(plan, gaps):
            due += g
            d = due - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            tk = srv.submit(s, *chunk_of(s, n))
            with lock:
                tickets.append((s, tk))
        done.set()

    add_ms = []
    th = threading.Thread(target=feed)
    t0 = time.perf_counter()
    th.start()
    k = 0
    try:
        while True:
            with lock:
                item = tickets[k] if k < len(tickets) else None
            if item is None:
                if done.is_set() and k >= len(tickets):
                    break
                time.sleep(0.0005)
                continue
            s, tk = item
            res, info = srv.wait(tk, out=keep)
            ta = time.perf_counter()
            tables[s].add_result(res)
            add_ms.append((time.perf_counter() - ta) * 1e3)
            infos.append(info)
            k += 1
        th.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        lat = np.array([i["done_ms"] - i["submit_ms"] for i in infos])
        wt = np.array([i["admit_ms"] - i["submit_ms"] for i in infos])
        span_s = (max(i["done_ms"] for i in infos) - min(i["submit_ms"] for i in infos)) / 1e3
        out = {"workload": "config5 shape: config1 index, 64 samples of log-uniform 0.5M-8M pairs x "
                           f"{args.serve_scale}, 75-150 bp, 131072-pair chunks, Poisson arrivals",
               "samples": 64, "chunks": len(plan), "pairs": int(sizes.sum()),
               "plain_pairs_per_s": plain, "arrival_pairs_per_s": rate, "capacity_pairs_per_s": capacity,
               "sustained_pairs_per_s": float(sizes.sum()) / span_s, "wall_s": wall,
               "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
               "p50_wait_ms": float(np.percentile(wt, 50)), "p99_wait_ms": float(np.percentile(wt, 99)),
               "slots": st["slots"], "batches": st["batches"], "batch_pairs": CH}
        # where the tail comes from: the slowest chunks (arrival order, time
        # since the first submit) and the waiter's class-table inserts
        first = min(i["submit_ms"] for i in infos)
        slow = np.argsort(lat)[::-1][:5]
        out["slowest"] = [{"chunk": int(c), "submit_s": round((infos[c]["submit_ms"] - first) / 1e3, 3),
                           "latency_ms": round(float(lat[c]), 1), "admit_wait_ms": round(float(wt[c]), 1)}
                          for c in slow]
        out["class_insert_ms"] = {"p50": round(float(np.percentile(add_ms, 50)), 3),
                                  "max": round(float(np.max(add_ms)), 1),
                                  "max_at_chunk": int(np.argmax(add_ms))}
        # per-sample EM: the device EM over the served table against the
        # oracle's EM over the oracle's table of the same chunks (a served
        # chunk's records are those of the chunk aligned alone)
        em_ms, rounds, same_tab, same_em = [], [], 0, 0
        ores = [orc.align_pairs(r1.copy(), r2.copy(), args.write_bam) for r1, r2 in pool] if orc is not None else None
        for s in range(64):
            g, o, k_r, ms = tables[s].em(ctx)
            em_ms.append(ms)
            rounds.append(k_r)
            if orc is None:
                continue
            r = ores[rlen[s]]
            parts = [types.SimpleNamespace(recs=r.recs[:2 * n], pos_pool=r.pos_pool, p_pool=r.p_pool)
                     for s2, n in plan if s2 == s]
            want = orc.classes(parts)
            same_tab += int(tables[s].fetch().key() == want.key())
            g0, o0, k0 = orc.em(want)
            same_em += int(k0 == k_r and np.array_equal(g.view(np.uint64), g0.view(np.uint64))
                           and np.array_equal(o.view(np.uint64), o0.view(np.uint64)))
        out["em"] = {"samples": 64, "device_ms_total": round(float(np.sum(em_ms)), 2),
                     "rounds_median": int(np.median(rounds)),
                     "class_tables_equal": None if orc is None else same_tab,
                     "em_bit_exact": None if orc is None else same_em,
                     "bit_exact": None if orc is None else bool(same_tab == 64 and same_em == 64)}
    finally:
        for tb in tables:
            tb.close()
        ctx.close()
    return out


def roofline(tm, dpx_instr_s, chunk, read_bytes, max_len):
    """Rooflines of one single-lane step of the batched form.

    Gap DP (the dominant kernels): SW_align cells evaluated (counted the
    way the reference visits them) per second of the DP kernels, against the
    measured DPX roof: __viaddmin_s16x2 instructions/s x 2 lanes / 2 DPX
    operations per cell (min3-with-add of the edit-distance cell update).
    Seed-table gathers: sector bytes moved per second of seed_probe against
    the measured HBM copy peak; per lookup one 32 B sector for the bucket
    offsets and one per binary-search probe, plus the reads' codes, offsets
    and the hit records written.  Mate rescue: ssw_align cells per second of
    the rescue kernels against the same DPX roof."""
    if tm is None:
        return None, None, None
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    src = "measured" if "hbm_gbs" in peaks else "fallback"
    dpx_cells = dpx_instr_s * 2 / 2 / 1e9   # Gcell/s
    traffic = _profile_traffic()

    dp_s = float(tm["dp_kernel_ms"]) / 1e3
    cells = int(tm["sw_cells"])
    dp = {"kernel": "k_dp_reg<4|8> + k_dp_generic (gap DP, all rounds)", "bound": "dpx",
          "achieved": cells / dp_s / 1e9 if dp_s > 0 else None, "peak": dpx_cells, "unit": "Gcell/s",
          "frac": (cells / dp_s / 1e9) / dpx_cells if dp_s > 0 else None,
          "traffic": traffic.get("k_dp_reg_bytes_per_cell", 0) * cells or None,
          "peak_source": "measured: DPX probe (hera_gpu_dpx_peak) on this GPU",
          "work": {"sw_cells": cells, "dp_jobs": int(tm["dp_jobs"]), "dp_calls": int(tm["dp_calls"]),
                   "kernel_ms": float(tm["dp_kernel_ms"])}}

    n_reads = 2 * chunk
    lookups, probes = int(tm["lookups"]), int(tm["probes"])
    spr = (max_len - 31) // 31 + 1 if max_len >= 31 else 1
    slots = n_reads * 2 * spr
    fixed = read_bytes + 12 * n_reads + 8 * slots
    useful = fixed + 8 * lookups + 16 * probes
    sectors = fixed + 32 * lookups + 32 * probes
    sd_s = float(tm["seed_kernel_ms"]) / 1e3
    seed = {"kernel": "k_seed (seed_probe: hash_get gathers, space 31)", "bound": "hbm",
            "achieved": sectors / sd_s / 1e9 if sd_s > 0 else None, "peak": hbm, "unit": "GB/s",
            "frac": (sectors / sd_s / 1e9) / hbm if sd_s > 0 else None,
            "traffic": traffic.get("k_seed_bytes_per_lookup", 0) * lookups or None,
            "peak_source": src,
            "sector_efficiency": (8 * lookups + 16 * probes) / (32 * lookups + 32 * probes)
            if lookups else None,
            "work": {"lookups": lookups, "probes": probes, "seed_hits": int(tm["seed_hits"]),
                     "useful_bytes": useful, "sector_bytes": sectors, "kernel_ms": float(tm["seed_kernel_ms"])}}

    rs_s = float(tm["rescue_kernel_ms"]) / 1e3
    sc = int(tm["ssw_cells"])
    rescue = {"kernel": "k_rescue_sw (ssw_align, warp per call)", "bound": "dpx",
              "achieved": sc / rs_s / 1e9 if rs_s > 0 else None, "peak": dpx_cells, "unit": "Gcell/s",
              "frac": (sc / rs_s / 1e9) / dpx_cells if rs_s > 0 else None, "traffic": None,
              "work": {"ssw_cells": sc, "kernel_ms": float(tm["rescue_kernel_ms"])}}
    return dp, seed, rescue


def _profile_traffic() -> dict:
    """Per-unit DRAM traffic of the top kernels from the committed ncu
    summary (profiles/traffic.json), scaled by the units of this run."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


if __name__ == "__main__":
    main()
