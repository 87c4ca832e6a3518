"""Benchmark: k-mers compacted per second on one B200 (plain single job).

Workload (default): one synthetic 1 Gbp genome at 41% GC with 5% repeat
families (300 bp-6 kb, 2-50 copies, 1-3% mutations per copy) and 0.1% SNPs,
k = 31, ~1B distinct canonical 31-mers, shuffled, in the reference's text
format, generated on the GPU from a seed.  A step is one pass of the whole
path (pack, minimizer bucketing, tiles, stitch) over that text.

  value  device-resident throughput: text already in HBM, lines left in HBM
  e2e    the same through uc_compact_host: pinned host text -> host lines,
         both copies inside the timed region
  --impl reference   the CPU arm: the reference path timed on the host cores
         over a bounded sample of the same workload

Under torchrun every rank runs its own replica (the path does not shard:
replicas only); value is the sum over ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-mers compacted/s on 1 B200, batched vs plain (bit-exact); HBM % peak; job p99"
UNIT = "k-mers/s"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(st: dict, text_bytes: int, k: int) -> dict:
    """Bytes each phase must move at minimum (every logical array element
    read or written once), from the run's own counts.  W = key bytes, 4-byte
    ids, 8 bytes of bucket ids per k-mer, 20 bytes per segment record."""
    W = 8 if k <= 31 else 16
    n, cp, S, ob = st["n_kmers"], st["n_copies"], st["n_segments"], st["out_bytes"]
    closed, segc = st["closed_bytes"], st["seg_chars"]
    return {
        "pack": text_bytes + n * (W + 8),                 # text in; keys and bucket ids out
        "bucket": n * (W + 8) + cp * (W + 4),             # keys and bucket ids in; copies out
        "tiles": cp * (W + 4) + closed + segc + S * 20,   # copies in; lines, segment chars and records out
        "stitch": S * 20 + segc + (ob - closed),          # segments in; cross-tile lines out
    }


def whole_path_bytes(st: dict, text_bytes: int, k: int) -> int:
    """B_alg of the whole path: in + n (7W + 14I) + out (each phase's minimum
    traffic summed, I = 4-byte ids)."""
    W = 8 if k <= 31 else 16
    return text_bytes + st["n_kmers"] * (7 * W + 14 * 4) + st["out_bytes"]


def traffic_per_copy(kernel: str):
    """DRAM bytes per bucketed copy of the tile kernels from the committed
    ncu capture (profiles/traffic.txt), or None.  Scaled by the run's copy
    count it is the traffic of one launch pair at the bench's size."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) >= 2 and f[0] == kernel:
            return float(f[1])
    return None


def lines_digest(buf) -> int:
    """Order-independent digest of the '\\n'-terminated lines of a uint8
    CUDA tensor: every byte weighted by a mix of its position in its line,
    summed per line, each line's sum mixed, and the mixes summed (mod 2^64).
    Equal multisets of lines give equal digests whatever their order, so a
    job's lines from the batched path and from the plain path compare
    without sorting; a line split, merged or changed changes it."""
    import torch
    from unitigcoarsening_b200 import synth
    n = buf.numel()
    if n == 0:
        return 0
    nl = buf == 10
    ends = torch.nonzero(nl).flatten()
    starts = torch.cat([torch.zeros(1, dtype=ends.dtype, device=buf.device), ends[:-1] + 1])
    line = torch.cumsum(nl.to(torch.int64), 0) - nl.to(torch.int64)
    if int(line[-1]) >= ends.numel():  # bytes after the last newline form a line of their own
        starts = torch.cat([starts, (ends[-1:] + 1) if ends.numel() else starts[:1]])
    rel = torch.arange(n, device=buf.device, dtype=torch.int64) - starts[line]
    v = (buf.to(torch.int64) + 1) * synth._mix(rel * -7046029254386353131 + 0x632BE59BD9B4E019)
    per = torch.zeros(starts.numel(), dtype=torch.int64, device=buf.device).index_add_(0, line, v)
    return int(synth._mix(per).sum().item()) & ((1 << 64) - 1)


def cpu_model() -> str:
    """lscpu's model name of the host cores (or /proc/cpuinfo's)."""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


REF_BIN = os.path.join(ROOT, "oracle", "_ref", "uc_ref_large")


def _cpu_sample(args, spec=None, k=None):
    """Bounded sample of the workload: the same genome model, shorter (or
    the given spec)."""
    import torch
    from unitigcoarsening_b200 import synth
    if spec is None:
        spec = synth.scale_plain(length=int(args.cpu_sample), seed=2)
    with torch.no_grad():
        return synth.make_text(spec, k or args.k, device="cpu").numpy().tobytes()


def _run_reference_binary(text: bytes, k: int, l: int, threads: int):
    """The reference's own driver (compiled from its sources against the
    Kokkos-API shim, OpenMP backend): returns (seconds from its "Total time"
    line, wall seconds)."""
    import re
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.txt")
        outp = os.path.join(td, "out.txt")
        with open(inp, "wb") as f:
            f.write(text)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="spread", OMP_PLACES="threads")
        t0 = time.perf_counter()
        r = subprocess.run([REF_BIN, inp, str(k), str(l), outp], capture_output=True, text=True, env=env,
                           timeout=600)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference exited {r.returncode}: {r.stderr[-300:]}")
        m = re.search(r"Total time: ([0-9.]+)s", r.stdout)
        return (float(m.group(1)) if m else wall), wall


def cpu_baseline(args, steps: int = 1, text: bytes | None = None, sample: str | None = None):
    """Reference CPU path (or, without its binary, the oracle port) timed on
    the host over a bounded sample; returns the cpu_baseline object."""
    if text is None:
        text = _cpu_sample(args)
        sample = (f"{args.cpu_sample / 1e6:g} Mbp genome of the same model (seed 2), {{n}} k-mers, "
                  f"k={args.k}, l={args.l}, text in a file, lines to a file")
    n = int(text[: text.index(b"\n")])
    if os.path.exists(REF_BIN):
        threads = os.cpu_count() or 1
        ts = [_run_reference_binary(text, args.k, args.l, threads)[0] for _ in range(steps)]
        sec = sum(ts) / len(ts)
        kind, cores = "reference", threads
    else:
        from oracle import oracle as O
        O.build()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            O.compact(text, args.k)
            ts.append(time.perf_counter() - t0)
        sec = sum(ts) / len(ts)
        kind, cores = "port", 1
    return {"value": n / sec, "unit": UNIT, "cores": cores, "kind": kind, "seconds": sec, "n_kmers": n,
            "cpu_model": cpu_model(), "nproc": os.cpu_count(), "sample": sample.format(n=n)}


def reference_throughput(args):
    for _ in range(args.warmup):
        cpu_baseline(args, steps=1)
    cb = cpu_baseline(args, steps=max(1, args.steps))
    cfg = {"workload": f"plain single job (bounded CPU sample): {args.cpu_sample / 1e6:g} Mbp genome, 41% GC, "
                       f"5% repeat families, 0.1% SNPs, k={args.k}", "k": args.k, "l": args.l,
           "n_kmers": cb["n_kmers"],
           "sample_of": f"the GPU arm's {args.genome / 1e9:g} Gbp job of the same model (~1.0B k-mers); "
                        f"this arm times {cb['n_kmers']} k-mers of it per step"}
    return {"value": cb["value"], "ms_per_step": cb["seconds"] * 1e3, "config": cfg, "cpu_baseline": cb}


def run_reference_arm(args, rank):
    """CPU arm: the reference path on the host cores over a bounded sample."""
    if rank != 0:
        return
    res = reference_throughput(args)
    line = {"metric": METRIC, "impl": "reference", "value": res["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8/u64", "data": "synthetic",
            "config": res["config"], "cpu_baseline": res["cpu_baseline"],
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def replica_totals(ms: float, n: int, dist=None, device: str = "cuda"):
    """Whole-job figures over independent replicas (one job per rank, no
    data-path collective): the step time is the slowest rank's, the value
    the k-mers of all ranks over that time.  Every rank takes the same two
    collectives and a barrier."""
    if dist is None:
        return ms, n / (ms / 1e3)
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([n], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    dist.barrier()
    ms_max = float(t.item())
    return ms_max, float(c.item()) / (ms_max / 1e3)


def measure_batched(args, device: int):
    """Many small jobs (log-normal lengths, median 3 Mbp, 0.5-8 Mbp, GC
    30-70%, 0.2% SNPs, k=31), device-resident.  The jobs are generated on
    the GPU in chunks of --batch-gen-chunk (untimed; all 4096 texts would not
    fit in HBM at once).  For each chunk, an untimed batched pass (the
    device arenas grow to the chunk's largest batch there), one timed pass of
    the plain loop (one compaction per job) and one timed pass of the batched
    form (--batch-chunk jobs per launch sequence, one tile queue each), then
    an untimed check that every job's lines are the same in both (order-free
    line digests).  Times are summed over the chunks."""
    import torch
    from unitigcoarsening_b200 import Compactor, synth
    comp = Compactor(device)
    C = max(1, args.batch_chunk)
    G = max(C, args.batch_gen_chunk // C * C)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    plain_ms = batch_ms = gen_s = 0.0
    n_total, launches, mismatched, warm = 0, 0, [], False
    for g0 in range(0, args.batch_jobs, G):
        ids = list(range(g0, min(args.batch_jobs, g0 + G)))
        t0 = time.perf_counter()
        with torch.no_grad():
            texts = [synth.make_text(synth.batched_job(j, seed=4), 31, device="cuda") for j in ids]
        torch.cuda.synchronize()
        gen_s += time.perf_counter() - t0
        caps = [comp.output_bound(t.numel(), 31) for t in texts]
        one = torch.empty(max(caps), dtype=torch.uint8, device="cuda")  # the plain loop reuses one buffer
        chunks = [list(range(i, min(i + C, len(texts)))) for i in range(0, len(texts), C)]
        bout = torch.empty(max(sum((caps[j] + 15) // 16 * 16 for j in ch) for ch in chunks) + 64,
                           dtype=torch.uint8, device="cuda")

        def plain(check=None):
            for i, t in enumerate(texts):
                r = comp.compact(t, 31, args.l, out=one)
                if check is not None:
                    check.append(lines_digest(r))

        def batched(check=None):
            n, nl = 0, 0
            for ch in chunks:
                res, st = comp.compact_batch([texts[j] for j in ch], 31, args.l, out=bout, stats=True)
                n += int(st["n_kmers"])
                nl += int(st["launches"])
                if check is not None:
                    check += [lines_digest(r) for r in res]
            return n, nl

        # untimed: every group's batched pass once first, so that the
        # context's device arenas already hold this group's largest batch
        # (growing an arena frees and allocates device memory, whose cost
        # varies from run to run and is not compaction work)
        if not warm:
            plain()
            warm = True
        batched()
        torch.cuda.synchronize()
        e0.record(stream)
        plain()
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms += e0.elapsed_time(e1)
        e0.record(stream)
        n, nl = batched()
        e1.record(stream)
        torch.cuda.synchronize()
        batch_ms += e0.elapsed_time(e1)
        n_total += n
        launches += nl
        dp, db = [], []
        plain(dp)
        batched(db)
        mismatched += [ids[i] for i in range(len(ids)) if dp[i] != db[i]]
        del texts, one, bout
        torch.cuda.empty_cache()
    comp.close()
    del comp
    torch.cuda.empty_cache()
    return {"workload": f"{args.batch_jobs} jobs: log-normal length (median 3 Mbp, 0.5-8 Mbp), GC 30-70%, "
                        f"0.2% SNPs, k=31, device-resident; batched {C} jobs per launch sequence; generated "
                        f"{G} jobs at a time (untimed)",
            "jobs": args.batch_jobs, "n_kmers": n_total,
            "batched": {"value": n_total / (batch_ms / 1e3), "ms": batch_ms, "launches": launches},
            "plain": {"value": n_total / (plain_ms / 1e3), "ms": plain_ms},
            "speedup": plain_ms / batch_ms, "per_job_lines_equal": not mismatched,
            "mismatched_jobs": mismatched[:16], "check": "order-free digest of each job's lines, plain vs batched",
            "gen_seconds": gen_s, "unit": UNIT}


def measure_configs(args, device: int):
    """The two other single-job shapes, device-resident, each on a fresh
    context: the small plain job (1 Mbp, uniform ACGT, 200 SNP bubbles,
    k=31) and the wide-k job (200 Mbp, 50% GC, 3% tandem repeats, 0.05% SNPs,
    k=63, 128-bit keys).  Mean of 3 timed steps after 2 warm-up steps."""
    import torch
    from unitigcoarsening_b200 import Compactor, synth
    res = {}
    for name, spec, k in [("small_plain_1Mbp_k31", synth.small_plain(), 31),
                          ("wide_k63_200Mbp", synth.wide_k(), 63)]:
        with torch.no_grad():
            text = synth.make_text(spec, k, device="cuda")
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        comp = Compactor(device)
        out = torch.empty(comp.output_bound(text.numel(), k), dtype=torch.uint8, device="cuda")
        l = min(args.l, k - 1)
        for _ in range(2):
            comp.compact(text, k, l, out=out)
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            r, st = comp.compact(text, k, l, out=out, stats=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        res[name] = {"value": st["n_kmers"] / (ms / 1e3), "unit": UNIT, "ms": ms, "n_kmers": int(st["n_kmers"]),
                     "k": k, "l_used": int(st["l_used"]), "text_bytes": int(text.numel()),
                     "phase_ms": {p: round(st["ms_" + p], 3) for p in ("pack", "bucket", "tiles", "stitch")}}
        if text.numel() < (1 << 30):
            # host memory to host memory through uc_compact_host (pinned), the
            # form comparable with the reference's file-to-file run
            htext = torch.empty(text.numel(), dtype=torch.uint8, pin_memory=True)
            htext.copy_(text)
            hout = torch.empty(comp.output_bound(text.numel(), k), dtype=torch.uint8, pin_memory=True)
            for _ in range(2):
                comp.compact_host(htext, k, l, out=hout)
            t0 = time.perf_counter()
            for _ in range(5):
                comp.compact_host(htext, k, l, out=hout)
            hs = (time.perf_counter() - t0) / 5
            res[name]["host_to_host"] = {"value": st["n_kmers"] / hs, "ms": hs * 1e3, "api": "uc_compact_host"}
            del htext, hout
        comp.close()
        del comp, text, out
        torch.cuda.empty_cache()
    return res


def measure_serving(args, device: int):
    """Serving loop: a pool of distinct jobs (k-mer counts log-uniform in
    [10k, 50M], k = 31 with p 0.7 else 63) in pinned host memory; capacity =
    the plain sequential host-to-host path over the pool.  Then (1) Poisson
    arrivals at 80% of that capacity, each a job drawn from the pool, served
    by uc_server (footprint admission, batching, overlapping lanes), with
    latency percentiles; (2) a saturation run: --serve-burst jobs submitted
    at once, whose completion rate is the server's sustained capacity."""
    import psutil
    import random
    import threading
    import torch
    from unitigcoarsening_b200 import Compactor, Server, UCError, synth
    pool, pool_bytes = [], 0
    host_cap = psutil.virtual_memory().available // 2  # the pool (results are dropped), and headroom
    t0 = time.perf_counter()
    with torch.no_grad():
        for j in range(args.serve_pool):
            spec, k = synth.served_job(j, seed=5)
            t = synth.make_text(spec, k, device="cuda")
            if pool and pool_bytes + t.numel() > host_cap:
                break
            h = torch.empty(t.numel(), dtype=torch.uint8, pin_memory=True)
            h.copy_(t)
            del t
            pool_bytes += h.numel()
            pool.append((h, k, int(bytes(h[:24].numpy()).split(b"\n")[0])))
    gen_s = time.perf_counter() - t0
    torch.cuda.empty_cache()
    # capacity: plain sequential path, host text to host lines (pinned both
    # ways, like the server's lanes); one output buffer of the largest size
    comp = Compactor(device)
    hout = torch.empty(max(comp.output_bound(h.numel(), k) for h, k, _ in pool), dtype=torch.uint8,
                       pin_memory=True)
    seq_s = 0.0
    for rep in range(2):
        t0 = time.perf_counter()
        for h, k, n in pool:
            comp.compact_host(h, k, min(args.l, k - 1), out=hout)
        if rep:
            seq_s = time.perf_counter() - t0
    comp.close()
    del comp, hout
    torch.cuda.empty_cache()
    pool_kmers = sum(n for _, _, n in pool)
    capacity = pool_kmers / seq_s
    mean_n = pool_kmers / len(pool)

    def serve(arrivals):
        results = [None] * len(arrivals)
        with Server(device=device, lanes=4, max_batch=32) as srv:
            tickets = [None] * len(arrivals)
            ready = threading.Semaphore(0)

            def waiter():
                for i in range(len(arrivals)):
                    ready.acquire()
                    try:
                        results[i] = srv.wait(tickets[i], timeout=600, fetch=False)[1]
                    except UCError as ex:
                        results[i] = {"status": ex.status, "latency_ms": 0.0}

            wt = threading.Thread(target=waiter)
            wt.start()
            t0 = time.perf_counter()
            for i, (ta, j) in enumerate(arrivals):
                d = ta - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                h, k, _ = pool[j]
                tickets[i] = srv.submit(h, k, min(args.l, k - 1))
                ready.release()
            wt.join()
            wall = time.perf_counter() - t0
            tot = srv.stats()
        bad = sum(1 for r in results if r["status"] != 0)
        served = sum(pool[j][2] for _, j in arrivals)
        lat = sorted(r["latency_ms"] for r in results)
        pct = lambda q: lat[min(len(lat) - 1, int(q * (len(lat) - 1) + 0.5))]
        return {"jobs": len(arrivals), "n_kmers": served, "wall_s": wall,
                "sustained": {"value": served / wall, "unit": UNIT}, "failed_jobs": bad,
                "latency_ms": {"p50": pct(0.5), "p99": pct(0.99), "max": lat[-1], "mean": sum(lat) / len(lat)},
                "batches": int(tot["batches"]), "batched_jobs": int(tot["batched_jobs"]),
                "pool_gb": tot["pool_bytes"] / 1e9, "pool_peak_gb": tot["pool_peak_bytes"] / 1e9}

    rate = 0.8 * capacity / mean_n  # jobs per second
    rnd = random.Random(7)
    arrivals, t = [], 0.0
    for _ in range(args.serve_jobs):
        t += rnd.expovariate(rate)
        arrivals.append((t, rnd.randrange(len(pool))))
    load = serve(arrivals)
    sat = None
    if args.serve_burst > 0:
        rnd = random.Random(11)
        sat = serve([(0.0, rnd.randrange(len(pool))) for _ in range(args.serve_burst)])
        sat["offered"] = "all jobs submitted at once (offered load far above capacity)"
        sat["vs_plain_sequential"] = sat["sustained"]["value"] / capacity
    return {"workload": f"Poisson arrivals at 80% of the plain sequential capacity; {args.serve_jobs} jobs drawn "
                        f"from {len(pool)} distinct jobs ({pool_bytes / 1e9:.1f} GB of text in pinned host "
                        f"memory), k-mer counts log-uniform in [10k, 50M], k = 31 (p 0.7) or 63, host memory to "
                        f"host memory", "jobs": args.serve_jobs, "distinct_jobs": len(pool),
            "offered_jobs_per_s": rate, "offered": {"value": 0.8 * capacity, "unit": UNIT},
            "sustained": load["sustained"], "plain_sequential": {"value": capacity, "unit": UNIT},
            "latency_ms": load["latency_ms"], "wall_s": load["wall_s"], "n_kmers": load["n_kmers"],
            "failed_jobs": load["failed_jobs"], "batches": load["batches"], "batched_jobs": load["batched_jobs"],
            "pool_gb": load["pool_gb"], "pool_peak_gb": load["pool_peak_gb"], "saturation": sat,
            "gen_seconds": gen_s}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--genome", type=float, default=1e9, help="genome length (bp)")
    ap.add_argument("--model", default="scale_plain", choices=["scale_plain", "wide_k", "small_plain"],
                    help="genome model of the timed job (the headline is scale_plain)")
    ap.add_argument("--k", type=int, default=31)
    ap.add_argument("--l", type=int, default=8)
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample", type=float, default=4e6, help="genome length of the CPU sample")
    ap.add_argument("--cpu-sample-large", type=float, default=16e6,
                    help="genome length of the larger CPU sample (0: skip)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (library defaults)")
    ap.add_argument("--tune-sample", type=float, default=2e8, help="genome length the autotuner times")
    ap.add_argument("--batch-jobs", type=int, default=4096, help="jobs of the batched-vs-plain comparison (0: skip)")
    ap.add_argument("--batch-chunk", type=int, default=64, help="jobs per batched launch sequence")
    ap.add_argument("--batch-gen-chunk", type=int, default=512, help="jobs generated on the GPU at a time")
    ap.add_argument("--no-configs", action="store_true", help="skip the small and wide-k single-job shapes")
    ap.add_argument("--serve-jobs", type=int, default=20000, help="arrivals of the serving measurement (0: skip)")
    ap.add_argument("--serve-pool", type=int, default=256, help="distinct jobs the arrivals draw from")
    ap.add_argument("--serve-burst", type=int, default=2000, help="jobs of the saturation run (0: skip)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from unitigcoarsening_b200 import Compactor, synth
    from unitigcoarsening_b200 import build as B
    B.build()
    comp = Compactor(local)

    # autotuner (untimed): the library's tuner on a sample of the same model
    tuning = None
    if not args.no_tune:
        with torch.no_grad():
            sample = synth.make_text(synth.scale_plain(length=int(args.tune_sample), seed=3 + rank), args.k,
                                     device="cuda")
        tuning = comp.autotune(sample, args.k, args.l, reps=3, max_ms=20000)
        del sample
        torch.cuda.empty_cache()

    t0 = time.time()
    seed = {"scale_plain": 2, "wide_k": 3, "small_plain": 1}[args.model] + rank
    spec = getattr(synth, args.model)(length=int(args.genome), seed=seed)
    with torch.no_grad():
        text = synth.make_text(spec, args.k, device="cuda")
    torch.cuda.synchronize()
    gen_s = time.time() - t0
    text_bytes = text.numel()
    torch.cuda.empty_cache()

    out = torch.empty(comp.output_bound(text_bytes, args.k), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    st = None
    for _ in range(max(3, args.warmup)):
        res, st = comp.compact(text, args.k, args.l, out=out, stats=True)
    torch.cuda.synchronize()
    n = int(st["n_kmers"])

    # timed region: device-resident text (> L2, so no flush is needed)
    phase = {"pack": 0.0, "bucket": 0.0, "tiles": 0.0, "stitch": 0.0}
    kern = {"tile_warp": 0.0, "tile_block": 0.0}
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            res, st = comp.compact(text, args.k, args.l, out=out, stats=True)
            for p in phase:
                phase[p] += st["ms_" + p]
            for p in kern:
                kern[p] += st["ms_" + p]
        ev1.record(stream)
        torch.cuda.synchronize()
    ms, value = replica_totals(ev0.elapsed_time(ev1) / args.steps, n, dist, "cuda")
    for p in phase:
        phase[p] /= args.steps
    for p in kern:
        kern[p] /= args.steps

    # roofline of the dominant kernels: the two tile kernels (warp tiles and
    # block tiles), timed by CUDA events on the library's stream around their
    # launches; algorithmic bytes = the tile phase's minimum traffic
    peak, peak_kind = peaks()
    alg = algorithmic_bytes(st, text_bytes, args.k)
    tile_ms = kern["tile_warp"] + kern["tile_block"]
    achieved = alg["tiles"] / (tile_ms / 1e3) / 1e9
    tpc = traffic_per_copy("tiles")
    whole = whole_path_bytes(st, text_bytes, args.k) / (ms / 1e3) / 1e9

    # e2e: host text -> host lines through the C ABI
    e2e = None
    if not args.no_e2e:
        import psutil
        need = 2 * text_bytes + (1 << 30)
        if psutil.virtual_memory().available > need:
            htext = torch.empty(text_bytes, dtype=torch.uint8, pin_memory=True)
            htext.copy_(text)
            hout = torch.empty(comp.output_bound(text_bytes, args.k), dtype=torch.uint8, pin_memory=True)
            del text, out
            torch.cuda.empty_cache()
            # one call: upload, compaction, download in sequence
            comp.compact_host(htext, args.k, args.l, out=hout)
            t1 = time.perf_counter()
            r, est = comp.compact_host(htext, args.k, args.l, out=hout, stats=True)
            single_s = time.perf_counter() - t1
            # steps through uc_compact_host_many: each step's text is uploaded
            # while the step before it finishes; every upload and download is
            # inside the timed region
            K = max(2, args.e2e_steps)
            comp.compact_host_many([htext] * 2, args.k, args.l, outs=[hout] * 2)
            t1 = time.perf_counter()
            res_many, mst = comp.compact_host_many([htext] * K, args.k, args.l, outs=[hout] * K, stats=True)
            e2e_s = (time.perf_counter() - t1) / K
            assert all(x.numel() == int(est["out_bytes"]) for x in res_many)
            e2e = {"value": world * n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": text_bytes,
                   "d2h_bytes_per_step": int(est["out_bytes"]), "ms_per_step": e2e_s * 1e3, "steps": K,
                   "pinned": True, "api": "uc_compact_host_many (next step's upload overlaps this step)",
                   "single_call": {"value": world * n / single_s, "ms": single_s * 1e3, "api": "uc_compact_host"}}
            del htext, hout
        else:
            e2e = {"value": None, "unit": UNIT, "skipped": f"host RAM below {need >> 30} GiB"}
    text = out = None
    torch.cuda.empty_cache()

    comp.close()
    del comp
    torch.cuda.empty_cache()
    batched = measure_batched(args, local) if args.batch_jobs > 0 else None
    configs = measure_configs(args, local) if not args.no_configs else None
    serving = measure_serving(args, local) if args.serve_jobs > 0 else None

    cpu = cpu_pairs = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(args)
        # the same configs on both sides: the small plain job exactly (the one
        # the reference runs on its CPU path), and a larger sample of the
        # headline model to show how the CPU rate moves with size
        c1 = cpu_baseline(args, text=_cpu_sample(args, synth.small_plain(), 31),
                          sample="small plain job: 1 Mbp uniform genome, 200 SNP bubbles, {n} k-mers, k=31, l=8")
        cpu_pairs = {"small_plain_1Mbp_k31": {"cpu_reference": c1,
                                              "gpu": (configs or {}).get("small_plain_1Mbp_k31"),
                                              "same_config": True}}
        if args.cpu_sample_large > 0:
            big = cpu_baseline(args, text=_cpu_sample(args, synth.scale_plain(length=int(args.cpu_sample_large),
                                                                              seed=2), args.k),
                               sample=f"{args.cpu_sample_large / 1e6:g} Mbp genome of the headline model (seed 2), "
                                      f"{{n}} k-mers, k={args.k}, l={args.l}")
            cpu_pairs["scale_plain_sample"] = {"cpu_reference": big, "gpu": None, "same_config": False,
                                               "note": "CPU rate at a larger sample of the headline model"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8/u64 (2-bit packed keys, 32-bit ids)", "data": "synthetic",
            "config": {"workload": (f"plain single job: {args.genome / 1e9:g} Gbp genome, 41% GC, 5% repeat "
                                    f"families, 0.1% SNPs, k={args.k}") if args.model == "scale_plain" else
                                   f"{args.model} job: {args.genome / 1e9:g} Gbp genome, k={args.k}",
                       "model": args.model, "k": args.k, "l": args.l,
                       "l_used": int(st["l_used"]),
                       "n_kmers": n, "text_bytes": text_bytes, "l2_flush": "inputs larger than L2",
                       "parallelism": f"replicas x{world}", "genome_seed": seed},
            "roofline": {"bound": "hbm", "kernel": "k_tile_warp + k_tile", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (tpc * st["n_copies"]) if tpc else None,
                         "algorithmic_bytes": alg["tiles"], "ms": tile_ms,
                         "whole_path_achieved": whole, "whole_path_frac": whole / peak},
            "phase_ms": phase, "kernel_ms": kern, "algorithmic_bytes": alg,
            "stats": {k2: (float(v) if isinstance(v, float) else int(v)) for k2, v in st.items()},
            "tuning": tuning,
            "batched_vs_plain": batched, "serving": serving, "other_configs": configs,
            "e2e": e2e, "cpu_baseline": cpu, "cpu_vs_gpu": cpu_pairs, "clocks": clk.summary(),
            "gpu_launches": int(st["launches"]) * args.steps,
            "gen_seconds": gen_s,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
