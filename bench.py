#!/usr/bin/env python
"""Iris comparisons/sec of the 3-party uniqueness hot path on B200.

Workload (the GPU plain drop-in configuration): 3 parties co-resident on one
GPU, 64 queries x 31 rotations (1984 query rows in 64 slots of 32) against
524,288 share-DB entries per party, threshold ratio 0.375 (A = 16384).  One
step = one batch, the DB scanned in chunks of 65,536 entries (--db-chunk): per
chunk the six limb GEMMs (3 parties x code/mask) in one tcgen05 launch, then
the fused threshold + open + rotation OR into the match bitmap.
One comparison = one (query iris, DB entry) pair over all 31 rotations,
computed jointly by the three parties.

  value -- comparisons/s with the queries already expanded in HBM;
  e2e   -- the same through the public API with host I/O inside every step:
           H2D of the six engines' base query shares from pinned memory,
           device-side rotation expansion, GEMMs, threshold, result merge and
           D2H of the per-query results.

The DB (60.4 GB for the three parties) is far larger than L2, so no L2 flush
is needed between steps.  Synthetic seeded data (no dataset exists for this
workload).  `--impl reference` times the CPU restatement of the reference's
CPU path (per-party rotation-aware dots, summed, thresholded, OR over
rotations) on the host cores.

Multi-GPU (torchrun): each rank hosts its own 524,288-entry shard of all three
parties (global entry g on rank g % N) and processes the same query batch; the
scan needs no collective (weak scaling); the end-to-end step merges the ranks'
match results with one all_gather (irisb200.shard); the max step time over
ranks is reported.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "iris-mpc_b200")]

METRIC = "iris comparisons/sec (3-party, 1 B200)"
UNIT = "comparisons/s"
DB_SEED = 0xDEADBEEF
Q_SEED = 42
K_CODE, K_MASK = 12800, 6400


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--db", type=int, default=524288, help="DB entries per party (per GPU)")
    ap.add_argument("--queries", type=int, default=64)
    ap.add_argument("--threshold-a", type=int, default=16384)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cublas", action="store_true")
    ap.add_argument("--mode", default="plain", choices=["plain", "serving", "sweep", "batched"],
                    help="plain: the drop-in batch (+ batched and serving legs); serving: Poisson sweep; "
                         "sweep: single-party GEMM and comparison-kernel roofline sweep; "
                         "batched: batch sizes --batch-sizes, batched engine vs plain slots")
    ap.add_argument("--batch-sizes", default="1,16,64,256", help="batched mode: requests per batch")
    ap.add_argument("--batched-requests", type=int, default=256, help="requests per batched-leg batch (0 = skip)")
    ap.add_argument("--rates", default="50,200,500,1000,2000", help="serving: offered loads, requests/s")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serving: arrival window per load")
    ap.add_argument("--chunk", type=int, default=65536, help="serving: DB chunk per step")
    ap.add_argument("--db-chunk", type=int, default=65536,
                    help="plain step: DB entries per GEMM + threshold launch pair (0 = whole DB per launch)")
    ap.add_argument("--serving-arms", default="served,plain", help="serving: which servers to run")
    ap.add_argument("--serving-rate", type=float, default=600.0,
                    help="default run: offered load of its serving leg, requests/s (0 = skip)")
    return ap.parse_args()


def measured_peaks() -> dict:
    """MEASURED_PEAKS.json (written beside the repository by the GPU pool's
    driver) as floats: hbm_gbs, bf16_tflops (burst), bf16_tflops_sustained;
    each None when absent.  A value may be a number or {"value": number}."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    raw = {}
    if os.path.exists(path):
        try:
            with open(path) as f:
                raw = json.load(f)
        except (OSError, ValueError):
            raw = {}

    def num(x):
        if isinstance(x, dict):
            x = x.get("value")
        try:
            return float(x) if x is not None else None
        except (TypeError, ValueError):
            return None
    out = {k: num(raw.get(k)) for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained")}
    out["present"] = os.path.exists(path)
    return out


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []  # (host time, csv line)
        self.proc = None
        self.windows = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def mark(self):
        """Context manager recording a timed window; summaries use samples inside windows."""
        sampler = self

        class _W:
            def __enter__(self_):
                self_.t0 = time.perf_counter()
                return self_

            def __exit__(self_, *exc):
                sampler.windows.append((self_.t0, time.perf_counter()))
        return _W()

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, window=None):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lo, hi = window if window else (float("-inf"), float("inf"))
        for t, ln in self.lines:
            if not (lo <= t <= hi + 0.25):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(n_query=8, n_db=8192, min_seconds=10.0):
    """The CPU restatement of the reference's CPU path on config 0's shape."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import oracle as O
    import workload as W
    O.build()
    codes, masks, cs, ms = W.make_db(O, n_db, DB_SEED)
    planted = {j: (int(j * 997 % n_db), (j % 31) - 15) for j in range(0, n_query, 10)}
    qc, qm, _ = W.make_queries(O, n_query, codes, masks, Q_SEED, planted)
    q_code = [W.rotated_rows(O, qc[p]) for p in range(3)]
    q_mask = [W.rotated_rows(O, qm[p]) for p in range(3)]
    cores = os.cpu_count() or 1
    reps, t0 = 0, time.perf_counter()
    while True:
        O.cpu_plain_match(q_code, q_mask, n_query, list(cs), list(ms), 16384, cores)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or reps >= 50:
            break
    value = reps * n_query * n_db / el
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n_query} queries x 31 rotations vs {n_db} entries, 3 parties, {reps} pass(es), "
                      f"{el:.1f} s, OpenMP on {cores} threads"}


def measure_int8_peak(torch, n=16384):
    """Dense INT8 denominator: cuBLAS int8 GEMM (torch._int_mm) n^3, best of 10."""
    a = torch.randint(-128, 127, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-128, 127, (n, n), dtype=torch.int8, device="cuda").t()
    for _ in range(3):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(10):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def cublas_limb_gemms(torch, m, n_rows, batches=6, clk=None):
    """The reference's dot products on this GPU: per party, 3 cublasGemmEx int8
    limb GEMMs for codes (K = 12800) and 3 for masks (K = 6400) via torch._int_mm
    (share_db.rs:62-112,823-843), i32 outputs, no reduction or masking.  Whole
    batches (3 parties x 6 GEMMs) run back to back after two warm-up batches,
    so the clocks settle under the power cap as they do for the fused kernel.
    Returns ms per batch (and the clock record of the timed window)."""
    n = (n_rows + 7) // 8 * 8
    a_code = torch.randint(-128, 127, (m, K_CODE), dtype=torch.int8, device="cuda")
    b_code = torch.randint(-128, 127, (n, K_CODE), dtype=torch.int8, device="cuda").t()
    a_mask = torch.randint(-128, 127, (m, K_MASK), dtype=torch.int8, device="cuda")
    b_mask = torch.randint(-128, 127, (n, K_MASK), dtype=torch.int8, device="cuda").t()

    def batch():
        for _ in range(3):
            for _ in range(3):
                torch._int_mm(a_code, b_code)
            for _ in range(3):
                torch._int_mm(a_mask, b_mask)
    for _ in range(2):
        batch()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    win = clk.mark() if clk else None
    if win:
        win.__enter__()
    s.record()
    for _ in range(batches):
        batch()
    e.record()
    e.synchronize()
    if win:
        win.__exit__(None, None, None)
    del a_code, b_code, a_mask, b_mask
    torch.cuda.empty_cache()
    ms = s.elapsed_time(e) / batches
    return ms, (clk.summary(clk.windows[-1]) if clk else None)


def request_mix(n, code, mask, planted, db_len, seed, p_reauth=0.2, p_append=0.0):
    """Requests of the batched/serving workloads: rotations 1/16/31 (uniform),
    50% mirrored, p_reauth reauth (target = the planted entry of a planted
    query, else a random entry), p_append appends; query j of the pool
    (code/mask [3][nq][K]) is used cyclically."""
    import numpy as np
    from irisb200.batched import Request
    rng = np.random.default_rng(seed)
    nq = code.shape[1]
    out = []
    for i in range(n):
        j = i % nq
        u = rng.random()
        if u < p_append:
            out.append(Request(code=None, mask=None, kind="append"))
            continue
        kind = "reauth" if rng.random() < p_reauth else "uniqueness"
        target = -1
        if kind == "reauth":
            target = planted[j][0] if j in planted else int(rng.integers(0, db_len))
        out.append(Request(code=code[:, j], mask=mask[:, j], n_rot=int(rng.choice([1, 16, 31])),
                           mirrored=bool(rng.random() < 0.5), kind=kind, target=target))
    return out


def comparisons_of(r, db_len):
    """(query orientation, DB entry) pairs a request is compared on: a
    uniqueness request scans the DB once per orientation, a reauth request
    compares each orientation with its one target."""
    k = 2 if r.mirrored else 1
    return k * db_len if r.kind == "uniqueness" else k


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_baseline()
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": "CPU plain method (reference CPU path restated in C, OpenMP): "
                                   "3 parties in-process, 8 queries x 31 rotations vs 8192 entries",
                       "threshold_ratio": 0.375},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    import irisb200

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    M, NQ = args.db, args.queries
    n_rows = NQ * 32
    A = args.threshold_a
    dm = irisb200.DeviceManager(local)
    seeds = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
    # batched leg: its request mix, and the query rows of its packed uniqueness pass
    reqs = None
    q_cap = n_rows
    if args.batched_requests and world == 1:
        from irisb200.batched import centred_rotations, pack
        nb = args.batched_requests
        bpl = {j: (int((j * 104729 + 7) % M), (j * 5) % 31 - 15) for j in range(0, nb, 10)}
        bc, bm = irisb200.synth_queries(DB_SEED + rank, Q_SEED + 1, nb, bpl)
        reqs = request_mix(nb, bc, bm, bpl, M, seed=7)
        lay = pack([list(centred_rotations(r.n_rot)) for r in reqs if r.kind == "uniqueness"
                    for _ in range(2 if r.mirrored else 1)])
        q_cap = max(n_rows, -(-lay.n_rows // 256) * 256)  # room for the 256-row tile padding
    ce = [irisb200.ShareDB(p, dm, M, q_cap, K_CODE, seeds[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, M, q_cap, K_MASK, seeds[p]) for p in range(3)]
    for e in ce + me:
        e.alloc_db(M + 256)  # room for the serving leg's appends
    t0 = time.perf_counter()
    irisb200.synth_db(ce, me, DB_SEED + rank, 0, M)
    synth_s = time.perf_counter() - t0
    c = irisb200.Circuits(dm, seeds)
    dc = irisb200.DistanceComparator(dm, NQ, M, match_list_cap=1 << 16)

    # 10% of the queries are planted near-duplicates of DB entries of this shard
    planted = {j: (int((j * 7919 + 13) % M), (j * 7) % 31 - 15) for j in range(0, NQ, 10)}
    pin_c = irisb200.PinnedArray((3, NQ, K_CODE), np.uint16)
    pin_m = irisb200.PinnedArray((3, NQ, K_MASK), np.uint16)
    irisb200.synth_queries(DB_SEED + rank, Q_SEED, NQ, planted, code_out=pin_c.array, mask_out=pin_m.array)
    slots = [(j, 0, 31, j) for j in range(NQ)]
    engines = ce + me
    mults = [1, 1, 1, 2, 2, 2]

    def upload():
        for p in range(3):
            ce[p].query_upload_slots(pin_c.array[p], slots)
            me[p].query_upload_slots(pin_m.array[p], slots)

    s0 = torch.cuda.ExternalStream(dm.stream(0), device=torch.device("cuda", local))

    # The DB is scanned in chunks of GEMM + threshold launch pairs, as the
    # reference's actor scans it (DB_CHUNK_SIZE per device): alternating the
    # tensor-bound GEMM with the ALU-bound threshold at this granularity keeps
    # the power-capped clock steadier than one long launch of each (measured
    # 160 ms per batch at 65,536 entries against 167 ms whole-DB).
    chunk = args.db_chunk if 0 < args.db_chunk < M else M
    chunks = [(o, min(chunk, M - o)) for o in range(0, M, chunk)]

    def scan(ev=None):
        for k, (off, ln) in enumerate(chunks):
            if ev:
                ev[k][0].record(s0)
            irisb200.dot_many(engines, mults, off, ln)
            if ev:
                ev[k][1].record(s0)
            dc.compare_threshold_open(c, ce, me, off, ln, NQ, A)
            if ev:
                ev[k][2].record(s0)

    def device_step(ev=None):
        dc.reset()
        scan(ev)

    clk = ClockSampler(local).__enter__()
    time.sleep(2.0)  # let nvidia-smi initialise before anything is timed
    upload()
    for _ in range(args.warmup):
        device_step()
    dm.synchronize()

    # ---------------- device-resident timing ----------------
    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in chunks] for _ in range(args.steps)]
    begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    dm.synchronize()
    torch.cuda.synchronize()
    with clk.mark():
        begin.record(s0)
        for i in range(args.steps):
            device_step(evs[i])
        end.record(s0)
        end.synchronize()
    dm.synchronize()
    total_ms = begin.elapsed_time(end)
    gemm_ms = [sum(e[0].elapsed_time(e[1]) for e in evs[i]) for i in range(args.steps)]  # per step, all chunks
    thr_ms = [sum(e[1].elapsed_time(e[2]) for e in evs[i]) for i in range(args.steps)]
    batch_ms = [evs[i][0][0].elapsed_time(evs[i][-1][2]) for i in range(args.steps)]
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    per_step = total_ms / args.steps
    comps = NQ * M * world
    value = comps / (per_step * 1e-3)

    # correctness guard on the measured run: the planted queries must match
    dc.join_db_matches(NQ, M)
    final, counters, _ = dc.fetch_final_results(NQ)
    planted_found = sum(1 for j, (e, _) in planted.items() if final[j] <= e and counters[j] >= 1)

    # ---------------- end-to-end timing through the public API ----------------
    h2d = 3 * NQ * (K_CODE + K_MASK) * 2
    d2h = NQ * 4 * 2 + NQ * irisb200.MAX_MATCHES_LEN * 4

    def e2e_step():
        upload()
        dc.reset()
        scan()
        dc.join_db_matches(NQ, M)
        res = dc.fetch_final_results(NQ)
        if dist:  # merge the shards' results (get_merged_results over ranks): one all_gather
            from irisb200.shard import exchange_results
            return exchange_results(*res, device=torch.device("cuda", local))
        return res

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if dist:
        dist.barrier()
    dm.synchronize()
    lat = []
    with clk.mark():
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ts = time.perf_counter()
            e2e_step()
            lat.append((time.perf_counter() - ts) * 1e3)
        e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = comps * args.steps / e2e_s

    # ---------------- batched uneven leg (same engines, same DB) ----------------
    batched = None
    if reqs:
        from irisb200.batched import BatchedEngine
        n_var = sum(2 if r.mirrored else 1 for r in reqs if r.kind == "uniqueness")
        n_reauth = sum(2 if r.mirrored else 1 for r in reqs if r.kind == "reauth")
        eng = BatchedEngine(dm, ce, me, c, max_variants=max(64, n_var), max_reauth=max(16, n_reauth),
                            threshold_a=A, seeds=seeds, autotune=True)
        for _ in range(max(2, args.warmup)):  # the first autotunes and captures
            eng.run(reqs)
        dm.synchronize()
        blat = []
        with clk.mark():
            tb = time.perf_counter()
            for _ in range(args.steps):  # one batch at a time
                ts = time.perf_counter()
                bres = eng.run(reqs)
                blat.append((time.perf_counter() - ts) * 1e3)
            tb = time.perf_counter() - tb
        plat = []
        tp = time.perf_counter()
        pend = None  # (ticket, submit time): two batches in flight
        for _ in range(args.steps):
            ts = time.perf_counter()
            ticket = eng.submit(reqs)
            if pend:
                eng.collect(pend[0])
                plat.append((time.perf_counter() - pend[1]) * 1e3)
            pend = (ticket, ts)
        eng.collect(pend[0])
        plat.append((time.perf_counter() - pend[1]) * 1e3)
        tp = time.perf_counter() - tp
        bcomp = sum(comparisons_of(r, M) for r in reqs)
        rows = sum(r.n_rot * (2 if r.mirrored else 1) for r in reqs if r.kind == "uniqueness")
        tuned = {str(k): list(v) for k, v in eng.tuned.items()}
        # A planted query is its DB entry rotated by r (4-coefficient blocks);
        # query row 15 - r undoes it, so only requests whose centred rotation
        # window holds that row can find the entry.
        from irisb200.batched import centred_rotations
        planted_hits = sum(1 for j, (e, _) in bpl.items()
                           if reqs[j].kind == "uniqueness" and e in bres[j].matches)
        planted_uniq = sum(1 for j in bpl if reqs[j].kind == "uniqueness")
        planted_window = sum(1 for j, (_, r) in bpl.items()
                             if reqs[j].kind == "uniqueness" and 15 - r in centred_rotations(reqs[j].n_rot))
        eng.close()
        batched = {
            "value": bcomp * args.steps / tb, "unit": UNIT,
            "vs_plain_e2e": (bcomp * args.steps / tb) / e2e_value,
            "latency_ms": {"p50": sorted(blat)[len(blat) // 2], "p99": max(blat)},
            "pipelined": {"value": bcomp * args.steps / tp, "unit": UNIT,
                          "latency_ms": {"p50": sorted(plat)[len(plat) // 2], "p99": max(plat)},
                          "what": "the same batches with two in flight (BatchedEngine.submit / collect: the "
                                  "host prepares batch k+1 while the GPU runs batch k); latency = submit to "
                                  "collect, including the wait for the batch ahead"},
            "config": {"workload": f"batched uneven launches: {nb} requests per batch, rotations 1/16/31, "
                                   "50% mirrored, 80% uniqueness (full DB) / 20% reauth (one target)",
                       "uniqueness_orientations": n_var, "reauth_orientations": n_reauth,
                       "uniqueness_query_rows": rows, "packed_rows": lay.n_rows, "comparisons_per_batch": bcomp,
                       "autotuned_tile_chunk": tuned,
                       "timing": "host wall clock per batch through BatchedEngine.run, one batch at a time "
                                 "(H2D of the shares, graph replay of the DB pass, reauth subset pass, D2H of "
                                 "the match lists)"},
            "planted_matches_found": f"{planted_hits}/{planted_window}",
            "planted_note": f"of the {planted_uniq} planted uniqueness requests, {planted_window} have the "
                            "planted rotation inside their rotation window",
            "clocks": clk.summary(clk.windows[-1]),
        }

    # ---------------- serving leg: continuous batching under Poisson arrivals ----------------
    serving = None
    if reqs and args.serving_rate > 0:
        from irisb200.serving import ContinuousServer
        nq_s = 512
        spl = {j: (int((j * 7919 + 13) % M), (j * 7) % 31 - 15) for j in range(0, nq_s, 10)}
        sqc, sqm = irisb200.synth_queries(DB_SEED + rank, Q_SEED + 2, nq_s, spl)
        app_c, app_m = append_records(ce, me, M)
        srv = ContinuousServer(dm, ce, me, c, chunk=65536, row_capacity=q_cap, max_variants=min(q_cap // 2, 2048),
                               max_reauth=64, threshold_a=A, seeds=seeds, db_capacity=M + 256)
        warm = request_mix(40, sqc, sqm, spl, M, seed=99)
        srv.serve([0.0] * len(warm), warm)
        serving = serve_load(srv, srv, args.serving_rate, 2.0, 0, (sqc, sqm, spl, M, app_c, app_m), clk)
        serving["vs_plain_value"] = serving["comparisons_per_s"] / value
        serving["config"] = {"workload": "continuous serving: Poisson arrivals, 80% uniqueness / 20% reauth, 1% "
                                         "appends, rotations 1/16/31, 50% mirrored, 2 s of arrivals",
                             "row_capacity": q_cap, "chunk": 65536}
        srv.close()
        for e in ce + me:
            e.set_db_len(M)
    cublas_ms = cublas_clk = None
    if rank == 0 and not args.no_cublas:
        cublas_ms, cublas_clk = cublas_limb_gemms(torch, M, NQ * 31, clk=clk)
    clk.__exit__(None, None, None)

    result = None
    if rank == 0:
        ops = 3 * 6 * (K_CODE + K_MASK) * (NQ * 31) * M  # algorithmic int8 ops per batch (all chunks)
        ops_launch = ops * chunks[0][1] / M  # per GEMM launch (one chunk)
        gemm_avg = statistics.mean(gemm_ms)  # per batch = sum over its chunk launches
        achieved = ops / (gemm_avg * 1e-3) / 1e12  # = ops per launch / mean launch duration
        peak = measure_int8_peak(torch)
        traffic = None
        prof = os.path.join(ROOT, "profiles", "gemm_limb_traffic.json")
        if os.path.exists(prof):
            with open(prof) as f:
                pj = json.load(f)
            # the profile's launch covers `entries` DB entries; DRAM bytes grow in
            # proportion to the entries a launch scans (one query-plane re-read per
            # sweep of the SMs over the DB slabs), so scale to this launch
            lg = pj.get("limb_gemm", {})
            if lg.get("dram_bytes_per_launch") and lg.get("entries"):
                traffic = lg["dram_bytes_per_launch"] * chunks[0][1] / lg["entries"]
        lat_sorted = sorted(batch_ms)
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "GPU plain drop-in: 3 parties co-resident on one B200, 64 queries x 31 rotations "
                                   "vs 524288 share-DB entries per party (per GPU)",
                       "db_entries_per_party": M, "queries": NQ, "rotations": 31, "query_rows": NQ * 31,
                       "padded_query_rows": n_rows, "threshold_a": A, "threshold_ratio": 0.375,
                       "l2": "no flush: inputs (60.4 GB share DB) exceed the 126 MB L2",
                       "parallelism": f"db-shard x{world}, 3 co-resident parties per GPU",
                       "db_chunk": chunks[0][1]},
            "latency_ms": {"p50": lat_sorted[len(lat_sorted) // 2], "p99": lat_sorted[-1],
                           "e2e_p50": sorted(lat)[len(lat) // 2], "e2e_p99": max(lat)},
            "kernels_ms": {"limb_gemm_6_engines": gemm_avg, "threshold_open_or": statistics.mean(thr_ms)},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": None, "unit": "TOPS",
                         "frac": None, "traffic": traffic,
                         "kernel": f"limb_gemm_kernel<256> (6 engines, one launch per {chunks[0][1]}-entry "
                                   f"DB chunk, {len(chunks)} per batch)",
                         "ops_per_launch": ops_launch,
                         "peak_source": "2 x measured dense bf16, sustained (MEASURED_PEAKS.json "
                                        "bf16_tflops_sustained; dense int8 issues at twice the bf16 rate on "
                                        "B200): the GEMM is timed over back-to-back steps",
                         "frac_of_burst": None,
                         "cublas_int8_measured_in_run_tops": peak,
                         "frac_of_cublas_int8_in_run": achieved / peak},
            "cublas_limb_gemm_ms_per_batch": cublas_ms,
            "cublas_limb_gemm_clocks": cublas_clk,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": 2 * len(chunks) * args.steps,
            "gpu_launches_e2e": (2 * len(chunks) + 7) * args.steps,
            "clocks": clk.summary(clk.windows[0]),
            "clocks_e2e": clk.summary(clk.windows[1]),
            "planted_matches_found": f"{planted_found}/{len(planted)}",
            "setup_s": {"synth_db": synth_s},
        }
        if batched:
            result["batched"] = batched
        if serving:
            result["serving"] = serving
        mp = measured_peaks()
        rf = result["roofline"]
        if mp["present"]:
            sus, burst = mp["bf16_tflops_sustained"], mp["bf16_tflops"]
            if not sus and burst:  # no sustained figure: the burst one, and say so
                sus = burst
                rf["peak_source"] = "2 x measured dense bf16, burst (MEASURED_PEAKS.json bf16_tflops; no sustained figure)"
            if not sus:
                rf["peak"] = 2 * 1400.0
                rf["frac"] = achieved / rf["peak"]
                rf["peak_source"] = "fallback: 2 x 1.4 PFLOP/s bf16 sustained (MEASURED_PEAKS.json has no bf16 figure)"
            if sus:
                rf["peak"] = 2 * sus
                rf["frac"] = achieved / (2 * sus)
            if burst:
                rf["frac_of_burst"] = achieved / (2 * burst)
        else:  # fallback figure of this GPU pool: 1.4 PFLOP/s bf16 sustained
            rf["peak"] = 2 * 1400.0
            rf["frac"] = achieved / rf["peak"]
            rf["peak_source"] = "fallback: 2 x 1.4 PFLOP/s bf16 sustained (MEASURED_PEAKS.json absent)"
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline()
        print(json.dumps(result), flush=True)

    for o in ce + me + [c, dc]:
        o.close()
    dm.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def _latency_stats(comps, requests, t0, db_lens):
    lat = sorted((c.done - c.arrival) * 1e3 for c in comps if requests[c.idx].kind != "append")
    if not lat:
        return {}
    end = max(c.done for c in comps)
    work = sum(comparisons_of(requests[c.idx], db_lens[c.idx]) for c in comps if requests[c.idx].kind != "append")
    return {"p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
            "max_ms": lat[-1], "mean_ms": statistics.mean(lat), "completed": len(comps),
            "requests_per_s": len(comps) / (end - t0), "comparisons_per_s": work / (end - t0)}


def append_records(ce, me, M, n=64, seed=3):
    """Records for append requests: copies of existing irises (re-enrolments),
    [3][n][K] code and mask shares, fetched before any timing."""
    import numpy as np
    ids = [int(x) for x in np.random.default_rng(seed).integers(0, M, n)]
    c = np.stack([np.stack([ce[p].fetch_records(e, 1)[0] for e in ids]) for p in range(3)])
    m = np.stack([np.stack([me[p].fetch_records(e, 1)[0] for e in ids]) for p in range(3)])
    return c, m


def serve_load(server, stats_src, lam, seconds, seed, pool, clk):
    """One open-loop Poisson run at `lam` requests/s for `seconds` of arrivals
    (80% uniqueness / 20% reauth, 1% appends, rotations 1/16/31, 50% mirrored)
    through server.serve; returns the latency and throughput figures."""
    import numpy as np
    qc, qm, planted, M, app_c, app_m = pool
    rng = np.random.default_rng(1000 + seed)
    n = max(20, int(lam * seconds))
    arrivals = np.cumsum(rng.exponential(1.0 / lam, n)).tolist()
    reqs = request_mix(n, qc, qm, planted, M, seed=2000 + seed, p_append=0.01)
    appends = {i: (app_c[:, i % app_c.shape[1]], app_m[:, i % app_c.shape[1]])
               for i, r in enumerate(reqs) if r.kind == "append"}
    lens, cur = [], server.db_len  # each request's DB scope: the appends that arrived before it
    for r in reqs:
        if r.kind == "append":
            cur += 1
        lens.append(cur)
    stats0 = dict(stats_src.stats) if stats_src else {}
    with clk.mark():
        t0 = time.perf_counter()
        comps = server.serve(arrivals, reqs, appends=appends, max_wall_s=300.0)
    st = _latency_stats(comps, reqs, t0, lens)
    st.update(offered_requests_per_s=lam, requests=n, appends=len(appends),
              reauth=sum(r.kind == "reauth" for r in reqs), clocks=clk.summary(clk.windows[-1]))
    if stats_src:
        d = {k: stats_src.stats[k] - stats0.get(k, 0) for k in stats_src.stats}
        n_st = max(1, d.get("steps", 0))
        st["steps"] = d.get("steps", 0)
        st["mean_rows_per_step"] = d.get("rows", 0) / n_st
        st["mean_used_rows_per_step"] = d.get("used_rows", 0) / n_st
        st["mean_step_interval_ms"] = (max(c.done for c in comps) - t0) * 1e3 / n_st
        st["host_s"] = {k: round(d.get(k, 0.0), 3) for k in ("launch_s", "layout_s", "wait_s")}
    return st


def run_serving(args):
    """Poisson arrivals against the resident 512K-entry DB: the continuous
    server and the plain batch-at-a-time drop-in at each offered load."""
    import numpy as np
    import torch

    import irisb200
    from irisb200.serving import ContinuousServer, PlainBatchServer, plan_row_capacity

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    torch.cuda.set_device(0)
    M, A, chunk = args.db, args.threshold_a, args.chunk
    dm = irisb200.DeviceManager(0)
    seeds = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
    rates = [float(x) for x in args.rates.split(",") if x]
    room = 64 + int(0.011 * max(rates) * args.serve_seconds * 2 * len(rates))
    cap = M + room
    # row capacity from the HBM left once the DB planes are resident (16 GB kept free)
    free, _ = dm.mem_info()
    db_bytes = cap * 3 * (K_CODE + K_MASK) * 2
    R = min(8192, max(2048, ((free - db_bytes - (16 << 30)) // (chunk * 12 + 6 * 4 * K_CODE)) // 64 * 64))
    ce = [irisb200.ShareDB(p, dm, chunk, R, K_CODE, seeds[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, chunk, R, K_MASK, seeds[p]) for p in range(3)]
    for e in ce + me:
        e.alloc_db(cap)
    irisb200.synth_db(ce, me, DB_SEED, 0, M)
    R_plan = plan_row_capacity(dm, chunk)
    c = irisb200.Circuits(dm, seeds)
    nq = 512
    planted = {j: (int((j * 7919 + 13) % M), (j * 7) % 31 - 15) for j in range(0, nq, 10)}
    qc, qm = irisb200.synth_queries(DB_SEED, Q_SEED + 2, nq, planted)
    app_c, app_m = append_records(ce, me, M)
    max_var = min(R // 2, 4096)
    srv = ContinuousServer(dm, ce, me, c, chunk=chunk, row_capacity=R, max_variants=max_var, max_reauth=64,
                           threshold_a=A, seeds=seeds, db_capacity=cap)
    plain = PlainBatchServer(dm, ce, me, c, chunk=chunk, max_slots=64, threshold_a=A, db_capacity=cap)
    # warm both paths (kernels, graphs of nothing, allocator pools)
    warm = request_mix(40, qc, qm, planted, M, seed=99)
    srv.serve([0.0] * len(warm), warm)
    plain.serve([0.0] * len(warm), warm)
    clk = ClockSampler(0).__enter__()
    time.sleep(2.0)
    pool = (qc, qm, planted, M, app_c, app_m)
    sweep = []
    for li, lam in enumerate(rates):
        row = {"offered_requests_per_s": lam}
        arms = [a for a in (("served", srv), ("plain", plain)) if a[0] in args.serving_arms.split(",")]
        for name, server in arms:
            row[name] = serve_load(server, srv if name == "served" else None, lam, args.serve_seconds, li, pool,
                                   clk)
        if "served" in row and "plain" in row:
            row["served_vs_plain_comparisons"] = (row["served"]["comparisons_per_s"] /
                                                  row["plain"]["comparisons_per_s"])
        sweep.append(row)
    clk.__exit__(None, None, None)
    ok = [r for r in sweep if "served" in r and r["served"]["p99_ms"] < 1000]
    okp = [r for r in sweep if "plain" in r and r["plain"]["p99_ms"] < 1000]
    best = max(ok, key=lambda r: r["served"]["comparisons_per_s"]) if ok else None
    bestp = max(okp, key=lambda r: r["plain"]["comparisons_per_s"]) if okp else None
    result = {
        "metric": "iris comparisons/sec (3-party, 1 B200), continuous serving vs plain batch-at-a-time; "
                  "p50/p99 request latency",
        "value": best["served"]["comparisons_per_s"] if best else None, "unit": UNIT, "n_gpus": 1,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "plain_value": bestp["plain"]["comparisons_per_s"] if bestp else None,
        "config": {"workload": f"serving: Poisson arrivals, {M} share-DB entries per party resident, 80% uniqueness "
                               "/ 20% reauth, 1% appends, rotations 1/16/31, 50% mirrored",
                   "row_capacity": R, "row_capacity_planned_from_free_hbm": R_plan, "chunk": chunk,
                   "max_variants": max_var, "threshold_a": A, "serve_seconds": args.serve_seconds,
                   "value_rule": "highest comparisons/s over the offered loads whose p99 latency is below 1 s",
                   "comparison": "one (query orientation, DB entry) pair; a reauth orientation is one comparison",
                   "plain": "batches of up to 64 orientations x 31 rotations, whole DB per batch, FIFO"},
        "sweep": sweep,
    }
    print(json.dumps(result), flush=True)
    srv.close()
    plain.close()
    for o in ce + me + [c]:
        o.close()
    dm.close()


def run_sweep(args):
    """Single-party limb GEMM over query rows x DB entries (K = 12800, as the
    reference's matmul bench) and the 3-party comparison kernel over element
    counts, each against its roofline."""
    import numpy as np
    import torch

    import irisb200

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    dm = irisb200.DeviceManager(0)
    s0 = torch.cuda.ExternalStream(dm.stream(0), device=torch.device("cuda", 0))
    mp = measured_peaks()
    hbm = (mp["hbm_gbs"] or 6650.0) * 1e9
    int8_peak = 2 * (mp["bf16_tflops"] or 1590.0) * 1e12
    peak_source = ("MEASURED_PEAKS.json: 2 x bf16 burst, hbm_gbs" if mp["hbm_gbs"] and mp["bf16_tflops"]
                   else "fallback for missing MEASURED_PEAKS.json figures: 6650 GB/s, 2 x 1590 TFLOP/s bf16 burst")

    def timed(fn, reps):
        fn()
        dm.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s0)
        for _ in range(reps):
            fn()
        b.record(s0)
        b.synchronize()
        return a.elapsed_time(b) / reps

    clk = ClockSampler(0).__enter__()
    time.sleep(2.0)
    gemm = []
    qs, ms = (64, 256, 1024), (262144, 1048576, 2097152)
    seeds = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
    eng = irisb200.ShareDB(0, dm, max(ms), max(qs), K_CODE, seeds[0])
    eng.alloc_db(max(ms))
    eng.fill_random(DB_SEED, max(ms))
    rng = np.random.default_rng(5)
    for q in qs:
        eng.query_upload(rng.integers(0, 65536, (q, K_CODE), dtype=np.uint16))
        for m in ms:
            with clk.mark():
                t = timed(lambda: eng.dot(0, m, 1, dm.stream(0)), 3)
            ops = 6 * K_CODE * q * m
            bound = min(int8_peak, 3 * q * hbm)
            gemm.append({"query_rows": q, "db_entries": m, "ms": t, "tops": ops / t / 1e9,
                         "bound": "hbm" if 3 * q * hbm < int8_peak else "tensor",
                         "frac": ops / (t * 1e-3) / bound, "clocks": clk.summary(clk.windows[-1])})
    eng.close()
    cmp_ = []
    c = irisb200.Circuits(dm, seeds)
    for e in (1 << 20, 1 << 23, 1 << 27, 1 << 30):
        bufs = [irisb200.DeviceBuffer(dm, 2 * e) for _ in range(6)]
        for i, b in enumerate(bufs):
            b.fill_random(1000 + i)
        ra = [irisb200.DeviceBuffer(dm, e // 8) for _ in range(3)]
        rb = [irisb200.DeviceBuffer(dm, e // 8) for _ in range(3)]
        op = irisb200.DeviceBuffer(dm, e // 8)
        with clk.mark():
            t = timed(lambda: c.compare_threshold_masked_many(bufs[:3], bufs[3:], e, 16384, ra, rb, op,
                                                              dm.stream(0)), 3)
        algo = e * 12 + e * 7 // 8  # 3 parties x (code + mask) u16 read; (a, b) bits x 3 + opened bits written
        cmp_.append({"elements": e, "ms": t, "elements_per_s": e / (t * 1e-3), "gbs": algo / t / 1e6,
                     "frac_hbm": algo / (t * 1e-3) / hbm, "bound": "alu (ChaCha12 + bit-sliced circuits)",
                     "clocks": clk.summary(clk.windows[-1])})
        for b in bufs + ra + rb + [op]:
            b.free()
    c.close()
    clk.__exit__(None, None, None)
    print(json.dumps({"metric": "limb GEMM TOPS and comparison elements/s (roofline sweep)", "value": None,
                      "unit": "TOPS", "n_gpus": 1, "data": "synthetic",
                      "config": {"workload": "single-party limb GEMM, K = 12800, query rows x DB entries; "
                                             "3-party compare_threshold_masked_many over element counts",
                                 "int8_peak_tops": int8_peak / 1e12, "hbm_gbs": hbm / 1e9,
                                 "peak_source": peak_source},
                      "gemm": gemm, "comparison": cmp_}), flush=True)
    dm.close()


def run_batched_sweep(args):
    """Config 3 over batch sizes: the same seeded request batches through the
    batched engine (packed rows, graphs, autotuner) and through the plain
    drop-in (every orientation in a 31-rotation slot, 64 slots per batch,
    reauth requests scanned against the whole DB as the plain path does)."""
    import numpy as np
    import torch

    import irisb200
    from irisb200.batched import BatchedEngine, centred_rotations, pack, pad_rows

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    M, A = args.db, args.threshold_a
    sizes = [int(x) for x in args.batch_sizes.split(",") if x]
    seeds = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
    nb = max(sizes)
    pl = {j: (int((j * 104729 + 7) % M), (j * 5) % 31 - 15) for j in range(0, nb, 10)}
    qc, qm = irisb200.synth_queries(DB_SEED, Q_SEED + 1, nb, pl)
    mixes = {b: request_mix(b, qc, qm, pl, M, seed=7 + b) for b in sizes}
    rows = max(-(-pad_rows(pack([list(centred_rotations(r.n_rot)) for r in mixes[b] if r.kind == "uniqueness"
                                  for _ in range(2 if r.mirrored else 1)]), 1 << 20).n_rows // 256) * 256
               for b in sizes)
    q_cap = max(2048, rows)
    dm = irisb200.DeviceManager(0)
    ce = [irisb200.ShareDB(p, dm, M, q_cap, K_CODE, seeds[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, M, q_cap, K_MASK, seeds[p]) for p in range(3)]
    for e in ce + me:
        e.alloc_db(M)
    irisb200.synth_db(ce, me, DB_SEED, 0, M)
    c = irisb200.Circuits(dm, seeds)
    dc = irisb200.DistanceComparator(dm, 64, M)
    clk = ClockSampler(0).__enter__()
    time.sleep(2.0)
    out = []
    for b in sizes:
        reqs = mixes[b]
        n_var = sum(2 if r.mirrored else 1 for r in reqs if r.kind == "uniqueness")
        n_re = sum(2 if r.mirrored else 1 for r in reqs if r.kind == "reauth")
        eng = BatchedEngine(dm, ce, me, c, max_variants=max(64, n_var), max_reauth=max(16, n_re), threshold_a=A,
                            seeds=seeds)
        for _ in range(2):
            eng.run(reqs)
        lat = []
        with clk.mark():
            for _ in range(args.steps):
                t0 = time.perf_counter()
                eng.run(reqs)
                lat.append((time.perf_counter() - t0) * 1e3)
        bclk = clk.summary(clk.windows[-1])
        eng.close()
        comps = sum(comparisons_of(r, M) for r in reqs)
        # the plain drop-in on the same requests: every orientation in a 31-rotation slot
        base_c, base_m = [], []
        for r in reqs:
            for mir in ([False, True] if r.mirrored else [False]):
                base_c.append([irisb200.mirror_query_share(r.code[p], True) if mir else r.code[p] for p in range(3)])
                base_m.append([irisb200.mirror_query_share(r.mask[p], False) if mir else r.mask[p] for p in range(3)])
        bc = np.ascontiguousarray(np.array(base_c, np.uint16).transpose(1, 0, 2))
        bm = np.ascontiguousarray(np.array(base_m, np.uint16).transpose(1, 0, 2))
        for e in ce + me:
            e.use_batch_counter(False)
            e.set_tile(0)
        c.use_batch_counter(False)

        def plain_pass():
            for s0 in range(0, bc.shape[1], 64):
                n = min(64, bc.shape[1] - s0)
                slots = [(j, 0, 31, j) for j in range(n)]
                for p in range(3):
                    ce[p].query_upload_slots(bc[p, s0:s0 + n], slots)
                    me[p].query_upload_slots(bm[p, s0:s0 + n], slots)
                dc.reset()
                irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, M)
                dc.compare_threshold_open(c, ce, me, 0, M, n, A)
                dc.join_db_matches(n, M)
                dc.fetch_final_results(n)
        plain_pass()
        plat = []
        with clk.mark():
            for _ in range(max(1, args.steps // 2)):
                t0 = time.perf_counter()
                plain_pass()
                plat.append((time.perf_counter() - t0) * 1e3)
        pclk = clk.summary(clk.windows[-1])
        lat.sort()
        plat.sort()
        out.append({"requests": b, "uniqueness_orientations": n_var, "reauth_orientations": n_re,
                    "comparisons_per_batch": comps,
                    "batched": {"comparisons_per_s": comps / (statistics.mean(lat) * 1e-3), "p50_ms": lat[len(lat) // 2],
                                "p99_ms": lat[-1], "clocks": bclk},
                    "plain": {"comparisons_per_s": comps / (statistics.mean(plat) * 1e-3),
                              "p50_ms": plat[len(plat) // 2], "p99_ms": plat[-1], "slot_batches": -(-bc.shape[1] // 64),
                              "clocks": pclk}})
        out[-1]["batched_vs_plain"] = out[-1]["batched"]["comparisons_per_s"] / out[-1]["plain"]["comparisons_per_s"]
    clk.__exit__(None, None, None)
    print(json.dumps({"metric": "iris comparisons/sec (3-party, 1 B200) batched vs plain; p50/p99 batch latency",
                      "value": None, "unit": UNIT, "n_gpus": 1, "data": "synthetic",
                      "config": {"workload": f"batched uneven launches over batch sizes, {M} entries per party, "
                                             "rotations 1/16/31, 50% mirrored, 80% uniqueness / 20% reauth",
                                 "timing": "host wall clock per batch, queries uploaded from host memory, "
                                           "match lists returned"},
                      "sizes": out}), flush=True)
    for o in ce + me + [c, dc]:
        o.close()
    dm.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "serving":
        run_serving(args)
    elif args.mode == "sweep":
        run_sweep(args)
    elif args.mode == "batched":
        run_batched_sweep(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
