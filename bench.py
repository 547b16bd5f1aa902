#!/usr/bin/env python
"""Iris comparisons/sec of the 3-party uniqueness hot path on B200.

Workload (the GPU plain drop-in configuration): 3 parties co-resident on one
GPU, 64 queries x 31 rotations (1984 query rows in 64 slots of 32) against
524,288 share-DB entries per party, threshold ratio 0.375 (A = 16384).  One
step = one batch, the DB scanned in chunks: per chunk the six limb GEMMs (3
parties x code/mask) in one tcgen05 launch, then the fused threshold + open +
rotation OR into the match bitmap.  The chunk length and the GEMM variant
(one-SM, two-SM, or the one-kernel fused scan) are picked on the batch by
irisb200.scan.PlainScan.tune, or fixed with --plain-path / --db-chunk.
One comparison = one (query iris, DB entry) pair over all 31 rotations,
computed jointly by the three parties.

  value -- comparisons/s with the queries already expanded in HBM;
  e2e   -- the same through the public API with host I/O inside every step:
           H2D of the six engines' base query shares from pinned memory,
           device-side rotation expansion, GEMMs, threshold, result merge and
           D2H of the per-query results.

Further legs of the default run, on the same engines and DB (rank 0 of a
1-GPU run): `latency` (200 plain batches after 20 warm-up, each bracketed by
CUDA events), `batched` (100 batches of 256 uneven requests through
BatchedEngine), `serving` (ContinuousServer at 300 / 600 / 1000 requests/s,
5 s of Poisson arrivals each), the cuBLAS limb GEMMs of the reference on the
same shapes, `fused_scan` (the plain batch on the one-kernel fused scan),
and `sweep` (the GEMM and comparison roofline sweep, each row timed for at
least a second with its own clock record).  `cpu_baseline` times the CPU
restatement of the reference's CPU path, `cpu_mpc_simulation` the whole
3-party protocol of the path on the CPU (masked dot shares, threshold
circuit, open, rotation OR), both on bounded samples.  `roofline` is the
limb GEMM's, `roofline_threshold` the threshold kernel's (instruction issue),
`cycles_per_batch` the GEMM's and cuBLAS's device time x sampled SM clock.

The DB (60.4 GB for the three parties) is far larger than L2, so no L2 flush
is needed between steps.  Synthetic seeded data (no dataset exists for this
workload).  `--impl reference` times the CPU restatement of the reference's
CPU path (per-party rotation-aware dots, summed, thresholded, OR over
rotations) on the host cores.

Multi-GPU (torchrun): each rank hosts its own 524,288-entry shard of all three
parties (global entry g on rank g % N) and processes a query batch of the
same shape (the same fresh queries; the planted 10% are near-duplicates of
entries of the rank's own shard); the scan needs no collective (weak
scaling); the end-to-end step merges the ranks' match results with one
all_gather (irisb200.shard); the max step time over ranks is reported.  The
secondary legs (fused scan, latency, batched, serving, sweep, CPU baselines)
run in 1-GPU runs only.
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
                    help="plain step with a fixed --plain-path: DB entries per launch pair (0 = whole DB "
                         "per launch); the tuned path picks its own")
    ap.add_argument("--serving-arms", default="served,plain", help="serving: which servers to run")
    ap.add_argument("--serving-rates-leg", default="300,600,1000",
                    help="default run: offered loads of its serving leg, requests/s (empty = skip)")
    ap.add_argument("--serving-gemm", default="pair", choices=["split", "pair"],
                    help="serving: the DB engines' GEMM (pair = the two-SM kernel where the 256-row tile applies)")
    ap.add_argument("--serving-leg-chunk", type=int, default=32768, help="default run: DB chunk per serving step")
    ap.add_argument("--serving-leg-seconds", type=float, default=5.0,
                    help="default run: seconds of Poisson arrivals per offered load of the serving leg")
    ap.add_argument("--latency-batches", type=int, default=200,
                    help="default run: plain batches timed one by one for the latency percentiles (0 = skip)")
    ap.add_argument("--latency-warmup", type=int, default=20, help="default run: warm-up batches before them")
    ap.add_argument("--batched-batches", type=int, default=100,
                    help="default run: batched-leg batches timed one at a time")
    ap.add_argument("--no-sweep", action="store_true", help="default run: skip the roofline sweep leg")
    ap.add_argument("--no-fused", action="store_true", help="default run: skip the fused-scan leg")
    ap.add_argument("--plain-path", default="tuned", choices=["tuned", "split", "pair", "fused"],
                    help="plain step: DB pass path (tuned = PlainScan.tune picks path and chunk on the batch)")
    ap.add_argument("--sweep-seconds", type=float, default=1.0,
                    help="sweep: minimum timed seconds per row (each row carries its own clock record)")
    return ap.parse_args()


def measured_peaks() -> dict:
    """MEASURED_PEAKS.json at the repository root (a STREAM-style copy and a
    cuBLAS bf16 GEMM measured on this kind of B200) as floats: hbm_gbs,
    bf16_tflops (burst), bf16_tflops_sustained; each None when absent.  A
    value may be a number or {"value": number}."""
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


_CPU_SAMPLES = {}


def _cpu_sample(n_query: int, n_db: int):
    """The seeded CPU sample (oracle module, workload module, DB and query
    shares, rotated query rows), built once per shape."""
    key = (n_query, n_db)
    if key not in _CPU_SAMPLES:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle import oracle as O
        import workload as W
        O.build()
        codes, masks, cs, ms = W.make_db(O, n_db, DB_SEED)
        planted = {j: (int(j * 997 % n_db), (j % 31) - 15) for j in range(0, n_query, 10)}
        qc, qm, _ = W.make_queries(O, n_query, codes, masks, Q_SEED, planted)
        q_code = [W.rotated_rows(O, qc[p]) for p in range(3)]
        q_mask = [W.rotated_rows(O, qm[p]) for p in range(3)]
        _CPU_SAMPLES[key] = (O, W, cs, ms, q_code, q_mask)
    return _CPU_SAMPLES[key]


def cpu_baseline(n_query=8, n_db=8192, min_seconds=10.0):
    """The CPU restatement of the reference's CPU path on config 0's shape."""
    O, W, cs, ms, q_code, q_mask = _cpu_sample(n_query, n_db)
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


def cpu_mpc_simulation(n_query=8, n_db=8192, n_entries=1024, min_seconds=10.0):
    """The full 3-party protocol of the path simulated on the CPU (a secondary
    CPU number beside cpu_baseline): per party the u16 dot shares of 32-row
    query slots (31 rotations + one zero row) against the party's DB shares
    with its zero-share mask (share_db.rs:815-821), the threshold circuit
    with its ChaCha12 randomness (protocol.rs:2519-2546), the open and the OR
    over each slot's 31 rotations; on the first `n_entries` entries of the
    cpu_baseline sample, checked against the plaintext predicate there."""
    import numpy as np
    O, W, cs, ms, q_code, q_mask = _cpu_sample(n_query, n_db)
    q_pad = 32 * n_query

    def slots(rows):
        out = np.zeros((q_pad, rows.shape[1]), np.uint16)
        for j in range(n_query):
            out[32 * j:32 * j + 31] = rows[31 * j:31 * j + 31]
        return out

    qs_code = [slots(q_code[p]) for p in range(3)]
    qs_mask = [slots(q_mask[p]) for p in range(3)]
    db_code = [np.ascontiguousarray(cs[p][:n_entries]) for p in range(3)]
    db_mask = [np.ascontiguousarray(ms[p][:n_entries]) for p in range(3)]
    keys = [W.SEEDS[p][0] for p in range(3)]

    def one_pass(batch):
        code_parts, mask_parts = [], []
        for p in range(3):
            own, prev = W.SEEDS[p]
            d = O.dot_u16(qs_code[p], db_code[p]).T
            code_parts.append(O.mask_dot_shares(d, 0, q_pad, 1, own, prev, O.DOM_CODE_DOT, 0, batch).reshape(-1))
            d = O.dot_u16(qs_mask[p], db_mask[p]).T
            mask_parts.append(O.mask_dot_shares(d, 0, q_pad, 2, own, prev, O.DOM_MASK_DOT, 0, batch).reshape(-1))
        rev = O.threshold_words(code_parts, mask_parts, 16384, keys, dev=0, batch=batch)["revealed"]
        return (rev.reshape(n_entries, n_query) & np.uint32(0x7FFFFFFF)).T != 0

    cores = os.cpu_count() or 1
    reps, t0 = 0, time.perf_counter()
    while True:
        got = one_pass(reps)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or reps >= 200:
            break
    expect = O.cpu_plain_match(q_code, q_mask, n_query, db_code, db_mask, 16384, cores).astype(bool)
    return {"value": reps * n_query * n_entries / el, "unit": UNIT, "cores": cores, "kind": "port",
            "equal_to_plaintext": bool(np.array_equal(got, expect)), "matches": int(got.sum()),
            "sample": f"{n_query} queries x 31 rotations (32-row slots) vs {n_entries} entries, 3 parties: "
                      f"masked dot shares, threshold circuit, open, rotation OR; {reps} pass(es), {el:.1f} s, "
                      f"OpenMP on {cores} threads"}


def pct(values, q: float) -> float:
    """Nearest-rank percentile q (0..100) of a non-empty sample."""
    v = sorted(values)
    k = max(0, min(len(v) - 1, -(-int(round(q * len(v))) // 100) - 1))
    return v[k]


def lat_summary(ms) -> dict:
    return {"n": len(ms), "p50": pct(ms, 50), "p90": pct(ms, 90), "p99": pct(ms, 99), "mean": statistics.mean(ms),
            "max": max(ms)}


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
    from irisb200.scan import PlainScan
    ps = PlainScan(dm, ce, me, c, dc, NQ, M, A)
    chunk = args.db_chunk if 0 < args.db_chunk < M else M

    def scan():
        ps.scan()

    def device_step():
        dc.reset()
        scan()

    clk = ClockSampler(local).__enter__()
    time.sleep(2.0)  # let nvidia-smi initialise before anything is timed
    upload()
    # The DB pass's path and chunk length: tuned on this batch (the library's
    # PlainScan.tune), or fixed by --plain-path / --db-chunk.
    if args.plain_path == "tuned":
        chosen = ps.tune()
    else:
        ps.configure((args.plain_path, 0 if args.plain_path == "fused" else 256, chunk))
        chosen = ps.cand
    chunks = ps.chunks()
    for _ in range(args.warmup):
        device_step()
    dm.synchronize()

    # ---------------- device-resident timing ----------------
    # per-chunk CUDA events of the library's DB pass, on the launching stream:
    # before each chunk, after its GEMM (or fused launch), after its threshold
    ps.set_timing(args.steps)
    begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    dm.synchronize()
    torch.cuda.synchronize()
    with clk.mark():
        begin.record(s0)
        for i in range(args.steps):
            device_step()
        end.record(s0)
        end.synchronize()
    dm.synchronize()
    clk_value = clk.summary(clk.windows[-1])
    total_ms = begin.elapsed_time(end)
    gemm_ms, thr_ms, batch_ms = ps.timings()  # per step, summed over its chunks
    ps.set_timing(0)
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

    # ---------------- fused-scan leg: the same batch, GEMM + threshold in one kernel per chunk ----------------
    fused = None
    if world == 1 and not args.no_fused and n_rows % 128 == 0:
        dcf = irisb200.DistanceComparator(dm, NQ, M, match_list_cap=1 << 16)

        def fused_step():
            dcf.reset()
            for off, ln in chunks:
                dcf.scan_fused(c, ce, me, off, ln, A, n_slots=NQ)
        for _ in range(args.warmup):
            fused_step()
        dm.synchronize()
        fa, fb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with clk.mark():
            fa.record(s0)
            for _ in range(args.steps):
                fused_step()
            fb.record(s0)
            fb.synchronize()
        f_ms = fa.elapsed_time(fb) / args.steps
        f_clk = clk.summary(clk.windows[-1])
        # the fused pass must give the two-launch pass's results on the same batch
        dcf.join_db_matches(NQ, M)
        ff = dcf.fetch_final_results(NQ)
        dc.reset()
        scan()
        dc.join_db_matches(NQ, M)
        fs = dc.fetch_final_results(NQ)
        same = all(np.array_equal(a, b) for a, b in zip(ff, fs))
        dcf.close()
        fused = {"value": comps / (f_ms * 1e-3), "unit": UNIT, "ms_per_batch": f_ms, "vs_value": per_step / f_ms,
                 "results_equal_two_launch_path": bool(same), "clocks": f_clk,
                 "kernel": f"fused_scan_kernel (six limb GEMMs + threshold/open/OR, 128x128 tiles, one launch per "
                           f"{chunks[0][1]}-entry chunk, {len(chunks)} per batch)",
                 "timing": "CUDA events around the timed steps on the launching stream, as for value"}
        if f_clk.get("sm_mhz"):
            fused["cycles_per_batch"] = f_ms * 1e-3 * f_clk["sm_mhz"] * 1e6

    # ---------------- latency leg: batches back to back, each bracketed by CUDA events ----------------
    latency = None
    if world == 1 and args.latency_batches > 0:
        for _ in range(args.latency_warmup):
            device_step()
        dm.synchronize()
        lev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.latency_batches)]
        with clk.mark():
            for a, b in lev:
                a.record(s0)
                device_step()
                b.record(s0)
            lev[-1][1].synchronize()
        lat_b = [a.elapsed_time(b) for a, b in lev]
        latency = lat_summary(lat_b)
        latency.update(warmup=args.latency_warmup, clocks=clk.summary(clk.windows[-1]),
                       comparisons_per_s=comps * len(lat_b) / (sum(lat_b) * 1e-3),
                       rows_x_entries_per_s=NQ * 31 * M * len(lat_b) / (sum(lat_b) * 1e-3),
                       timing="device time of each plain batch (comparator reset, one GEMM + threshold/open/OR "
                              "launch pair per DB chunk of the chosen path, or one fused launch per chunk), CUDA "
                              "events on the launching stream, batches back to back "
                              "after the warm-up; queries resident")

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
    clk_e2e = clk.summary(clk.windows[-1])
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = comps * args.steps / e2e_s

    ps.restore()
    ps.close()
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
        n_bb = max(args.steps, args.batched_batches)
        with clk.mark():
            tb = time.perf_counter()
            for _ in range(n_bb):  # one batch at a time
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
            "value": bcomp * n_bb / tb, "unit": UNIT, "batches": n_bb,
            "vs_plain_e2e": (bcomp * n_bb / tb) / e2e_value,
            "rows_x_entries_per_s": (rows * M + sum(r.n_rot * (2 if r.mirrored else 1) for r in reqs
                                                    if r.kind == "reauth")) * n_bb / tb,
            "latency_ms": lat_summary(blat),
            "pipelined": {"value": bcomp * args.steps / tp, "unit": UNIT, "batches": args.steps,
                          "latency_ms": lat_summary(plat),
                          "what": "the same batches with two in flight (BatchedEngine.submit / collect: the "
                                  "host prepares batch k+1 while the GPU runs batch k); latency = submit to "
                                  "collect, including the wait for the batch ahead"},
            "config": {"workload": f"batched uneven launches: {nb} requests per batch, rotations 1/16/31, "
                                   "50% mirrored, 80% uniqueness (full DB) / 20% reauth (one target)",
                       "uniqueness_orientations": n_var, "reauth_orientations": n_reauth,
                       "uniqueness_query_rows": rows, "packed_rows": lay.n_rows, "comparisons_per_batch": bcomp,
                       "autotuned_tile_chunk": tuned,
                       "autotune_ms_per_pass": {str(k): [[list(cd), round(ms, 1)] for cd, ms in v]
                                                for k, v in eng.tune_log.items()},
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
    rates = [float(x) for x in args.serving_rates_leg.split(",") if x]
    if reqs and rates:
        from irisb200.serving import ContinuousServer
        nq_s = 512
        spl = {j: (int((j * 7919 + 13) % M), (j * 7) % 31 - 15) for j in range(0, nq_s, 10)}
        sqc, sqm = irisb200.synth_queries(DB_SEED + rank, Q_SEED + 2, nq_s, spl)
        app_c, app_m = append_records(ce, me, M)
        srv = ContinuousServer(dm, ce, me, c, chunk=args.serving_leg_chunk, row_capacity=q_cap,
                               max_variants=min(q_cap // 2, 2048), max_reauth=64, threshold_a=A, seeds=seeds,
                               db_capacity=M + 256, gemm_pair=args.serving_gemm == "pair")
        warm = request_mix(40, sqc, sqm, spl, M, seed=99)
        srv.serve([0.0] * len(warm), warm)
        loads = []
        for li, lam in enumerate(rates):
            st = serve_load(srv, srv, lam, args.serving_leg_seconds, li, (sqc, sqm, spl, M, app_c, app_m), clk)
            st["vs_plain_value"] = st["comparisons_per_s"] / value
            st["rows_x_entries_per_s"] = (st["mean_used_rows_per_step"] * args.serving_leg_chunk /
                                          (st["mean_step_interval_ms"] * 1e-3))
            loads.append(st)
        under = [x for x in loads if x["p99_ms"] < 1000.0]
        over = [x for x in loads if x["p99_ms"] >= 1000.0]
        serving = {
            "loads": loads,
            "saturation_requests_per_s": max(x["requests_per_s"] for x in loads),
            "p99_below_1s_up_to_offered": max((x["offered_requests_per_s"] for x in under), default=None),
            "p99_above_1s_from_offered": min((x["offered_requests_per_s"] for x in over), default=None),
            "config": {"workload": "continuous serving: Poisson arrivals, 80% uniqueness / 20% reauth, 1% appends, "
                                   f"rotations 1/16/31, 50% mirrored, {args.serving_leg_seconds:g} s of arrivals per "
                                   "offered load",
                       "row_capacity": q_cap, "chunk": args.serving_leg_chunk, "gemm": args.serving_gemm,
                       "saturation": "the highest completed requests/s over the offered loads (a request counts "
                                     "from its arrival to its completion; the rate runs to the last completion)"},
        }
        srv.close()
        for e in ce + me:
            e.set_db_len(M)
    cublas_ms = cublas_clk = None
    if rank == 0 and not args.no_cublas:
        cublas_ms, cublas_clk = cublas_limb_gemms(torch, M, NQ * 31, clk=clk)
    peak = measure_int8_peak(torch) if rank == 0 else None
    # the 3-party DB is freed before the sweep's single-party DBs are built
    for o in ce + me + [c, dc]:
        o.close()
    sweep = None
    if rank == 0 and world == 1 and not args.no_sweep:
        sweep = sweep_leg(dm, clk, args.sweep_seconds)
    clk.__exit__(None, None, None)

    result = None
    if rank == 0:
        ops = 3 * 6 * (K_CODE + K_MASK) * (NQ * 31) * M  # algorithmic int8 ops per batch (all chunks)
        ops_launch = ops * chunks[0][1] / M  # per GEMM launch (one chunk)
        gemm_avg = statistics.mean(gemm_ms)  # per batch = sum over its chunk launches
        achieved = ops / (gemm_avg * 1e-3) / 1e12  # = ops per launch / mean launch duration
        traffic = traffic_source = None
        # algorithmic DRAM bytes of one launch: the six engines' DB limb planes
        # once, their query planes once, the u16 dot shares written
        alg_bytes = (chunks[0][1] * 3 * 2 * (K_CODE + K_MASK) + 3 * n_rows * (K_CODE + K_MASK) * 2
                     + chunks[0][1] * n_rows * 2 * 6)
        prof = os.path.join(ROOT, "profiles", "gemm_limb_traffic.json")
        if os.path.exists(prof):
            with open(prof) as f:
                pj = json.load(f)
            # a capture of this launch's own chunk length when the profile has
            # one; else the path's capture scaled by the entries a launch scans
            # (an estimate: the query planes' share of the bytes changes with it)
            key = {"split": "limb_gemm", "pair": "limb_gemm_pair", "fused": "fused_scan"}[chosen[0]]
            own = pj.get(key + "_by_chunk", {}).get(str(chunks[0][1]), {})
            lg = pj.get(key, {})
            if own.get("dram_bytes_per_launch"):
                traffic = own["dram_bytes_per_launch"]
                traffic_source = f"ncu capture of a {chunks[0][1]}-entry launch (profiles/gemm_limb_traffic.json)"
            elif lg.get("dram_bytes_per_launch") and lg.get("entries"):
                traffic = lg["dram_bytes_per_launch"] * chunks[0][1] / lg["entries"]
                traffic_source = (f"ncu capture of a {lg['entries']}-entry launch scaled to {chunks[0][1]} entries "
                                  "(profiles/gemm_limb_traffic.json)")
        thr_avg = statistics.mean(thr_ms)
        mhz = clk_value.get("sm_mhz")
        n_sm = dm.sm_count()
        cycles = {"limb_gemm_6_engines": gemm_avg * 1e-3 * mhz * 1e6 if mhz else None,
                  "limb_gemm_sm_mhz": mhz,
                  "cublas_limb_gemms": (cublas_ms * 1e-3 * cublas_clk["sm_mhz"] * 1e6
                                        if cublas_ms and cublas_clk and cublas_clk.get("sm_mhz") else None),
                  "cublas_sm_mhz": cublas_clk.get("sm_mhz") if cublas_clk else None,
                  "how": "CUDA-event time per batch x the median SM clock sampled during that leg "
                         "(both arms run under the 1000 W power cap)"}
        if cycles["limb_gemm_6_engines"] and cycles["cublas_limb_gemms"]:
            cycles["fused_over_cublas"] = cycles["limb_gemm_6_engines"] / cycles["cublas_limb_gemms"]
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
                       "db_chunk": chunks[0][1], "db_pass_path": chosen[0],
                       "db_pass_choice": ("PlainScan.tune on the batch, ms per pass (first round, then the "
                                          "finalists' means over the interleaved rounds): "
                                          + "; ".join(f"{p}/{t}/{ch}: {ms:.1f}" for (p, t, ch), ms in ps.tune_log))
                                         if ps.tune_log else "fixed (--plain-path)"},
            "latency_ms": {"p50": pct(batch_ms, 50), "p99": pct(batch_ms, 99), "of": f"the {args.steps} timed steps",
                           "e2e_p50": pct(lat, 50), "e2e_p99": pct(lat, 99)},
            "kernels_ms": {"limb_gemm_6_engines": gemm_avg, "threshold_open_or": thr_avg},
            "cycles_per_batch": cycles,
            "rows_x_entries_per_s": NQ * 31 * M * world / (per_step * 1e-3),
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": None, "unit": "TOPS",
                         "frac": None, "traffic": traffic, "traffic_source": traffic_source,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel": {"split": "limb_gemm_kernel<256>", "pair": "limb_gemm_pair_kernel (cta_group::2)",
                                    "fused": "fused_scan_kernel (GEMM and threshold: time includes the threshold)"}
                                   [chosen[0]] + f" (6 engines, one launch per {chunks[0][1]}-entry DB chunk, "
                                   f"{len(chunks)} per batch)",
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
            "gpu_launches": (1 if chosen[0] == "fused" else 2) * len(chunks) * args.steps,
            "gpu_launches_e2e": ((1 if chosen[0] == "fused" else 2) * len(chunks) + 7) * args.steps,
            "clocks": clk_value,
            "clocks_e2e": clk_e2e,
            "planted_matches_found": f"{planted_found}/{len(planted)}",
            "setup_s": {"synth_db": synth_s},
        }
        result["roofline_threshold"] = threshold_roofline(thr_avg, M * NQ, n_sm, mhz, chunks)
        if fused:
            result["fused_scan"] = fused
        if latency:
            result["latency"] = latency
        if batched:
            result["batched"] = batched
        if serving:
            result["serving"] = serving
        if sweep:
            result["sweep"] = sweep
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
        else:  # fallback: 1.4 PFLOP/s bf16 sustained, measured earlier on B200s at the 1000 W cap
            rf["peak"] = 2 * 1400.0
            rf["frac"] = achieved / rf["peak"]
            rf["peak_source"] = "fallback: 2 x 1.4 PFLOP/s bf16 sustained (MEASURED_PEAKS.json absent)"
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline()
            result["cpu_mpc_simulation"] = cpu_mpc_simulation()
        print(json.dumps(result), flush=True)

    dm.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def threshold_roofline(thr_ms: float, words: int, n_sm: int, sm_mhz, chunks) -> dict:
    """Roofline of the fused threshold kernel per batch.  It is bound by its
    integer instruction issue (ChaCha12 and the bit-sliced adders), not by
    HBM: one thread evaluates one 32-element word, so the thread instructions
    per word come from an ncu count of the same kernel
    (profiles/threshold_bitmap_counters.json, smsp__inst_executed per warp),
    and the ceiling is one warp instruction per SM sub-partition per clock:
    SMs x 4 x 32 lanes x the SM clock sampled during the timed steps.  The HBM
    fraction (its 6 x 64 bytes of dot shares read per word) is given beside."""
    out = {"bound": "alu", "unit": "thread instructions/s", "words_per_batch": words,
           "words_per_s": words / (thr_ms * 1e-3), "ms_per_batch": thr_ms,
           "kernel": f"threshold_bitmap_kernel<128, 3> ({len(chunks)} launches per batch)",
           "achieved": None, "peak": None, "frac": None, "inst_per_word": None}
    prof = os.path.join(ROOT, "profiles", "threshold_bitmap_counters.json")
    if os.path.exists(prof):
        with open(prof) as f:
            pj = json.load(f)
        ipw = pj.get("inst_per_word")
        out["inst_per_word"] = ipw
        out["counters_source"] = pj.get("source")
        if pj.get("alu_pipe_pct") is not None:
            # the binding pipe: the integer ALU pipe is busier than the issue
            # slots (87.5% against 71.3% in the capture), so it sets the limit
            out["binding_pipe"] = {"pipe": "alu", "frac": pj["alu_pipe_pct"] / 100.0,
                                   "issue_frac": pj.get("issue_active_pct", 0.0) / 100.0,
                                   "source": "ncu sm__inst_executed_pipe_alu (pct of peak sustained active), "
                                             "small case of the same kernel, profiles/threshold_bitmap_16k_full.md"}
        if ipw:
            out["achieved"] = ipw * words / (thr_ms * 1e-3)
    if sm_mhz:
        out["peak"] = n_sm * 4 * 32 * sm_mhz * 1e6
        out["peak_source"] = f"{n_sm} SMs x 4 sub-partitions x 32 lanes x {sm_mhz:.0f} MHz (median sampled clock)"
        if out["achieved"]:
            out["frac"] = out["achieved"] / out["peak"]
    hbm = measured_peaks()["hbm_gbs"] or 6650.0
    out["hbm_bytes_per_batch"] = words * 6 * 64
    out["hbm_gbs"] = words * 6 * 64 / (thr_ms * 1e-3) / 1e9
    out["frac_hbm"] = out["hbm_gbs"] / hbm
    return out


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
                           threshold_a=A, seeds=seeds, db_capacity=cap, gemm_pair=args.serving_gemm == "pair")
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
                   "gemm": args.serving_gemm,
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


def sweep_leg(dm, clk, min_s: float = 1.0) -> dict:
    """The GEMM / comparison roofline sweep (configuration 2), each row timed
    with CUDA events over at least `min_s` seconds of back-to-back launches so
    that it carries its own clock record.

    GEMM: one party's code engine (K = 12800, no zero-share mask: the
    reference's matmul bench engine has no comms) over query rows Q x DB
    entries M, Q in {64, 256, 1024} x M in {256K, 1M, 2M} at the library's
    tile, the other tile width at 1M entries for Q = 256 and 1024, and the
    reference bench's job (iris-mpc-gpu/benches/matmul.rs:17-20: 8 x 300,000
    entries x 930 rows, spread over 8 GPUs there) on one GPU; the two-SM
    (cta_group::2) kernel at 1M entries for Q = 256 and 1024.  Bound: streaming
    the DB (3 Q int8 ops per DB byte at the measured HBM bandwidth) or 2 x the
    measured dense bf16 burst peak (int8 issues at twice the bf16 rate),
    whichever is lower.

    Comparison: compare_threshold_masked_many (flat) over 2^20, 2^25 and 2^30
    elements of three parties' u16 code and mask shares."""
    import numpy as np
    import torch

    import irisb200

    s0 = torch.cuda.ExternalStream(dm.stream(0), device=torch.device("cuda", dm.device))
    mp = measured_peaks()
    hbm = (mp["hbm_gbs"] or 6650.0) * 1e9
    int8_peak = 2 * (mp["bf16_tflops"] or 1590.0) * 1e12
    peak_source = ("MEASURED_PEAKS.json: 2 x bf16 burst (bf16_tflops), hbm_gbs" if mp["hbm_gbs"] and mp["bf16_tflops"]
                   else "fallback for missing MEASURED_PEAKS.json figures: 6650 GB/s, 2 x 1590 TFLOP/s bf16 burst")

    def timed(fn):
        """(ms per launch, launches, clock record) over >= min_s seconds."""
        fn()
        dm.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s0)
        fn()
        b.record(s0)
        b.synchronize()
        est = max(a.elapsed_time(b), 1e-3)
        reps = max(3, int(min_s * 1e3 / est) + 1)
        with clk.mark():
            a.record(s0)
            for _ in range(reps):
                fn()
            b.record(s0)
            b.synchronize()
        return a.elapsed_time(b) / reps, reps, clk.summary(clk.windows[-1])

    seeds = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
    K256, K1M, K2M, KREF = 262144, 1048576, 2097152, 2400000
    rows_plan = [(q, m, 0) for q in (64, 256, 1024) for m in (K256, K1M, K2M)]
    rows_plan += [(256, K1M, 256), (1024, K1M, 128), (256, K1M, "pair"), (1024, K1M, "pair"), (930, KREF, 0)]
    eng = irisb200.ShareDB(0, dm, KREF, 1024, K_CODE, seeds[0], is_remote=False)
    gemm = []
    try:
        eng.alloc_db(KREF)
        eng.fill_random(DB_SEED, KREF)
        rng = np.random.default_rng(5)
        cur_q = None
        for q, m, tile in sorted(rows_plan, key=lambda r: (r[0], str(r[2]), r[1])):
            if q != cur_q:
                eng.query_upload(rng.integers(0, 65536, (q, K_CODE), dtype=np.uint16))
                cur_q = q
            eng.set_pair(tile == "pair")  # the two-SM kernel on the 256-row tile
            eng.set_tile(256 if tile == "pair" else tile)
            t, reps, ck = timed(lambda: eng.dot(0, m, 1, dm.stream(0)))
            ops = 6 * K_CODE * q * m
            hbm_bound = 3 * q * hbm
            bound = min(int8_peak, hbm_bound)
            row = {"query_rows": q, "db_entries": m, "tile": tile or "auto", "ms": t, "launches": reps,
                   "tops": ops / t / 1e9, "comparisons_per_s": m * q / 31 / (t * 1e-3),
                   "bound": "hbm" if hbm_bound < int8_peak else "tensor", "bound_tops": bound / 1e12,
                   "frac": ops / (t * 1e-3) / bound, "clocks": ck}
            if ck.get("sm_mhz"):
                row["ops_per_sm_cycle"] = ops / (t * 1e-3) / (ck["sm_mhz"] * 1e6) / dm.sm_count()
            if (q, m) == (930, KREF):
                row["what"] = ("the reference matmul bench's job (2.4M entries x 930 rows x 12800) on one GPU; "
                               "the reference spreads it over 8 GPUs (300,000 entries each)")
            gemm.append(row)
        eng.set_pair(False)
        eng.set_tile(0)
    finally:
        eng.close()

    cmp_ = []
    c = irisb200.Circuits(dm, seeds)
    try:
        for e in (1 << 20, 1 << 25, 1 << 30):
            bufs = [irisb200.DeviceBuffer(dm, 2 * e) for _ in range(6)]
            ra = [irisb200.DeviceBuffer(dm, e // 8) for _ in range(3)]
            rb = [irisb200.DeviceBuffer(dm, e // 8) for _ in range(3)]
            op = irisb200.DeviceBuffer(dm, e // 8)
            try:
                for i, b in enumerate(bufs):
                    b.fill_random(1000 + i)
                t, reps, ck = timed(lambda: c.compare_threshold_masked_many(bufs[:3], bufs[3:], e, 16384, ra, rb, op,
                                                                            dm.stream(0)))
            finally:
                for b in bufs + ra + rb + [op]:
                    b.free()
            algo = e * 12 + e * 7 // 8  # 3 parties x (code + mask) u16 read; (a, b) bits x 3 + opened bits written
            cmp_.append({"elements": e, "ms": t, "launches": reps, "elements_per_s": e / (t * 1e-3),
                         "gbs": algo / t / 1e6, "frac_hbm": algo / (t * 1e-3) / hbm,
                         "bound": "alu (ChaCha12 + bit-sliced circuits)", "clocks": ck})
    finally:
        c.close()
    return {"gemm": gemm, "comparison": cmp_,
            "config": {"workload": "configuration 2: single-party limb GEMM (K = 12800) over query rows x DB "
                                   "entries; 3-party compare_threshold_masked_many over element counts",
                       "int8_peak_tops": int8_peak / 1e12, "hbm_gbs": hbm / 1e9, "peak_source": peak_source,
                       "min_seconds_per_row": min_s,
                       "timing": "CUDA events around back-to-back launches on the launching stream; the DB "
                                 "(6.7-61 GB) exceeds L2, so no flush"}}


def run_sweep(args):
    """The roofline sweep alone (sweep_leg) as one JSON line."""
    import torch

    import irisb200

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    dm = irisb200.DeviceManager(0)
    clk = ClockSampler(0).__enter__()
    time.sleep(2.0)
    try:
        sw = sweep_leg(dm, clk, args.sweep_seconds)
    finally:
        clk.__exit__(None, None, None)
    print(json.dumps({"metric": "limb GEMM TOPS and comparison elements/s (roofline sweep)", "value": None,
                      "unit": "TOPS", "n_gpus": 1, "data": "synthetic", **sw}), flush=True)
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
