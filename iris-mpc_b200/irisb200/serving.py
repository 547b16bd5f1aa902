"""Continuous batching over a resident share DB.

The reference's actor takes one batch at a time from its job queue
(iris-mpc-gpu/src/server/actor.rs:584-644) and scans the whole DB for it
(actor.rs:2246-2589).  Here the DB scan is circular and split into chunks:
every step runs the six limb GEMMs and the fused threshold/open/OR for one
chunk and for every query row currently in flight.  A request that arrives
while others are on the GPU is admitted at the next chunk boundary as soon as
its rows fit, so its work overlaps with the requests already scanning; it
completes after it has visited every chunk of the DB as it was when it was
admitted (entries appended later are not part of its result, so a request's
result does not depend on what else is in flight).  Its matches accumulate in
its own bitmap rows (one per orientation), cleared when the rows are reused.

Query rows keep stable positions: each variant (a request's normal or mirrored
orientation) occupies a contiguous run of rows inside one 32-row word, placed
first-fit when it is admitted and freed when it completes.  Its base shares
are written once into the engines' resident base pool (pool index = its
bitmap row); a layout change re-expands the rows from the pool on the device.
The row capacity is planned from free HBM when the server starts.

Reauth requests (one target entry, actor.rs:1465-1475) run on a gathered
subset at the next step boundary.  Append requests write a new record at the
end of the resident DB (write_db_at_index, actor.rs:3547-3600); requests
admitted afterwards scan it.  The device batch counter advances every step
(fresh ChaCha randomness per chunk) without a host round trip.
"""
from __future__ import annotations

import collections
import heapq
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import IRIS_CODE_LENGTH, MASK_CODE_LENGTH, DistanceComparator, ShareDB, dot_many, mirror_query_share
from .batched import MULTS, Request, Result, centred_rotations, pack

RESULT_BYTES_PER_ROW_ENTRY = 2 * 6  # u16 dot share per (row, entry) for 6 engines


def plan_row_capacity(dm, chunk: int, reserve_bytes: int = 8 << 30, cap: int = 8192) -> int:
    """Query rows the server can keep in flight, from the free HBM: each row
    costs a u16 result per chunk entry for the six engines plus its limb
    planes and staging (admission by free HBM)."""
    free, _ = dm.mem_info()
    per_row = chunk * RESULT_BYTES_PER_ROW_ENTRY + 6 * 4 * IRIS_CODE_LENGTH
    rows = max(64, (max(free - reserve_bytes, 0) // per_row) // 64 * 64)
    return int(min(rows, cap))


def split_record_i8(record: np.ndarray):
    """u16 share coefficients -> the stored i8 limb planes (byte - 128) that
    irs_sharedb_load_records_i8 takes."""
    r = np.ascontiguousarray(record, np.uint16)
    lo = ((r & 0xFF).astype(np.uint8) ^ 0x80).view(np.int8)
    hi = ((r >> 8).astype(np.uint8) ^ 0x80).view(np.int8)
    return lo, hi


def _first_run(occupied: int, n: int) -> int:
    """Lowest bit position f with bits f..f+n-1 clear in a 32-bit word, or -1."""
    free = ~occupied & 0xFFFFFFFF
    x = free
    for i in range(1, n):
        x &= free >> i
    if not x:
        return -1
    return (x & -x).bit_length() - 1


@dataclass
class _Variant:
    vid: int                 # bitmap row and base-pool index
    mirrored: bool
    rots: list               # rotation indices (centred)
    slot: int = -1
    first: int = -1


@dataclass
class _Flight:
    req: Request
    idx: int
    arrival: float
    db_len: int              # DB entries as of admission: the request's scope
    variants: list
    needed: set              # chunk indices still to visit


@dataclass
class Completion:
    idx: int
    arrival: float
    done: float
    result: Result


class ContinuousServer:
    """Continuous-batching server over the six resident engines (party p code
    at code_engines[p], mask at mask_engines[p]).  The engines hold the DB
    (alloc_db with room for appends) and must be created with max_db_length
    >= chunk (result rows) and query_length >= row_capacity, with row_capacity
    above max_variants (the base pool shares the query staging)."""

    def __init__(self, dm, code_engines, mask_engines, circuits, chunk: int = 65536, row_capacity: int = 2048,
                 max_variants: int = 512, max_reauth: int = 64, threshold_a: int = 16384, seeds=None,
                 db_capacity: int | None = None):
        if max_variants + 2 > row_capacity:
            raise ValueError("row_capacity must exceed max_variants (base pool and row table share the staging)")
        self.dm = dm
        self.ce, self.me = list(code_engines), list(mask_engines)
        self.c = circuits
        self.A = threshold_a
        self.chunk = max(32, chunk // 32 * 32)
        self.row_capacity = row_capacity // 32 * 32
        self.n_slot_cap = self.row_capacity // 32
        self.slot_occ = [0] * self.n_slot_cap
        self.slot_vars = [[] for _ in range(self.n_slot_cap)]
        self.max_variants = max_variants
        self.db_len = self.ce[0].db_len()
        self.db_capacity = db_capacity or self.db_len
        self.dc = DistanceComparator(dm, max_variants, max(self.db_capacity, 64), match_list_cap=1 << 16)
        self.dc.reset()
        self.free_variants = list(range(max_variants))  # min-heap: low ids keep pool writes contiguous
        self.pending_bases = {}  # vid -> (code [3][12800], mask [3][6400]) not yet in the device pool
        seeds = seeds or [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
        self.max_reauth = max_reauth
        nsub = 2 * max_reauth
        self.sce = [ShareDB(p, dm, nsub, nsub * 32, IRIS_CODE_LENGTH, seeds[p]) for p in range(3)]
        self.sme = [ShareDB(p, dm, nsub, nsub * 32, MASK_CODE_LENGTH, seeds[p]) for p in range(3)]
        for e in self.sce + self.sme:
            e.alloc_db(nsub)
        self.sdc = DistanceComparator(dm, nsub, max(nsub, 64), match_list_cap=1 << 12)
        for e in self.ce + self.me + self.sce + self.sme:
            e.use_batch_counter(True)
        circuits.use_batch_counter(True)
        dm.set_batch_counter(1)
        self.flight = []
        self.layout_dirty = False
        self.next_chunk = 0
        self.steps = 0
        self.rows_active = 0
        self.stats = collections.Counter()  # rows and variants per step, for occupancy reports

    # -- placement -------------------------------------------------------------
    def n_chunks(self, db_len: int | None = None) -> int:
        n = self.db_len if db_len is None else db_len
        return max(1, math.ceil(n / self.chunk))

    def _place(self, n: int):
        for s in range(self.n_slot_cap):
            f = _first_run(self.slot_occ[s], n)
            if f >= 0:
                return s, f
        return None

    def _occupy(self, v: _Variant, s: int, f: int) -> None:
        n = len(v.rots)
        self.slot_occ[s] |= ((1 << n) - 1) << f
        self.slot_vars[s].append(v)
        v.slot, v.first = s, f

    def _release(self, v: _Variant) -> None:
        n = len(v.rots)
        self.slot_occ[v.slot] &= ~(((1 << n) - 1) << v.first) & 0xFFFFFFFF
        self.slot_vars[v.slot].remove(v)

    def can_admit(self, r: Request) -> bool:
        if r.kind != "uniqueness":
            return True
        need_v = 2 if r.mirrored else 1
        if len(self.free_variants) < need_v:
            return False
        placed = []
        ok = True
        for _ in range(need_v):
            where = self._place(r.n_rot)
            if where is None:
                ok = False
                break
            tmp = _Variant(-1, False, [0] * r.n_rot)
            self._occupy(tmp, *where)
            placed.append(tmp)
        for tmp in placed:
            self._release(tmp)
        return ok

    def admit(self, r: Request, idx: int, arrival: float) -> None:
        """Places the request's variants and writes their base shares into
        the resident pool (pool index = bitmap row)."""
        variants = []
        for mir in ([False, True] if r.mirrored else [False]):
            where = self._place(r.n_rot)
            if where is None:
                raise RuntimeError("admit() without room: call can_admit() first")
            v = _Variant(heapq.heappop(self.free_variants), mir, list(centred_rotations(r.n_rot)))
            self._occupy(v, *where)
            variants.append(v)
            code = np.stack([mirror_query_share(r.code[p], True) if mir else r.code[p] for p in range(3)])
            mask = np.stack([mirror_query_share(r.mask[p], False) if mir else r.mask[p] for p in range(3)])
            self.pending_bases[v.vid] = (code, mask)
        f = _Flight(r, idx, arrival, self.db_len, variants, set(range(math.ceil(self.db_len / self.chunk))))
        self.flight.append(f)
        self.layout_dirty = True

    def _layout(self):
        """Row table and segment table of the current placement."""
        used = [s for s in range(self.n_slot_cap) if self.slot_occ[s]]
        n_slots = used[-1] + 1 if used else 1
        row_desc = np.full(n_slots * 32, 0xFFFFFFFF, np.uint32)
        seg_start, seg_query, seg_mask = [0], [], []
        for s in range(n_slots):
            for v in sorted(self.slot_vars[s], key=lambda x: x.first):
                n = len(v.rots)
                row_desc[s * 32 + v.first: s * 32 + v.first + n] = (v.vid << 8) | np.array(v.rots, np.uint32)
                seg_query.append(v.vid)
                seg_mask.append((((1 << n) - 1) << v.first) & 0xFFFFFFFF)
            seg_start.append(len(seg_query))
        return row_desc, np.array(seg_start, np.uint32), np.array(seg_query, np.uint32), np.array(seg_mask, np.uint32)

    def _flush_bases(self) -> None:
        """Writes the newly admitted variants' base shares into the device
        pool, one copy per engine per contiguous run of pool indices."""
        vids = sorted(self.pending_bases)
        runs, start = [], 0
        for i in range(1, len(vids) + 1):
            if i == len(vids) or vids[i] != vids[i - 1] + 1:
                runs.append(vids[start:i])
                start = i
        for run in runs:
            code = np.stack([self.pending_bases[v][0] for v in run], axis=1)  # [3][n][12800]
            mask = np.stack([self.pending_bases[v][1] for v in run], axis=1)
            for p in range(3):
                self.ce[p].query_put_base(run[0], code[p])
                self.me[p].query_put_base(run[0], mask[p])
        self.pending_bases.clear()

    def _upload_layout(self) -> None:
        self._flush_bases()
        row_desc, seg_start, seg_query, seg_mask = self._layout()
        for e in self.ce + self.me:
            e.query_expand_rows(self.max_variants, row_desc)
        self.dc.set_segments(seg_start, seg_query, seg_mask)
        self.rows_active = row_desc.size
        self.layout_dirty = False

    # -- request kinds handled at step boundaries ---------------------------------
    def append(self, code_records: np.ndarray, mask_records: np.ndarray) -> int:
        """Writes one new DB record per party (code [3][12800], mask [3][6400],
        DB-format shares) at the end of the DB; returns its index."""
        idx = self.db_len
        if idx >= self.db_capacity:
            raise ValueError("DB capacity exhausted")
        for p in range(3):
            self.ce[p].load_records_i8(idx, *split_record_i8(code_records[p][None]))
            self.me[p].load_records_i8(idx, *split_record_i8(mask_records[p][None]))
            self.ce[p].set_db_len(idx + 1)
            self.me[p].set_db_len(idx + 1)
        self.db_len = idx + 1
        return idx

    def run_reauth(self, items) -> list:
        """items: [(idx, arrival, Request)] -> [Completion]."""
        for _, _, r in items:
            if not 0 <= r.target < self.db_len:
                raise ValueError(f"reauth target {r.target} is not in the DB")
        variants = [(j, False) for j in range(len(items))] + \
                   [(j, True) for j, (_, _, r) in enumerate(items) if r.mirrored]
        ids = np.array([items[j][2].target for j, _ in variants], np.uint32)
        for p in range(3):
            self.sce[p].gather_records(self.ce[p], ids)
            self.sme[p].gather_records(self.me[p], ids)
        layout = pack([list(centred_rotations(items[j][2].n_rot)) for j, _ in variants])
        bc = np.zeros((3, len(variants), IRIS_CODE_LENGTH), np.uint16)
        bm = np.zeros((3, len(variants), MASK_CODE_LENGTH), np.uint16)
        for v, (j, mir) in enumerate(variants):
            r = items[j][2]
            for p in range(3):
                bc[p, v] = mirror_query_share(r.code[p], True) if mir else r.code[p]
                bm[p, v] = mirror_query_share(r.mask[p], False) if mir else r.mask[p]
        for p in range(3):
            self.sce[p].query_upload_rows(bc[p], layout.row_desc)
            self.sme[p].query_upload_rows(bm[p], layout.row_desc)
        self.dm.advance_batch_counter()
        n = len(variants)
        self.sdc.reset()
        self.sdc.set_segments(layout.seg_start, layout.seg_query, layout.seg_mask)
        dot_many(self.sce + self.sme, MULTS, 0, n)
        self.sdc.compare_threshold_open_prepared(self.c, self.sce, self.sme, 0, n, self.A)
        rows = self.sdc.fetch_rows(0, n, n)
        now = time.perf_counter()
        out = {j: Result() for j in range(len(items))}
        for v, (j, mir) in enumerate(variants):
            hit = bool(rows[v, v])  # variant v against its own target (subset record v)
            if mir:
                out[j].reauth_mirror_match = hit
            else:
                out[j].reauth_match = hit
        return [Completion(items[j][0], items[j][1], now, out[j]) for j in range(len(items))]

    # -- the chunk step -------------------------------------------------------------
    def _finish(self, done: list) -> list:
        """Match lists of the completed requests' bitmap rows (one compaction
        launch per distinct DB snapshot), rows cleared for reuse."""
        tf = time.perf_counter()
        by_len = collections.defaultdict(list)
        for f in done:
            for v in f.variants:
                by_len[f.db_len].append(v)
        hits = {}
        for db_len, vs in by_len.items():
            counts, ids = self.dc.take_rows([v.vid for v in vs], db_len, clear=True)
            for v, n, row in zip(vs, counts, ids):
                hits[v.vid] = row[: min(int(n), len(row))].tolist()
        now = time.perf_counter()
        out = []
        for f in done:
            res = Result()
            for v in f.variants:
                if v.mirrored:
                    res.mirror_matches = hits[v.vid]
                else:
                    res.matches = hits[v.vid]
                self._release(v)
                heapq.heappush(self.free_variants, v.vid)
            out.append(Completion(f.idx, f.arrival, now, res))
        self.layout_dirty = True
        self.stats["finish_s"] += time.perf_counter() - tf
        return out

    def step(self) -> list:
        """One DB chunk for every request in flight; returns completions."""
        empty = [f for f in self.flight if not f.needed]
        if empty:  # admitted against an empty DB
            self.flight = [f for f in self.flight if f.needed]
            return self._finish(empty)
        if not self.flight:
            return []
        if self.layout_dirty:
            tl = time.perf_counter()
            self._upload_layout()
            self.stats["layout_s"] += time.perf_counter() - tl
        k = self.next_chunk % self.n_chunks()
        off = k * self.chunk
        ln = min(self.chunk, self.db_len - off)
        self.dm.advance_batch_counter()
        dot_many(self.ce + self.me, MULTS, off, ln)
        self.dc.compare_threshold_open_prepared(self.c, self.ce, self.me, off, ln, self.A)
        self.steps += 1
        self.stats["steps"] += 1
        self.stats["rows"] += self.rows_active
        self.stats["used_rows"] += sum(bin(x).count("1") for x in self.slot_occ)
        self.stats["entries"] += ln
        self.next_chunk = (k + 1) % self.n_chunks()
        done, keep = [], []
        for f in self.flight:
            f.needed.discard(k)
            (keep if f.needed else done).append(f)
        if not done:
            return []
        self.flight = keep
        return self._finish(done)

    def serve(self, arrivals, requests, appends=None, max_wall_s: float = 600.0, lookahead: int = 256) -> list:
        """Open-loop run: request i arrives at arrivals[i] seconds after start.
        appends: {request index: (code_records, mask_records)} for requests of
        kind "append".  Waiting requests are admitted in arrival order; one
        that does not fit yet is passed by later ones that do (within
        `lookahead` waiting requests), but never by an append, so every
        request sees exactly the appends that arrived before it.  Returns the
        completions (latency = done - arrival)."""
        t0 = time.perf_counter()
        pending = collections.deque(sorted(range(len(requests)), key=lambda i: arrivals[i]))
        waiting = collections.deque()
        completions = []
        total = len(requests)
        while len(completions) < total:
            now = time.perf_counter() - t0
            if now > max_wall_s:
                raise TimeoutError("serving run exceeded its wall-clock budget")
            while pending and arrivals[pending[0]] <= now:
                waiting.append(pending.popleft())
            reauth_items = []
            kept = collections.deque()
            barrier = False
            scanned = 0
            while waiting:
                i = waiting.popleft()
                r = requests[i]
                if barrier or scanned >= lookahead:
                    kept.append(i)
                    continue
                scanned += 1
                if r.kind == "append":
                    if kept:  # earlier requests still wait: the append waits behind them
                        barrier = True
                        kept.append(i)
                        continue
                    code, mask = appends[i]
                    self.append(code, mask)
                    completions.append(Completion(i, t0 + arrivals[i], time.perf_counter(), Result()))
                elif r.kind == "reauth":
                    reauth_items.append((i, t0 + arrivals[i], r))
                elif self.can_admit(r):
                    self.admit(r, i, t0 + arrivals[i])
                else:
                    kept.append(i)
            waiting = kept
            th = time.perf_counter()
            for start in range(0, len(reauth_items), self.max_reauth):
                completions += self.run_reauth(reauth_items[start:start + self.max_reauth])
            ts = time.perf_counter()
            self.stats["reauth_s"] += ts - th
            if self.flight:
                completions += self.step()
                self.stats["step_call_s"] += time.perf_counter() - ts
            elif pending and not waiting:
                time.sleep(max(0.0, min(0.002, arrivals[pending[0]] - (time.perf_counter() - t0))))
        self.dm.synchronize()
        return completions

    def close(self) -> None:
        for o in self.sce + self.sme + [self.dc, self.sdc]:
            o.close()


class PlainBatchServer:
    """The plain drop-in served one batch at a time, as the reference's actor
    does (actor.rs:584-644): the requests that have arrived are taken in
    order, every orientation of every request (reauth included) gets one
    32-row slot with all 31 rotations, the whole DB is scanned chunk by chunk
    for the batch, and all its requests complete together.  A batch holds up
    to `max_slots` orientations (64 in the plain drop-in)."""

    def __init__(self, dm, code_engines, mask_engines, circuits, chunk: int = 65536, max_slots: int = 64,
                 threshold_a: int = 16384, db_capacity: int | None = None):
        self.dm = dm
        self.ce, self.me = list(code_engines), list(mask_engines)
        self.c = circuits
        self.A = threshold_a
        self.chunk = chunk
        self.max_slots = max_slots
        self.db_capacity = db_capacity or self.ce[0].db_len()
        self.dc = DistanceComparator(dm, max_slots, max(self.db_capacity, 64), match_list_cap=1 << 16)
        for e in self.ce + self.me:
            e.use_batch_counter(True)  # fresh ChaCha batch id per chunk from the device counter
        circuits.use_batch_counter(True)
        self.batches = 0

    @property
    def db_len(self) -> int:
        return self.ce[0].db_len()

    def append(self, code_records: np.ndarray, mask_records: np.ndarray) -> int:
        idx = self.db_len
        if idx >= self.db_capacity:
            raise ValueError("DB capacity exhausted")
        for p in range(3):
            self.ce[p].load_records_i8(idx, *split_record_i8(code_records[p][None]))
            self.me[p].load_records_i8(idx, *split_record_i8(mask_records[p][None]))
            self.ce[p].set_db_len(idx + 1)
            self.me[p].set_db_len(idx + 1)
        return idx

    def run_batch(self, items) -> list:
        """items: [(idx, arrival, Request)] of uniqueness/reauth requests."""
        variants = [(j, mir) for j, (_, _, r) in enumerate(items) for mir in ([False, True] if r.mirrored else [False])]
        if len(variants) > self.max_slots:
            raise ValueError("batch exceeds the slot capacity")
        base_c = np.zeros((3, len(variants), IRIS_CODE_LENGTH), np.uint16)
        base_m = np.zeros((3, len(variants), MASK_CODE_LENGTH), np.uint16)
        for v, (j, mir) in enumerate(variants):
            r = items[j][2]
            for p in range(3):
                base_c[p, v] = mirror_query_share(r.code[p], True) if mir else r.code[p]
                base_m[p, v] = mirror_query_share(r.mask[p], False) if mir else r.mask[p]
        slots = [(v, 0, 31, v) for v in range(len(variants))]
        for p in range(3):
            self.ce[p].query_upload_slots(base_c[p], slots)
            self.me[p].query_upload_slots(base_m[p], slots)
        db_len = self.db_len
        self.dc.reset()
        for off in range(0, db_len, self.chunk):
            ln = min(self.chunk, db_len - off)
            self.dm.advance_batch_counter()
            dot_many(self.ce + self.me, MULTS, off, ln)
            self.dc.compare_threshold_open(self.c, self.ce, self.me, off, ln, len(variants), self.A)
        counts, ids = self.dc.take_rows(list(range(len(variants))), db_len, clear=False)
        rows = None
        if any(r.kind == "reauth" for _, _, r in items):
            rows = self.dc.fetch_rows(0, len(variants), db_len)
        now = time.perf_counter()
        out = {j: Result() for j in range(len(items))}
        for v, (j, mir) in enumerate(variants):
            r = items[j][2]
            if r.kind == "reauth":
                hit = bool(rows[v, r.target])
                if mir:
                    out[j].reauth_mirror_match = hit
                else:
                    out[j].reauth_match = hit
            else:
                hits = ids[v, : min(int(counts[v]), ids.shape[1])].tolist()
                if mir:
                    out[j].mirror_matches = hits
                else:
                    out[j].matches = hits
        self.batches += 1
        return [Completion(items[j][0], items[j][1], now, out[j]) for j in range(len(items))]

    def serve(self, arrivals, requests, appends=None, max_wall_s: float = 600.0) -> list:
        """Open-loop run with the arrivals of ContinuousServer.serve."""
        t0 = time.perf_counter()
        order = collections.deque(sorted(range(len(requests)), key=lambda i: arrivals[i]))
        completions = []
        while order:
            now = time.perf_counter() - t0
            if now > max_wall_s:
                raise TimeoutError("serving run exceeded its wall-clock budget")
            if arrivals[order[0]] > now:
                time.sleep(max(0.0, min(0.002, arrivals[order[0]] - now)))
                continue
            items, used = [], 0
            while order and arrivals[order[0]] <= now:
                i = order[0]
                r = requests[i]
                if r.kind == "append":
                    if items:
                        break  # appends take effect between batches, in arrival order
                    order.popleft()
                    code, mask = appends[i]
                    self.append(code, mask)
                    completions.append(Completion(i, t0 + arrivals[i], time.perf_counter(), Result()))
                    continue
                need = 2 if r.mirrored else 1
                if used + need > self.max_slots:
                    break
                order.popleft()
                items.append((i, t0 + arrivals[i], r))
                used += need
            if items:
                completions += self.run_batch(items)
        self.dm.synchronize()
        return completions

    def close(self) -> None:
        self.dc.close()
