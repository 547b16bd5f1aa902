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

from . import (IRIS_CODE_LENGTH, MASK_CODE_LENGTH, MAX_MATCHES_LEN, DistanceComparator, Event, IrisError,
               PinnedArray, ShareDB, dot_many, mirror_query_share)
from .batched import MULTS, Request, Result, attach_bases, centred_rotations, pack, padded_rows

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
    above max_variants (the base pool shares the query staging).

    serve() runs the device work one step ahead of the host: step k+1 (its
    uploads, GEMMs, threshold and the match-list compaction of the requests
    that finish with it) is enqueued before the host waits for step k's
    results, with the library in its asynchronous host mode and every host
    buffer it reads or writes page-locked and double-buffered."""

    def __init__(self, dm, code_engines, mask_engines, circuits, chunk: int = 32768, row_capacity: int = 2048,
                 max_variants: int = 512, max_reauth: int = 64, threshold_a: int = 16384, seeds=None,
                 db_capacity: int | None = None, gemm_pair: bool = True):
        if max_variants + 2 > row_capacity:
            raise ValueError("row_capacity must exceed max_variants (base pool and row table share the staging)")
        self.dm = dm
        self.ce, self.me = list(code_engines), list(mask_engines)
        # the DB engines' GEMM: the two-SM kernel where the 256-row tile applies
        # (irs_sharedb_set_pair); close() restores the library's default.  The
        # defaults (two-SM GEMM, 32,768-entry steps) are the measured best of
        # the server on 524,288 entries: higher saturation and lower p99 than
        # the one-SM GEMM or 65,536-entry steps, and higher saturation than
        # 16,384- or 8,192-entry steps
        for e in self.ce + self.me:
            e.set_pair(gemm_pair)
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
        self.pending_bases = set()  # pool indices written on the host, not yet copied to the device pool
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
        self._alloc_host(nsub)
        self.flight = []
        self.layout_dirty = False
        self.next_chunk = 0
        self.steps = 0
        self.rows_active = 0
        self.stats = collections.Counter()  # rows and variants per step, for occupancy reports

    def _alloc_host(self, nsub: int) -> None:
        """Page-locked host buffers: the base-query pool mirror (one slot per
        pool index, written once per admission) and two sets (one per step in
        flight) of row tables, segment tables, compaction outputs and reauth
        staging."""
        V, R = self.max_variants, self.row_capacity
        P = PinnedArray
        self.h_pool_c = P((3, V, IRIS_CODE_LENGTH), np.uint16)
        self.h_pool_m = P((3, V, MASK_CODE_LENGTH), np.uint16)
        self.h_rows = [P((R,), np.uint32) for _ in range(2)]
        self.h_seg = [(P((self.n_slot_cap + 1,), np.uint32), P((R,), np.uint32), P((R,), np.uint32))
                      for _ in range(2)]
        self.h_take = [(P((V,), np.uint32), P((V,), np.uint32), P((V, MAX_MATCHES_LEN), np.uint32))
                       for _ in range(2)]
        self.h_r_ids = [P((nsub,), np.uint32) for _ in range(2)]
        self.h_r_base = [(P((3, nsub, IRIS_CODE_LENGTH), np.uint16), P((3, nsub, MASK_CODE_LENGTH), np.uint16))
                         for _ in range(2)]
        self.h_r_rows = [P((nsub * 32,), np.uint32) for _ in range(2)]
        self.h_r_seg = [(P((nsub + 1,), np.uint32), P((nsub * 32,), np.uint32), P((nsub * 32,), np.uint32))
                        for _ in range(2)]
        self.h_r_take = [(P((nsub,), np.uint32), P((nsub,), np.uint32), P((nsub, MAX_MATCHES_LEN), np.uint32))
                         for _ in range(2)]
        self.events = [Event(), Event()]
        self.par = 0
        # pool indices of completed variants, reusable once their step's event has
        # completed (a pinned pool slot may still be read by a queued copy before)
        self.cooling = [[], []]

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
        the host copy of the pool (pool index = bitmap row); the next step
        copies them to the device.  A mirrored variant's slot holds the plain
        share: its rows carry the mirror bit and the device mirrors them."""
        variants = []
        for mir in ([False, True] if r.mirrored else [False]):
            where = self._place(r.n_rot)
            if where is None:
                raise RuntimeError("admit() without room: call can_admit() first")
            v = _Variant(heapq.heappop(self.free_variants), mir, list(centred_rotations(r.n_rot)))
            self._occupy(v, *where)
            variants.append(v)
            for p in range(3):
                self.h_pool_c.array[p, v.vid] = r.code[p]
                self.h_pool_m.array[p, v.vid] = r.mask[p]
            self.pending_bases.add(v.vid)
        f = _Flight(r, idx, arrival, self.db_len, variants, set(range(math.ceil(self.db_len / self.chunk))))
        self.flight.append(f)
        self.layout_dirty = True

    def _layout(self):
        """Row table and segment table of the current placement."""
        used = [s for s in range(self.n_slot_cap) if self.slot_occ[s]]
        n_slots = used[-1] + 1 if used else 1
        # empty rows pad the table for the GEMM's widest tile (padded_rows); the
        # threshold kernel only visits the slots that carry segments
        n_rows = min(padded_rows(n_slots * 32, self.row_capacity), self.row_capacity)
        row_desc = np.full(n_rows, 0xFFFFFFFF, np.uint32)
        seg_start, seg_query, seg_mask = [0], [], []
        for s in range(n_slots):
            for v in sorted(self.slot_vars[s], key=lambda x: x.first):
                n = len(v.rots)
                row_desc[s * 32 + v.first: s * 32 + v.first + n] = \
                    (v.vid << 8) | (0x80 if v.mirrored else 0) | np.array(v.rots, np.uint32)
                seg_query.append(v.vid)
                seg_mask.append((((1 << n) - 1) << v.first) & 0xFFFFFFFF)
            seg_start.append(len(seg_query))
        return row_desc, np.array(seg_start, np.uint32), np.array(seg_query, np.uint32), np.array(seg_mask, np.uint32)

    def _flush_bases(self) -> None:
        """Copies the newly admitted variants' base shares from the pinned
        host pool into the device pool, one copy per engine per contiguous
        run of pool indices."""
        vids = sorted(self.pending_bases)
        start = 0
        for i in range(1, len(vids) + 1):
            if i == len(vids) or vids[i] != vids[i - 1] + 1:
                a, n = vids[start], i - start
                for p in range(3):
                    self.ce[p].query_put_base(a, self.h_pool_c.array[p, a:a + n])
                    self.me[p].query_put_base(a, self.h_pool_m.array[p, a:a + n])
                start = i
        self.pending_bases.clear()

    def _upload_layout(self) -> None:
        self._flush_bases()
        row_desc, seg_start, seg_query, seg_mask = self._layout()
        rt = self.h_rows[self.par].array[: row_desc.size]
        rt[:] = row_desc
        ss, sq, sm = (x.array for x in self.h_seg[self.par])
        ss[: seg_start.size] = seg_start
        sq[: seg_query.size] = seg_query
        sm[: seg_mask.size] = seg_mask
        for e in self.ce + self.me:
            e.query_expand_rows(self.max_variants, rt)
        self.dc.set_segments(ss[: seg_start.size], sq[: seg_query.size], sm[: seg_mask.size])
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

    def _launch_reauth(self, items):
        """Enqueues one reauth batch (items: [(idx, arrival, Request)]) on the
        gathered subset; returns the handler that turns its compacted rows
        into completions once the step's event has completed."""
        for _, _, r in items:
            if not 0 <= r.target < self.db_len:
                raise ValueError(f"reauth target {r.target} is not in the DB")
        par = self.par
        variants = [(j, False) for j in range(len(items))] + \
                   [(j, True) for j, (_, _, r) in enumerate(items) if r.mirrored]
        n = len(variants)
        ids = self.h_r_ids[par].array[:n]
        ids[:] = [items[j][2].target for j, _ in variants]
        for p in range(3):
            self.sce[p].gather_records(self.ce[p], ids)
            self.sme[p].gather_records(self.me[p], ids)
        layout = attach_bases(pack([list(centred_rotations(items[j][2].n_rot)) for j, _ in variants]),
                              range(n), [mir for _, mir in variants])
        bc, bm = (x.array for x in self.h_r_base[par])
        for v, (j, _) in enumerate(variants):
            r = items[j][2]
            for p in range(3):
                bc[p, v] = r.code[p]
                bm[p, v] = r.mask[p]
        rt = self.h_r_rows[par].array[: layout.n_rows]
        rt[:] = layout.row_desc
        for p in range(3):
            self.sce[p].query_upload_rows(bc[p, :n], rt)
            self.sme[p].query_upload_rows(bm[p, :n], rt)
        ss, sq, sm = (x.array for x in self.h_r_seg[par])
        ns, nq = layout.seg_start.size, layout.seg_query.size
        ss[:ns], sq[:nq], sm[:nq] = layout.seg_start, layout.seg_query, layout.seg_mask
        self.dm.advance_batch_counter()
        self.sdc.reset()
        self.sdc.set_segments(ss[:ns], sq[:nq], sm[:nq])
        dot_many(self.sce + self.sme, MULTS, 0, n)
        self.sdc.compare_threshold_open_prepared(self.c, self.sce, self.sme, 0, n, self.A)
        rows, counts, tids = (x.array for x in self.h_r_take[par])
        rows[:n] = np.arange(n, dtype=np.uint32)
        self.sdc.take_rows_into(rows[:n], n, counts, tids, clear=True)

        def handler(now):
            out = {j: Result() for j in range(len(items))}
            for v, (j, mir) in enumerate(variants):
                hit = v in tids[v, : min(int(counts[v]), MAX_MATCHES_LEN)]  # against its own target (record v)
                if mir:
                    out[j].reauth_mirror_match = bool(hit)
                else:
                    out[j].reauth_match = bool(hit)
            return [Completion(items[j][0], items[j][1], now, out[j]) for j in range(len(items))]
        return handler

    # -- the chunk step -------------------------------------------------------------
    def _launch_step(self):
        """Enqueues one DB chunk for every request in flight and the match
        compaction of the requests it completes (their rows are released on
        the host at once: every later use of those rows is ordered after the
        compaction on the device).  Returns the completion handler or None."""
        empty = [f for f in self.flight if not f.needed]  # admitted against an empty DB
        if not self.flight:
            return None
        done = list(empty)
        keep = [f for f in self.flight if f.needed]
        if keep:
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
            still = []
            for f in keep:
                f.needed.discard(k)
                (still if f.needed else done).append(f)
            keep = still
        self.flight = keep
        if not done:
            return None
        rows, counts, ids = (x.array for x in self.h_take[self.par])
        by_len = collections.defaultdict(list)
        for f in done:
            for v in f.variants:
                by_len[f.db_len].append(v)
        where, off = {}, 0
        for db_len, vs in by_len.items():
            n = len(vs)
            rows[off:off + n] = [v.vid for v in vs]
            if db_len:
                self.dc.take_rows_into(rows[off:off + n], db_len, counts[off:off + n], ids[off:off + n],
                                       clear=True)
            else:
                counts[off:off + n] = 0
            for i, v in enumerate(vs):
                where[v.vid] = off + i
            off += n
        for f in done:
            for v in f.variants:
                self._release(v)
                self.cooling[self.par].append(v.vid)
        self.layout_dirty = True

        def handler(now):
            out = []
            for f in done:
                res = Result()
                for v in f.variants:
                    i = where[v.vid]
                    hits = ids[i, : min(int(counts[i]), MAX_MATCHES_LEN)].tolist()
                    if v.mirrored:
                        res.mirror_matches = hits
                        res.mirror_match_count = int(counts[i])
                    else:
                        res.matches = hits
                        res.match_count = int(counts[i])
                out.append(Completion(f.idx, f.arrival, now, res))
            return out
        return handler

    def _collect(self, pending) -> list:
        ev, handlers, par = pending
        tw = time.perf_counter()
        ev.synchronize()
        self.stats["wait_s"] += time.perf_counter() - tw
        for vid in self.cooling[par]:
            heapq.heappush(self.free_variants, vid)
        self.cooling[par].clear()
        code = self.dm.error_code()
        if code:
            raise IrisError(code, "a kernel reported a device error during serving")
        now = time.perf_counter()
        out = []
        for h in handlers:
            out += h(now)
        return out

    def serve(self, arrivals, requests, appends=None, max_wall_s: float = 600.0, lookahead: int = 256) -> list:
        """Open-loop run: request i arrives at arrivals[i] seconds after start.
        appends: {request index: (code_records, mask_records)} for requests of
        kind "append".  Waiting requests are admitted in arrival order; one
        that does not fit yet is passed by later ones that do (within
        `lookahead` waiting requests), but never by an append, so every
        request sees exactly the appends that arrived before it.  Returns the
        completions (latency = done - arrival)."""
        t0 = time.perf_counter()
        order = collections.deque(sorted(range(len(requests)), key=lambda i: arrivals[i]))
        waiting = collections.deque()
        completions = []
        total = len(requests)
        pending = None  # (event, handlers) of the step in flight
        self.dm.set_host_sync(False)
        try:
            while len(completions) < total:
                now = time.perf_counter() - t0
                if now > max_wall_s:
                    raise TimeoutError("serving run exceeded its wall-clock budget")
                while order and arrivals[order[0]] <= now:
                    waiting.append(order.popleft())
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
                    elif r.kind == "reauth" and len(reauth_items) < self.max_reauth:
                        reauth_items.append((i, t0 + arrivals[i], r))
                    elif r.kind == "uniqueness" and self.can_admit(r):
                        self.admit(r, i, t0 + arrivals[i])
                    else:
                        kept.append(i)
                waiting = kept
                ts = time.perf_counter()
                handlers = []
                if reauth_items:
                    handlers.append(self._launch_reauth(reauth_items))
                h = self._launch_step()
                if h:
                    handlers.append(h)
                launched = None
                if handlers:
                    ev = self.events[self.par]
                    ev.record(self.dm.stream(0))
                    launched = (ev, handlers, self.par)
                    self.par ^= 1
                self.stats["launch_s"] += time.perf_counter() - ts
                if pending:
                    completions += self._collect(pending)
                pending = launched
                if pending is None and not self.flight and order and not waiting:
                    time.sleep(max(0.0, min(0.002, arrivals[order[0]] - (time.perf_counter() - t0))))
            if pending:
                completions += self._collect(pending)
        finally:
            self.dm.synchronize()
            self.dm.set_host_sync(True)
        return completions

    def checkpoint(self) -> dict:
        """The server's resumable state between serve() calls: the device
        batch counter (with the parties' seeds, the whole ChaCha state) and
        the DB length (the DB itself stays resident)."""
        return {"batch_counter": self.dm.batch_counter(), "db_len": self.db_len}

    def restore(self, state: dict) -> None:
        """Resumes from checkpoint(): later steps draw fresh randomness after
        the saved counter, and requests scan the saved DB length."""
        if self.flight:
            raise RuntimeError("restore() with requests in flight")
        if state["db_len"] > self.db_capacity:
            raise ValueError("checkpointed DB length exceeds the capacity")
        self.dm.set_batch_counter(int(state["batch_counter"]))
        self.db_len = int(state["db_len"])
        for e in self.ce + self.me:
            e.set_db_len(self.db_len)

    def close(self) -> None:
        self.dm.synchronize()
        for e in self.ce + self.me:
            e.set_pair(False)
        for o in self.sce + self.sme + [self.dc, self.sdc]:
            o.close()
        for e in self.events:
            e.close()


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
                    out[j].mirror_match_count = int(counts[v])
                else:
                    out[j].matches = hits
                    out[j].match_count = int(counts[v])
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
