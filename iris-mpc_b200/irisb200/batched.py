"""Batched launches of uneven requests on the resident share DB.

A batch mixes uniqueness requests (the query against the whole DB) and reauth
requests (the query against one target entry, iris-mpc-gpu/src/server/
actor.rs:1465-1475), each with 1..31 centred rotations
(IrisRotation::centered, iris-mpc-common/src/galois_engine.rs:651-653) and
optionally a mirrored variant (galois_engine.rs:218-225,520-543;
server/mod.rs:156-176).  Instead of one 32-row slot per query iris (the plain
drop-in), the rows of all variants are packed densely into 32-row words: a
word may carry several queries, each a contiguous run of rows, and the
threshold kernel ORs each run separately (segment table).  Reauth variants
run on a gathered subset (the target records copied device-to-device,
prefetch_subset share_db.rs:344-407) instead of the whole DB.

The device work of a batch -- comparator reset, the six limb GEMMs and the
fused threshold/open/OR per DB chunk, the result merge -- is captured once per
layout into a CUDA graph and replayed (the DB pass itself is the library's
native irs_scan_run over the segment table); the ChaCha batch id comes from
the device batch counter, so a replay draws fresh randomness.  The library's
native tuner (irs_scan_tune) picks, per padded row count, by timing each
candidate's pass (and the three fastest again, interleaved, against the
clock's drift): the path
(the GEMM launch then the threshold launch per chunk, the same with the two-SM
GEMM, or the one-kernel fused GEMM + threshold scan), the GEMM's tile width
along the query rows and the DB chunk length.

A request and its mirrored variant share one uploaded base share; the row
descriptor's mirror bit makes the device build the mirrored rotations.
submit() prepares a batch in page-locked buffers and only enqueues it, so
two batches can be in flight; collect() returns a batch's results.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import (IRIS_CODE_LENGTH, MASK_CODE_LENGTH, MAX_MATCHES_LEN, Circuits, DeviceManager, DistanceComparator,
               Event, Graph, IrisError, PinnedArray, ShareDB, dot_many)
from .scan import PlainScan

MULTS = [1, 1, 1, 2, 2, 2]


def centred_rotations(n_rot: int) -> range:
    """Indices into all_rotations() of the n centred rotations (15 = centre)."""
    if not 1 <= n_rot <= 31:
        raise ValueError("1..31 rotations")
    lo = (31 - n_rot) // 2
    return range(lo, lo + n_rot)


@dataclass
class Request:
    """One query iris of a batch.  code/mask: the three parties' preprocessed
    query shares, [3][12800] and [3][6400] u16."""
    code: np.ndarray
    mask: np.ndarray
    n_rot: int = 31
    mirrored: bool = False
    kind: str = "uniqueness"  # or "reauth"
    target: int = -1


@dataclass
class Result:
    matches: list = field(default_factory=list)         # matched entries (uniqueness, normal orientation)
    mirror_matches: list = field(default_factory=list)  # matched entries of the mirrored variant
    reauth_match: bool | None = None
    reauth_mirror_match: bool | None = None
    match_count: int | None = None         # untruncated number of matches (lists keep the lowest 256)
    mirror_match_count: int | None = None


@dataclass
class Ticket:
    """A submitted batch (BatchedEngine.submit); collect() returns its results."""
    par: int
    requests: list
    uniq: list
    reauth: list
    results: list | None = None


def full_face_mirror_attack(request: Request, result: Result) -> bool:
    """Full-face mirror attack detection (iris-mpc-gpu/src/server/actor.rs:
    1316-1336): a uniqueness request whose normal orientation matches no DB
    entry while its mirrored orientation matches one.  Other request kinds,
    and requests without a mirrored orientation, are never flagged."""
    return (request.kind == "uniqueness" and request.mirrored and not result.matches
            and bool(result.mirror_matches))


@dataclass
class Layout:
    """Dense packing of the variants' rows into 32-row words."""
    row_desc: np.ndarray   # [rows] (src << 8) | (mirror << 7) | rotation, 0xFFFFFFFF = empty
    seg_start: np.ndarray  # [n_slots + 1]
    seg_query: np.ndarray  # [n_seg] variant index (bitmap row)
    seg_mask: np.ndarray   # [n_seg] rows of the slot belonging to the variant
    n_rows: int
    n_slots: int


def pack(variant_rows: list) -> Layout:
    """First-fit decreasing packing of variants (each a list of rotation
    indices, reported as bitmap row = its index) into 32-row words without
    splitting a variant across words."""
    order = sorted(range(len(variant_rows)), key=lambda v: -len(variant_rows[v]))
    slots = []  # each: list of (variant, first row, n)
    fill = []
    for v in order:
        n = len(variant_rows[v])
        for s, used in enumerate(fill):
            if used + n <= 32:
                slots[s].append((v, used, n))
                fill[s] += n
                break
        else:
            slots.append([(v, 0, n)])
            fill.append(n)
    n_slots = len(slots)
    row_desc = np.full(n_slots * 32, 0xFFFFFFFF, np.uint32)
    seg_start = [0]
    seg_query, seg_mask = [], []
    for s, segs in enumerate(slots):
        for v, first, n in segs:
            for k, rot in enumerate(variant_rows[v]):
                row_desc[s * 32 + first + k] = (v << 8) | rot
            seg_query.append(v)
            seg_mask.append(((1 << n) - 1) << first if n < 32 else 0xFFFFFFFF)
        seg_start.append(len(seg_query))
    return Layout(row_desc, np.array(seg_start, np.uint32), np.array(seg_query, np.uint32),
                  np.array(seg_mask, np.uint32), n_slots * 32, n_slots)


def attach_bases(layout: Layout, base_of, mirrored) -> Layout:
    """Points the rows of variant v at base query base_of[v], mirrored on the
    device (bit 7 of the row descriptor) when mirrored[v]: a request and its
    mirrored variant share one uploaded base."""
    d = layout.row_desc.copy()
    live = d != 0xFFFFFFFF
    v = d[live] >> 8
    flag = np.where(np.asarray(mirrored, bool)[v], 0x80, 0).astype(np.uint32)
    d[live] = (np.asarray(base_of, np.uint32)[v] << 8) | flag | (d[live] & 0x7F)
    return Layout(d, layout.seg_start, layout.seg_query, layout.seg_mask, layout.n_rows, layout.n_slots)


def padded_rows(n_rows: int, cap: int) -> int:
    """Query rows to run for `n_rows` packed rows, padded for the GEMM tile the
    library picks (gemm_block_n_for): 64 rows stay 64 (the pass streams the
    DB), up to 768 rows pad to a multiple of 128, above to a multiple of 256."""
    if n_rows <= 64:
        n = 64
    elif n_rows <= 768:
        n = -(-n_rows // 128) * 128
    else:
        n = -(-n_rows // 256) * 256
    return min(n, max(cap // 64 * 64, n_rows))


def pad_rows(layout: Layout, cap: int) -> Layout:
    """Pads the row table with empty rows (padded_rows); the segment table is
    unchanged, so the threshold kernel still visits only the packed slots."""
    n = padded_rows(layout.n_rows, cap)
    if n <= layout.n_rows:
        return layout
    rd = np.full(n, 0xFFFFFFFF, np.uint32)
    rd[: layout.n_rows] = layout.row_desc
    return Layout(rd, layout.seg_start, layout.seg_query, layout.seg_mask, n, layout.n_slots)


class BatchedEngine:
    """Runs batches of Requests against the six resident engines (party p code
    at code_engines[p], mask at mask_engines[p])."""

    def __init__(self, dm: DeviceManager, code_engines, mask_engines, circuits: Circuits, max_variants: int = 512,
                 max_reauth: int = 512, threshold_a: int = 16384, seeds=None, autotune: bool = True,
                 path: str | None = None):
        self.dm = dm
        self.ce, self.me = list(code_engines), list(mask_engines)
        self.c = circuits
        self.threshold_a = threshold_a
        self.max_variants = max_variants
        self.db_len = self.ce[0].db_len()
        self.dc = DistanceComparator(dm, max_variants, max(self.ce[0].db_len(), 64), match_list_cap=1 << 20)
        # reauth subset: one record per reauth variant
        self.max_reauth = max_reauth
        seeds = seeds or [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
        rows_cap = max_reauth * 2 * 32
        self.sce = [ShareDB(p, dm, max_reauth, rows_cap, IRIS_CODE_LENGTH, seeds[p]) for p in range(3)]
        self.sme = [ShareDB(p, dm, max_reauth, rows_cap, MASK_CODE_LENGTH, seeds[p]) for p in range(3)]
        for e in self.sce + self.sme:
            e.alloc_db(max_reauth)
        self.sdc = DistanceComparator(dm, max_reauth, max_reauth, match_list_cap=1 << 16)
        for e in self.ce + self.me + self.sce + self.sme:
            e.use_batch_counter(True)
        circuits.use_batch_counter(True)
        self._pin = None     # page-locked buffers, two sets (allocated on first use)
        self._pinned = []    # their PinnedArray owners
        self._events = None
        self._inflight = [None, None]
        self._par = 0
        self.graphs = {}
        # the DB pass and its tuner, native (irs_scan_*), over the packed rows
        self.scan = PlainScan(dm, self.ce, self.me, circuits, self.dc, 1, self.db_len, threshold_a)
        self.tuned = {}       # padded rows -> chosen (path, tile, chunk)
        self.tune_log = {}    # padded rows -> [(candidate, ms per DB pass)]
        self.autotune = autotune
        if path not in (None, "split", "pair", "fused"):
            raise ValueError("path is None (tuned), 'split', 'pair' or 'fused'")
        self.fixed = path     # restricts the candidates to one path

    # -- configuration -----------------------------------------------------
    def _chunks(self, n: int, chunk: int):
        out, off = [], 0
        while off < n:
            ln = min(chunk, n - off)
            out.append((off, ln))
            off += ln
        return out

    def _capture(self) -> Graph:
        """The DB pass of the configured candidate as a graph: comparator
        reset, the library's native pass (irs_scan_run, segment table), merge."""
        def body():
            self.dc.reset()
            self.scan.scan()
            self.dc.join_db_matches(self.max_variants, self.db_len)
        return Graph.capture(self.dm, body)

    @staticmethod
    def _candidates(n_rows: int, db_len: int):
        """(path, tile, DB chunk) candidates for a padded row count.
        path "split": the GEMM launch (tile = its query-row width) then the
        threshold launch per chunk; "pair": the same with the two-SM GEMM on
        the 256-row tile; "fused": the one-kernel GEMM + threshold scan
        (128-row tiles).  The 64-row GEMM tile is a candidate up to 768 rows,
        where the pass is close to streaming the DB.  Chunks of 131,072 down to
        8,192 entries: under the power cap, shorter GEMM + threshold
        alternations keep the SM clock higher (two-SM GEMM on a 524,288-entry
        plain batch: 163.7 ms per batch at 32,768-entry chunks, 157-161 at
        16,384, 154-156 at 8,192 on one GPU), while very short launches lose
        their last partial wave; the fused kernel is timed on the three
        longest."""
        n_pad = (n_rows + 63) // 64 * 64
        full = (db_len + 31) // 32 * 32
        chunks = sorted({min(full, c) for c in (131072, 65536, 32768, 16384, 8192)}, reverse=True)
        tiles = [t for t in (256, 128, 64) if n_pad % t == 0 and (t != 64 or n_pad <= 768)] or [64]
        out = [("split", t, ch) for t in tiles for ch in chunks]
        if n_pad % 256 == 0:
            out += [("pair", 256, ch) for ch in chunks]
        if n_pad % 128 == 0:
            out += [("fused", 128, ch) for ch in chunks[:3]]
        return out

    def _run_db_pass(self, layout: Layout, cand) -> None:
        path, tile, chunk = cand
        key = (layout.n_slots, path, tile, chunk, self.db_len)
        self.scan.set_rows(layout.n_rows, True)
        self.scan.configure(cand)  # engines' GEMM variant and tile; the fused ring before any capture
        g = self.graphs.get(key)
        if g is None:
            g = self._capture()
            self.graphs[key] = g
        g.launch(self.dm.stream(0))

    def _tune(self, layout: Layout):
        """The (path, tile, chunk) for this padded row count: the library's
        native tuner (irs_scan_tune) times every candidate on the batch at hand
        -- a warm pass, then two consecutive passes each (the power-capped
        clock needs them to settle) -- then re-times the three fastest
        interleaved over two rounds (the clock drifts during a tuning run by as
        much as the candidates differ) and keeps the best mean; once per
        padded row count."""
        n_pad = (layout.n_rows + 63) // 64 * 64
        if n_pad in self.tuned:
            return self.tuned[n_pad]
        cands = self._candidates(layout.n_rows, self.db_len)
        if self.fixed is not None:
            cands = [c for c in cands if c[0] == self.fixed] or cands
        if not self.autotune or len(cands) == 1:
            self.tuned[n_pad] = cands[0]
            return cands[0]
        self.scan.set_rows(layout.n_rows, True)
        only = self.fixed if any(c[0] == self.fixed for c in cands) else None
        best = self.scan.tune(only_path=only)
        self.tune_log[n_pad] = list(self.scan.tune_log)
        self.tuned[n_pad] = best
        return best

    # -- one batch -----------------------------------------------------------
    def run(self, requests: list) -> list:
        """Runs one batch and returns its results (submit + collect)."""
        return self.collect(self.submit(requests))

    def _variants(self, requests):
        uniq, reauth = [], []  # (request index, mirrored?)
        for i, r in enumerate(requests):
            dst = reauth if r.kind == "reauth" else uniq
            dst.append((i, False))
            if r.mirrored:
                dst.append((i, True))
        if len(uniq) > self.max_variants or len(reauth) > self.max_reauth:
            raise ValueError("batch exceeds the engine's variant capacity")
        for i, _ in reauth:
            if not 0 <= requests[i].target < self.db_len:
                raise ValueError(f"reauth target {requests[i].target} of request {i} is not in the DB")
        return uniq, reauth

    def _buffers(self):
        """Two sets of page-locked host buffers, one per batch in flight."""
        if self._pin is None:
            def P(shape, dtype):
                a = PinnedArray(shape, dtype)
                self._pinned.append(a)
                return a.array
            nu, nr = self.max_variants, self.max_reauth
            R, Rr = self.ce[0].query_length, self.sce[0].query_length
            self._pin = [{
                "ucode": P((3, nu, IRIS_CODE_LENGTH), np.uint16), "umask": P((3, nu, MASK_CODE_LENGTH), np.uint16),
                "urows": P((R,), np.uint32),
                "useg": (P((R // 32 + 1,), np.uint32), P((nu,), np.uint32), P((nu,), np.uint32)),
                "final": P((nu,), np.uint32), "counters": P((nu,), np.uint32),
                "matches": P((nu, MAX_MATCHES_LEN), np.uint32),
                "rids": P((nr,), np.uint32),
                "rcode": P((3, nr, IRIS_CODE_LENGTH), np.uint16), "rmask": P((3, nr, MASK_CODE_LENGTH), np.uint16),
                "rrows": P((Rr,), np.uint32),
                "rseg": (P((Rr // 32 + 1,), np.uint32), P((nr,), np.uint32), P((nr,), np.uint32)),
                "rbits": P((nr, self.sdc.row_words()), np.uint32),
            } for _ in range(2)]
            self._events = [Event(), Event()]
        return self._pin

    @staticmethod
    def _fill_bases(requests, variants, code, mask):
        """One base share per request, written into code [3][*][12800] / mask
        [3][*][6400] (a mirrored variant reads its request's base through the
        mirror bit); returns (bases, base index per variant, mirrored flags)."""
        order = list(dict.fromkeys(i for i, _ in variants))
        index = {i: k for k, i in enumerate(order)}
        for k, i in enumerate(order):
            code[:, k] = requests[i].code
            mask[:, k] = requests[i].mask
        return len(order), [index[i] for i, _ in variants], [mir for _, mir in variants]

    def _stage(self, requests, variants, code, mask, rows, seg, cap: int, pad: bool):
        """Bases, row table and segment table of one pass in the page-locked
        buffers; returns (layout, bases, rows used, segments used)."""
        nb, base_of, mirrored = self._fill_bases(requests, variants, code, mask)
        layout = attach_bases(pack([list(centred_rotations(requests[i].n_rot)) for i, _ in variants]),
                              base_of, mirrored)
        if pad:
            layout = pad_rows(layout, cap)
        if layout.n_rows > rows.size:
            raise ValueError("batch exceeds the engine's query-row capacity")
        rows[: layout.n_rows] = layout.row_desc
        ss, sq, sm = seg
        ns, nq = layout.seg_start.size, layout.seg_query.size
        ss[:ns], sq[:nq], sm[:nq] = layout.seg_start, layout.seg_query, layout.seg_mask
        return layout, nb, layout.n_rows, (ns, nq)

    def submit(self, requests: list) -> "Ticket":
        """Prepares one batch in page-locked buffers and enqueues its device
        work (the DB pass and the reauth pass, then the result copies),
        returning without waiting; collect() returns its results.  Two
        batches can be in flight, so the host prepares batch k+1 while the
        GPU runs batch k; submitting a third first collects the batch whose
        buffers it reuses."""
        uniq, reauth = self._variants(requests)
        par = self._par
        if self._inflight[par] is not None:
            self.collect(self._inflight[par])
        buf = self._buffers()[par]
        if uniq:
            ulay, unb, urows, (uns, unq) = self._stage(requests, uniq, buf["ucode"], buf["umask"], buf["urows"],
                                                       buf["useg"], self.ce[0].query_length, pad=True)
        if reauth:
            rlay, rnb, rrows, (rns, rnq) = self._stage(requests, reauth, buf["rcode"], buf["rmask"], buf["rrows"],
                                                       buf["rseg"], self.sce[0].query_length, pad=False)
            ids = buf["rids"][: len(reauth)]
            ids[:] = [requests[i].target for i, _ in reauth]
        self.dm.set_host_sync(False)
        try:
            self.dm.advance_batch_counter()  # fresh ChaCha batch id for both passes
            if uniq:
                rt = buf["urows"][:urows]
                for p in range(3):
                    self.ce[p].query_upload_rows(buf["ucode"][p, :unb], rt)
                    self.me[p].query_upload_rows(buf["umask"][p, :unb], rt)
                ss, sq, sm = buf["useg"]
                self.dc.set_segments(ss[:uns], sq[:unq], sm[:unq])
                cand = self._tune(ulay)  # times candidates (synchronously) once per padded size
                self._run_db_pass(ulay, cand)
                n = len(uniq)
                self.dc.fetch_final_results_into(n, buf["final"][:n], buf["counters"][:n], buf["matches"][:n])
            if reauth:
                n = len(reauth)
                for p in range(3):
                    self.sce[p].gather_records(self.ce[p], ids)
                    self.sme[p].gather_records(self.me[p], ids)
                rt = buf["rrows"][:rrows]
                for p in range(3):
                    self.sce[p].query_upload_rows(buf["rcode"][p, :rnb], rt)
                    self.sme[p].query_upload_rows(buf["rmask"][p, :rnb], rt)
                for e in self.sce + self.sme:
                    e.set_pair(False)
                    e.set_tile(0)
                self.sdc.reset()
                ss, sq, sm = buf["rseg"]
                self.sdc.set_segments(ss[:rns], sq[:rnq], sm[:rnq])
                dot_many(self.sce + self.sme, MULTS, 0, n)
                self.sdc.compare_threshold_open_prepared(self.c, self.sce, self.sme, 0, n, self.threshold_a)
                self.sdc.fetch_rows_into(0, n, buf["rbits"][:n])
            self._events[par].record(self.dm.stream(0))
        except BaseException:
            self.dm.synchronize()  # nothing may still read the buffers
            raise
        finally:
            self.dm.set_host_sync(True)
        t = Ticket(par, requests, uniq, reauth)
        self._inflight[par] = t
        self._par ^= 1
        return t

    def collect(self, ticket: "Ticket") -> list:
        """Waits for a submitted batch and returns its results (per request:
        sorted DB matches of each uniqueness orientation, the match bit of
        each reauth orientation against its target)."""
        if ticket.results is not None:
            return ticket.results
        self._events[ticket.par].synchronize()
        self._inflight[ticket.par] = None
        code = self.dm.error_code()
        if code:
            raise IrisError(code, "a kernel reported a device error during a batched launch")
        buf = self._pin[ticket.par]
        results = [Result() for _ in ticket.requests]
        counters, matches = buf["counters"], buf["matches"]
        for v, (i, mir) in enumerate(ticket.uniq):
            ids = sorted(matches[v, :min(int(counters[v]), MAX_MATCHES_LEN)].tolist())
            if mir:
                results[i].mirror_matches = ids
                results[i].mirror_match_count = int(counters[v])
            else:
                results[i].matches = ids
                results[i].match_count = int(counters[v])
        bits = buf["rbits"]
        for v, (i, mir) in enumerate(ticket.reauth):
            hit = bool((int(bits[v, v // 32]) >> (v % 32)) & 1)  # variant v against subset record v
            if mir:
                results[i].reauth_mirror_match = hit
            else:
                results[i].reauth_match = hit
        ticket.results = results
        return results

    def close(self) -> None:
        self.dm.synchronize()
        for g in self.graphs.values():
            g.close()
        self.graphs.clear()
        self.scan.restore()  # the DB engines go back to the library's default GEMM
        self.scan.close()
        for o in self.sce + self.sme + [self.dc, self.sdc]:
            o.close()
        for a in self._pinned:
            a.free()
        for e in self._events or []:
            e.close()
        self._pinned = []
        self._pin = self._events = None
