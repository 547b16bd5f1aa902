"""The plain drop-in's DB pass, autotuned.

The reference's actor scans the share DB in chunks (DB_CHUNK_SIZE per device,
iris-mpc-gpu/src/server/actor.rs:2246-2589): per chunk the dot products of the
three parties' code and mask shares (Phase 1), then the threshold protocol
and the open with the rotation OR (Phase 2).  PlainScan runs that pass over
this library's resident engines for one uploaded batch of 31-rotation query
slots, along one of three paths per chunk -- the limb GEMM launch then the
threshold launch ("split"), the same with the two-SM GEMM ("pair"), or the
one-kernel fused scan ("fused") -- and `tune()` picks the path and the chunk
length by timing each candidate on the batch at hand, as BatchedEngine does
for packed batches.  Results are identical on every path.
"""
from __future__ import annotations

import time

from . import dot_many
from .batched import MULTS, BatchedEngine


class PlainScan:
    """One uploaded batch of `n_slots` 32-row query slots (rows 0..30 valid,
    slot s reported as query s) against entries [0, db_len) of the six
    engines (party p code at code_engines[p], mask at mask_engines[p]), with
    results in DistanceComparator `dc`."""

    def __init__(self, dm, code_engines, mask_engines, circuits, dc, n_slots: int, db_len: int,
                 threshold_a: int = 16384):
        self.dm, self.c, self.dc = dm, circuits, dc
        self.ce, self.me = list(code_engines), list(mask_engines)
        self.n_slots, self.db_len, self.threshold_a = n_slots, db_len, threshold_a
        self.cand = ("split", 0, 65536)
        self.tune_log = []

    def candidates(self):
        """(path, tile, chunk) candidates for the batch's padded rows."""
        return BatchedEngine._candidates(self.n_slots * 32, self.db_len)

    def configure(self, cand) -> None:
        path, tile, _ = cand
        for e in self.ce + self.me:
            e.set_pair(path == "pair")
            e.set_tile(tile if path != "fused" else 0)
        if path == "fused":  # allocates the comparator's ring before any capture
            self.dc.scan_fused(self.c, self.ce, self.me, 0, 0, self.threshold_a, n_slots=self.n_slots)
        self.cand = cand

    def chunks(self):
        ch = self.cand[2]
        return [(o, min(ch, self.db_len - o)) for o in range(0, self.db_len, ch)]

    def scan(self, events=None) -> None:
        """One pass over the DB (no comparator reset).  events: optional list,
        per chunk, of three callables recorded before the chunk, between its
        two launches (split / pair) and after it."""
        path = self.cand[0]
        for k, (off, ln) in enumerate(self.chunks()):
            if events:
                events[k][0]()
            if path == "fused":
                self.dc.scan_fused(self.c, self.ce, self.me, off, ln, self.threshold_a, n_slots=self.n_slots)
                if events:
                    events[k][1]()
            else:
                dot_many(self.ce + self.me, MULTS, off, ln)
                if events:
                    events[k][1]()
                self.dc.compare_threshold_open(self.c, self.ce, self.me, off, ln, self.n_slots, self.threshold_a)
            if events:
                events[k][2]()

    def _time(self, cand, passes: int) -> float:
        """Seconds per pass of `passes` consecutive passes after a warm one."""
        self.configure(cand)
        self.dc.reset()
        self.scan()
        self.dm.synchronize()
        t0 = time.perf_counter()
        for _ in range(passes):
            self.dc.reset()
            self.scan()
        self.dm.synchronize()
        return (time.perf_counter() - t0) / passes

    def tune(self, cands=None, passes: int = 2, finalists: int = 3, rounds: int = 2):
        """Times `passes` consecutive passes of each candidate after a warm
        pass (the power-capped clock settles differently for each path), then
        re-times the `finalists` fastest interleaved for `rounds` rounds (the
        clock drifts over a tuning run, and candidates timed far apart are not
        comparable at the 2% level) and keeps the best mean of those rounds;
        returns it.  tune_log: (candidate, ms per pass) of the first round,
        then (candidate, mean ms over the interleaved rounds) per finalist."""
        self.tune_log = []
        first = []
        for cand in cands or self.candidates():
            el = self._time(cand, passes)
            first.append((el, cand))
            self.tune_log.append((cand, el * 1e3))
        first.sort(key=lambda x: x[0])
        top = [c for _, c in first[:max(1, finalists)]]
        if len(top) > 1 and rounds > 0:
            acc = {c: 0.0 for c in top}
            for _ in range(rounds):
                for c in top:
                    acc[c] += self._time(c, passes)
            means = {c: acc[c] / rounds for c in top}
            self.tune_log += [(c, means[c] * 1e3) for c in top]
            best = min(top, key=lambda c: means[c])
        else:
            best = top[0]
        self.configure(best)
        return best

    def restore(self) -> None:
        """The engines back to the library's default GEMM."""
        for e in self.ce + self.me:
            e.set_pair(False)
            e.set_tile(0)
