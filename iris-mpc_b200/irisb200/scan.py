"""The plain drop-in's DB pass, autotuned (the library's irs_scan_*).

The reference's actor scans the share DB in chunks (DB_CHUNK_SIZE per device,
iris-mpc-gpu/src/server/actor.rs:2246-2589): per chunk the dot products of the
three parties' code and mask shares (Phase 1), then the threshold protocol
and the open with the rotation OR (Phase 2).  PlainScan drives the library's
native pass (csrc/scan.cu) over the resident engines for one uploaded batch
of 31-rotation query slots, along one of three paths per chunk -- the limb
GEMM launch then the threshold launch ("split"), the same with the two-SM
GEMM ("pair"), or the one-kernel fused scan ("fused") -- and `tune()` picks
the path, the tile width and the chunk length by timing each candidate on the
batch at hand, as BatchedEngine does for packed batches.  Results are
identical on every path.
"""
from __future__ import annotations

import ctypes as C

from . import SCAN_PATHS, ScanCandidate, ScanTiming, _check, lib


def _cand(c: ScanCandidate):
    return (SCAN_PATHS[c.path], int(c.tile), int(c.chunk))


class PlainScan:
    """One uploaded batch of `n_slots` 32-row query slots (rows 0..30 valid,
    slot s reported as query s) against entries [0, db_len) of the six
    engines (party p code at code_engines[p], mask at mask_engines[p]), with
    results in DistanceComparator `dc`.  The handles must outlive it."""

    def __init__(self, dm, code_engines, mask_engines, circuits, dc, n_slots: int, db_len: int,
                 threshold_a: int = 16384):
        self.dm, self.c, self.dc = dm, circuits, dc
        self.ce, self.me = list(code_engines), list(mask_engines)
        self.n_slots, self.db_len, self.threshold_a = n_slots, db_len, threshold_a
        hc = (C.c_void_p * 3)(*[e.h for e in self.ce])
        hm = (C.c_void_p * 3)(*[e.h for e in self.me])
        h = C.c_void_p()
        _check(lib().irs_scan_init(dm.h, dc.h, circuits.h, C.cast(hc, C.c_void_p), C.cast(hm, C.c_void_p), n_slots,
                                   db_len, threshold_a, C.byref(h)))
        self.h = h.value
        self.tune_log = []

    @property
    def cand(self):
        """The configured (path, tile, chunk)."""
        c = ScanCandidate()
        _check(lib().irs_scan_current(self.h, C.byref(c)))
        return _cand(c)

    def candidates(self):
        """(path, tile, chunk) candidates for the batch's padded rows."""
        n = C.c_size_t()
        _check(lib().irs_scan_candidates(self.h, None, 0, C.byref(n)))
        arr = (ScanCandidate * n.value)()
        _check(lib().irs_scan_candidates(self.h, arr, n.value, C.byref(n)))
        return [_cand(c) for c in arr]

    def set_rows(self, n_rows: int, use_segments: bool) -> None:
        """Packed uneven rows: candidates for `n_rows` padded rows (0 = the
        slots'), and the threshold through the comparator's segment table."""
        _check(lib().irs_scan_set_rows(self.h, n_rows, int(use_segments)))

    def configure(self, cand) -> None:
        path, tile, chunk = cand
        _check(lib().irs_scan_configure(self.h, SCAN_PATHS.index(path), int(tile), int(chunk)))

    def chunks(self):
        ch = self.cand[2]
        return [(o, min(ch, self.db_len - o)) for o in range(0, self.db_len, ch)]

    def scan(self, stream=None) -> None:
        """One pass over the DB (no comparator reset), on party 0's stream
        unless `stream` is given."""
        _check(lib().irs_scan_run(self.h, stream))

    def set_timing(self, max_passes: int) -> None:
        """Per-chunk CUDA events for the next `max_passes` passes (0 = off;
        cleared by configure)."""
        _check(lib().irs_scan_set_timing(self.h, max_passes))

    def timings(self, reset: bool = True):
        """Per timed pass: (GEMM ms, threshold ms, whole-pass ms) lists; waits
        for the passes' events."""
        n = C.c_size_t()
        _check(lib().irs_scan_timings(self.h, None, None, None, 0, C.byref(n), 0))
        g, t, p = (C.c_double * max(1, n.value))(), (C.c_double * max(1, n.value))(), (C.c_double * max(1, n.value))()
        _check(lib().irs_scan_timings(self.h, C.cast(g, C.c_void_p), C.cast(t, C.c_void_p), C.cast(p, C.c_void_p),
                                      n.value, C.byref(n), int(reset)))
        return list(g)[:n.value], list(t)[:n.value], list(p)[:n.value]

    def tune(self, passes: int = 2, finalists: int = 3, rounds: int = 2, only_path: str | None = None):
        """Times `passes` consecutive passes of each candidate after a warm
        pass (the power-capped clock settles differently for each path), then
        re-times the `finalists` fastest interleaved for `rounds` rounds (the
        clock drifts over a tuning run, and candidates timed far apart are not
        comparable at the 2% level), configures the best mean and returns it;
        `only_path` restricts the candidates to one path.
        tune_log: (candidate, ms per pass) of the first round, then
        (candidate, mean ms over the interleaved rounds) per finalist."""
        cap = len(self.candidates()) + max(0, finalists)
        log = (ScanTiming * cap)()
        chosen, n = ScanCandidate(), C.c_size_t()
        op = -1 if only_path is None else SCAN_PATHS.index(only_path)
        _check(lib().irs_scan_tune(self.h, passes, finalists, rounds, op, C.byref(chosen), log, cap, C.byref(n)))
        self.tune_log = [(_cand(x.cand), float(x.ms)) for x in log[:min(n.value, cap)]]
        return _cand(chosen)

    def restore(self) -> None:
        """The engines back to the library's default GEMM."""
        _check(lib().irs_scan_restore(self.h))

    def close(self) -> None:
        if self.h:
            lib().irs_scan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
