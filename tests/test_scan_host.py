"""Host logic of the plain DB pass (irisb200.scan.PlainScan), no GPU: the
chunking of the DB, the tuner's selection (every candidate timed once, the
three fastest re-timed interleaved, the best mean kept) and the engines'
configuration per path, on fake engines and a fake clock."""
from __future__ import annotations

import pytest

from irisb200.scan import PlainScan


class _Engine:
    def __init__(self):
        self.pair, self.tile = None, None

    def set_pair(self, on):
        self.pair = on

    def set_tile(self, t):
        self.tile = t


class _Comparator:
    def __init__(self):
        self.fused_calls = []

    def scan_fused(self, c, ce, me, off, ln, a, n_slots=0):
        self.fused_calls.append((off, ln))

    def reset(self):
        pass


class _DM:
    def synchronize(self):
        pass


def _scan(db_len=100_000):
    ce = [_Engine() for _ in range(3)]
    me = [_Engine() for _ in range(3)]
    return PlainScan(_DM(), ce, me, None, _Comparator(), n_slots=64, db_len=db_len)


def test_chunks_cover_the_db():
    ps = _scan(100_000)
    ps.cand = ("split", 256, 32768)
    assert ps.chunks() == [(0, 32768), (32768, 32768), (65536, 32768), (98304, 1696)]
    ps.cand = ("pair", 256, 131072)
    assert ps.chunks() == [(0, 100_000)]


def test_configure_sets_every_engine():
    ps = _scan()
    ps.configure(("pair", 256, 32768))
    assert all(e.pair and e.tile == 256 for e in ps.ce + ps.me)
    ps.configure(("fused", 128, 65536))
    assert all(e.pair is False and e.tile == 0 for e in ps.ce + ps.me)
    assert ps.dc.fused_calls == [(0, 0)]  # the comparator's ring, allocated before any capture
    ps.restore()
    assert all(e.pair is False and e.tile == 0 for e in ps.ce + ps.me)


def test_tune_retimes_finalists_interleaved(monkeypatch):
    """A candidate that was fast in the first round only by clock drift loses
    to the best mean of the interleaved rounds."""
    ps = _scan()
    cands = [("split", 256, 65536), ("pair", 256, 32768), ("pair", 256, 16384), ("fused", 128, 65536)]
    first = {cands[0]: 0.150, cands[1]: 0.149, cands[2]: 0.151, cands[3]: 0.180}
    later = {cands[0]: 0.149, cands[1]: 0.155, cands[2]: 0.150}
    order = []

    def fake_time(cand, passes):
        order.append(cand)
        seen = order.count(cand)
        return first[cand] if seen == 1 else later[cand]

    monkeypatch.setattr(ps, "_time", fake_time)
    best = ps.tune(cands)
    # first round in candidate order, then the three fastest, interleaved, twice
    top = [cands[1], cands[0], cands[2]]
    assert order == cands + top + top
    assert best == cands[0]
    assert ps.cand == best
    assert [c for c, _ in ps.tune_log] == cands + top
    assert ps.tune_log[len(cands)][1] == pytest.approx(later[cands[1]] * 1e3)


def test_tune_single_candidate(monkeypatch):
    ps = _scan()
    monkeypatch.setattr(ps, "_time", lambda cand, passes: 0.1)
    assert ps.tune([("split", 256, 32768)]) == ("split", 256, 32768)
    assert len(ps.tune_log) == 1
