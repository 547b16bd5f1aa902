"""Host-side logic of the batched launch (no GPU): the row descriptors that
point variants at shared base queries with the mirror bit, and the
expansion rule the device applies to them (rotation of the mirrored share)
checked against the oracle's mirror_share / rotate_share."""
from __future__ import annotations

import numpy as np

from oracle import oracle
from irisb200.batched import attach_bases, centred_rotations, pack


def expand_row(base: np.ndarray, d: int) -> np.ndarray:
    """The row that expand_rows_kernel builds for descriptor d from the base
    queries `base` [n][K], restated with numpy (4-coefficient columns)."""
    K = base.shape[1]
    src, rot, mirror = d >> 8, d & 0x7F, bool(d & 0x80)
    left = 15 - rot
    cols = base[src].reshape(K // 800, 200, 4).astype(np.int64)
    src_col = (np.arange(200) + left) % 200
    if mirror:
        src_col = np.where(src_col < 100, 99 - src_col, 299 - src_col)
    out = cols[:, src_col, :]
    if mirror and K == 12800:
        out[8:] = -out[8:]
    return (out % 65536).astype(np.uint16).reshape(K)


def test_attach_bases_sets_source_and_mirror_bit():
    variants = [list(centred_rotations(n)) for n in (31, 31, 16, 1, 1)]
    base_of = [0, 0, 1, 2, 2]
    mirrored = [False, True, False, False, True]
    lay = pack(variants)
    out = attach_bases(lay, base_of, mirrored)
    assert (lay.row_desc == out.row_desc).sum() == (lay.row_desc == 0xFFFFFFFF).sum() + \
        sum(len(r) for v, r in enumerate(variants) if base_of[v] == v and not mirrored[v])
    for r, d in enumerate(lay.row_desc):
        if d == 0xFFFFFFFF:
            assert out.row_desc[r] == 0xFFFFFFFF
            continue
        v = int(d) >> 8
        e = int(out.row_desc[r])
        assert e >> 8 == base_of[v]
        assert bool(e & 0x80) == mirrored[v]
        assert e & 0x7F == int(d) & 0xFF
    assert np.array_equal(out.seg_query, lay.seg_query) and np.array_equal(out.seg_mask, lay.seg_mask)


def test_device_mirror_rule_matches_oracle():
    rng = np.random.default_rng(11)
    for K, flip in ((12800, True), (6400, False)):
        base = rng.integers(0, 65536, (2, K), dtype=np.uint16)
        mirrored = oracle.mirror_share(base[1], flip)
        for rot in range(31):
            assert np.array_equal(expand_row(base, (1 << 8) | 0x80 | rot), oracle.rotate_share(mirrored, rot))
            assert np.array_equal(expand_row(base, (0 << 8) | rot), oracle.rotate_share(base[0], rot))


class _Obj:
    """Records calls; any method is a no-op."""

    def __init__(self, **kw):
        self.calls = []
        self.__dict__.update(kw)

    def __getattr__(self, name):
        def f(*a, **k):
            self.calls.append(name)
        return f


class _Buf:
    def __init__(self, shape, dtype):
        self.array = np.zeros(shape, dtype)

    def free(self):
        self.array = None


def _fake_engine(monkeypatch):
    """A BatchedEngine over fake device objects: the comparator reports
    variant v of the DB pass as matching entry 100 + v, and reauth variant v
    as matching its target when v is even."""
    import irisb200.batched as B
    from irisb200 import MAX_MATCHES_LEN

    class DM(_Obj):
        def set_host_sync(self, on):
            self.calls.append(("host_sync", bool(on)))

        def error_code(self):
            return 0

    class DC(_Obj):
        def fetch_final_results_into(self, n, final, counters, matches):
            assert not dm.calls or dm.calls[-1] != ("host_sync", True)
            counters[:n] = 1
            matches[:n, 0] = 100 + np.arange(n)

    class SDC(_Obj):
        def row_words(self):
            return 4

        def fetch_rows_into(self, first, n, out):
            out[:n] = 0
            for v in range(0, n, 2):
                out[v, v // 32] |= np.uint32(1 << (v % 32))

    class Graph:
        @staticmethod
        def capture(dm_, fn):
            fn()
            return _Obj()

    dm = DM()
    monkeypatch.setattr(B, "PinnedArray", _Buf)
    monkeypatch.setattr(B, "Event", _Obj)
    monkeypatch.setattr(B, "Graph", Graph)
    monkeypatch.setattr(B, "dot_many", lambda *a, **k: None)
    e = B.BatchedEngine.__new__(B.BatchedEngine)
    e.dm, e.c = dm, _Obj()
    e.ce = [_Obj(query_length=1024) for _ in range(3)]
    e.me = [_Obj(query_length=1024) for _ in range(3)]
    e.sce = [_Obj(query_length=8 * 64) for _ in range(3)]
    e.sme = [_Obj(query_length=8 * 64) for _ in range(3)]
    e.dc, e.sdc = DC(), SDC()
    e.scan = _Obj()  # the native DB pass (irs_scan_*): configure / run are no-ops here
    e.threshold_a, e.max_variants, e.max_reauth, e.db_len = 16384, 16, 8, 4096
    e._pin, e._pinned, e._events, e._inflight, e._par = None, [], None, [None, None], 0
    e.graphs, e.tuned, e.autotune, e.tune_log, e.fixed = {}, {}, False, {}, None
    assert MAX_MATCHES_LEN >= 1
    return e, dm


def test_submit_collect_maps_results_and_reuses_buffers(monkeypatch):
    from irisb200.batched import Request
    e, dm = _fake_engine(monkeypatch)
    z = np.zeros((3, 12800), np.uint16), np.zeros((3, 6400), np.uint16)

    def req(n, mir, kind="uniqueness", t=-1):
        return Request(code=z[0], mask=z[1], n_rot=n, mirrored=mir, kind=kind, target=t)
    batch = [req(31, True), req(16, False), req(1, True, "reauth", 7), req(31, False, "reauth", 9), req(1, False)]
    ta = e.submit(batch)
    tb = e.submit(batch)
    assert ta.par != tb.par and ta.results is None
    tc = e.submit(batch)  # reuses ta's buffers
    assert ta.results is not None and tc.par == ta.par
    for t in (ta, tb, tc):
        res = e.collect(t)
        # uniqueness variants in order: (0, normal), (0, mirror), (1, normal), (4, normal)
        assert res[0].matches == [100] and res[0].mirror_matches == [101]
        assert res[1].matches == [102] and res[4].matches == [103]
        # reauth variants: (2, normal) v0 hit, (2, mirror) v1 miss, (3, normal) v2 hit
        assert res[2].reauth_match is True and res[2].reauth_mirror_match is False
        assert res[3].reauth_match is True
    # every submit ran with host sync off and restored it afterwards
    syncs = [c for c in dm.calls if isinstance(c, tuple)]
    assert syncs == [("host_sync", False), ("host_sync", True)] * 3
    assert dm.calls.count("advance_batch_counter") == 3
    e.close()
    assert e._pin is None


def test_submit_rejects_oversized_batches(monkeypatch):
    import pytest
    from irisb200.batched import Request
    e, dm = _fake_engine(monkeypatch)
    for x in e.ce + e.me:
        x.query_length = 256  # 8 words of 32 rows
    z = np.zeros((3, 12800), np.uint16), np.zeros((3, 6400), np.uint16)
    with pytest.raises(ValueError):
        e.submit([Request(code=z[0], mask=z[1], n_rot=31, mirrored=True) for _ in range(9)])  # 18 variants > 16
    with pytest.raises(ValueError):  # 12 variants fit the count, but need 12 words of rows
        e.submit([Request(code=z[0], mask=z[1], n_rot=31, mirrored=True) for _ in range(6)])
    with pytest.raises(ValueError):  # reauth target outside the DB
        e.submit([Request(code=z[0], mask=z[1], n_rot=1, kind="reauth", target=e.db_len)])
    assert e._inflight == [None, None]
    assert not any(isinstance(c, tuple) for c in dm.calls)  # failed before any device work


def test_submit_edge_batches(monkeypatch):
    """An empty batch, a reauth-only batch and a uniqueness-only batch each
    complete; only the passes a batch needs are enqueued."""
    from irisb200.batched import Request
    e, dm = _fake_engine(monkeypatch)
    z = np.zeros((3, 12800), np.uint16), np.zeros((3, 6400), np.uint16)
    assert e.run([]) == []
    assert "compare_threshold_open_prepared" not in e.sdc.calls and not e.graphs
    res = e.run([Request(code=z[0], mask=z[1], n_rot=1, kind="reauth", target=3)])
    assert res[0].reauth_match is True and res[0].matches == [] and not e.graphs
    res = e.run([Request(code=z[0], mask=z[1], n_rot=16)])
    assert res[0].matches == [100] and res[0].reauth_match is None and e.graphs
    e.close()


def test_autotuner_candidates():
    """The tuner's candidates: the two-launch path at every tile width that
    divides the padded rows (the 64-row tile only up to 768 rows), the two-SM
    GEMM where the 256-row tile applies, the fused scan where the rows are a
    multiple of 128; the two-launch paths at 131,072 down to 8,192-entry
    chunks, the fused scan at the three longest (all capped at the DB)."""
    from irisb200.batched import BatchedEngine
    c = BatchedEngine._candidates(2048, 524288)
    assert ("split", 256, 131072) in c and ("split", 128, 32768) in c
    assert not any(t == 64 for _, t, _ in c)
    assert ("pair", 256, 65536) in c and ("fused", 128, 32768) in c
    assert ("pair", 256, 8192) in c and ("split", 256, 16384) in c and ("fused", 128, 16384) not in c
    assert len(c) == 2 * 5 + 5 + 3
    c = BatchedEngine._candidates(640, 524288)
    assert {t for p, t, _ in c if p == "split"} == {128, 64}
    assert not any(p == "pair" for p, _, _ in c) and any(p == "fused" for p, _, _ in c)
    c = BatchedEngine._candidates(64, 1000)
    assert c == [("split", 64, 1024)]
