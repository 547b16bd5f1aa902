"""GPU parity of the fused scan (irs_dc_scan_fused): the six limb GEMMs and
the threshold / open / rotation OR of a DB chunk in one persistent kernel.

Its results must equal the two-launch path (irs_sharedb_dot_many +
irs_dc_compare_threshold_open) bit for bit -- the dot shares and the circuit
keystream sit at the same positions -- and the CPU path on the same shares
(the predicate of iris-mpc-gpu/tests/threshold.rs:110-124, ORed over
rotations): match bitmap, match list, the anonymised-statistics distance
records (which carry every party's code and mask dot share of each match), for
plain 31-rotation slots and for packed uneven rows with a segment table, over
chunks with a ragged last tile, and from a captured CUDA graph."""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
import workload as W

pytestmark = pytest.mark.gpu

N_DB = 2000  # not a multiple of the 128-entry tile
N_Q = 8
DB_SEED = 0xDEADBEEF
Q_SEED = 42
PLANTED = {1: (17, 3), 5: (1900, -15), 6: (640, 15)}
MULTS = [1, 1, 1, 2, 2, 2]
CHUNKS = ((0, 1024), (1024, N_DB - 1024))


@pytest.fixture(scope="module")
def data(oracle):
    codes, masks, cs, ms = W.make_db(oracle, N_DB, DB_SEED)
    qc, qm, _ = W.make_queries(oracle, N_Q, codes, masks, Q_SEED, PLANTED)
    return dict(cs=cs, ms=ms, qc=qc, qm=qm)


def _setup(dm, data, n_rows):
    ce = [irisb200.ShareDB(p, dm, N_DB, n_rows, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, N_DB, n_rows, 6400, W.SEEDS[p]) for p in range(3)]
    for p in range(3):
        ce[p].alloc_db(N_DB)
        me[p].alloc_db(N_DB)
        ce[p].load_records(0, data["cs"][p])
        me[p].load_records(0, data["ms"][p])
    for e in ce + me:
        e.set_batch(3)
    return ce, me


def _close(objs):
    for o in objs:
        o.close()


def _dist_set(dc):
    entry, row, code, mask, n = dc.fetch_distances(1 << 14)
    return sorted((int(entry[i]), int(row[i]), tuple(int(x) for x in code[:, i]), tuple(int(x) for x in mask[:, i]))
                  for i in range(min(n, entry.size)))


def test_fused_plain_slots_equal_two_launch_path_and_cpu(dm, oracle, data):
    ce, me = _setup(dm, data, N_Q * 32)
    c = irisb200.Circuits(dm, W.SEEDS)
    c.set_batch(3)
    dcs = [irisb200.DistanceComparator(dm, N_Q, N_DB) for _ in range(2)]
    try:
        slots = [(j, 0, 31, j) for j in range(N_Q)]
        for p in range(3):
            ce[p].query_upload_slots(data["qc"][p], slots)
            me[p].query_upload_slots(data["qm"][p], slots)
        for dc in dcs:
            dc.enable_distance_capture(1 << 14)
        for off, ln in CHUNKS:
            irisb200.dot_many(ce + me, MULTS, off, ln)
            dcs[0].compare_threshold_open(c, ce, me, off, ln, N_Q, 16384)
            dcs[1].scan_fused(c, ce, me, off, ln, 16384, n_slots=N_Q)
        dm.synchronize()
        bm = [irisb200.bitmap_get(dc.fetch_bitmap(N_Q, N_DB), N_Q, N_DB) for dc in dcs]
        assert np.array_equal(bm[0], bm[1]), "fused scan differs from the two-launch path"
        exp = W.expected_bitmap(oracle, data["qc"], data["qm"], data["cs"], data["ms"], 16384)
        assert np.array_equal(bm[1], exp), "fused scan differs from the CPU path"
        for j, (e, _) in PLANTED.items():
            assert bm[1][j, e] == 1
        pairs = [sorted(map(tuple, dc.fetch_matches().tolist())) for dc in dcs]
        assert pairs[0] == pairs[1] == sorted(zip(*np.nonzero(exp)))
        d0, d1 = _dist_set(dcs[0]), _dist_set(dcs[1])
        assert d0 and d0 == d1, "distance records (per-party dot shares of the matches) differ"
        # final results through the usual merge
        res = []
        for dc in dcs:
            dc.join_db_matches(N_Q, N_DB)
            res.append(dc.fetch_final_results(N_Q))
        assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    finally:
        _close(dcs + [c] + ce + me)


def test_fused_segments_and_graph_replay(dm, oracle, data):
    """Packed uneven rows (1 / 16 / 31 centred rotations, mirrored variants)
    with a segment table; the fused scan captured in a graph and replayed
    equals the two-launch path and the CPU path per variant."""
    from irisb200.batched import attach_bases, centred_rotations, pack, pad_rows
    variants = [(j, n, mir) for j, n, mir in
                [(0, 31, False), (1, 16, False), (1, 16, True), (2, 1, False), (3, 31, True), (4, 16, False),
                 (5, 31, False), (5, 31, True), (6, 1, True), (7, 16, False), (6, 31, False), (2, 16, True)]]
    lay = pack([list(centred_rotations(n)) for _, n, _ in variants])
    lay = attach_bases(lay, [j for j, _, _ in variants], [m for _, _, m in variants])
    n_rows = 512
    lay = pad_rows(lay, n_rows)
    assert lay.n_rows % 128 == 0
    nv = len(variants)
    ce, me = _setup(dm, data, n_rows)
    c = irisb200.Circuits(dm, W.SEEDS)
    c.set_batch(3)
    dcs = [irisb200.DistanceComparator(dm, nv, N_DB) for _ in range(2)]
    g = None
    try:
        for p in range(3):
            ce[p].query_upload_rows(data["qc"][p], lay.row_desc)
            me[p].query_upload_rows(data["qm"][p], lay.row_desc)
        for dc in dcs:
            dc.set_segments(lay.seg_start, lay.seg_query, lay.seg_mask)
        for off, ln in CHUNKS:
            irisb200.dot_many(ce + me, MULTS, off, ln)
            dcs[0].compare_threshold_open_prepared(c, ce, me, off, ln, 16384)
        # the first fused call allocates the ring, then the captured replay
        dcs[1].scan_fused(c, ce, me, 0, 64, 16384, use_segments=True)
        dm.synchronize()

        def body():
            dcs[1].reset()
            for off, ln in CHUNKS:
                dcs[1].scan_fused(c, ce, me, off, ln, 16384, use_segments=True)
        g = irisb200.Graph.capture(dm, body)
        g.launch(dm.stream(0))
        dm.synchronize()
        bm = [irisb200.bitmap_get(dc.fetch_bitmap(nv, N_DB), nv, N_DB) for dc in dcs]
        assert np.array_equal(bm[0], bm[1]), "fused graph replay differs from the two-launch path"
        for v, (j, n, mir) in enumerate(variants):
            hits = W.expected_variant_hits(oracle, data["cs"], data["ms"], data["qc"][:, j], data["qm"][:, j],
                                           list(centred_rotations(n)), mir, np.arange(N_DB), 16384)
            assert np.nonzero(bm[1][v])[0].tolist() == hits, f"variant {v}"
    finally:
        if g is not None:
            g.close()
        _close(dcs + [c] + ce + me)


def test_fused_rejects_narrow_row_padding(dm, data):
    """The fused kernel's query tile is 128 rows: 64 padded rows are refused
    on the host, before any launch."""
    ce, me = _setup(dm, data, 64)
    c = irisb200.Circuits(dm, W.SEEDS)
    dc = irisb200.DistanceComparator(dm, 2, N_DB)
    try:
        slots = [(j, 0, 31, j) for j in range(2)]
        for p in range(3):
            ce[p].query_upload_slots(data["qc"][p][:2], slots)
            me[p].query_upload_slots(data["qm"][p][:2], slots)
        with pytest.raises(irisb200.IrisError) as ei:
            dc.scan_fused(c, ce, me, 0, 1024, 16384, n_slots=2)
        assert ei.value.code == -1 and "128" in str(ei.value)
        dm.synchronize()
    finally:
        _close([dc, c] + ce + me)


def test_plain_scan_every_candidate(dm, oracle, data):
    """PlainScan (the plain drop-in's autotuned DB pass) gives the CPU path's
    bitmap on every (path, tile, chunk) candidate, and tune() picks one of
    them."""
    from irisb200.scan import PlainScan
    ce, me = _setup(dm, data, N_Q * 32)
    c = irisb200.Circuits(dm, W.SEEDS)
    dc = irisb200.DistanceComparator(dm, N_Q, N_DB)
    try:
        slots = [(j, 0, 31, j) for j in range(N_Q)]
        for p in range(3):
            ce[p].query_upload_slots(data["qc"][p], slots)
            me[p].query_upload_slots(data["qm"][p], slots)
        exp = W.expected_bitmap(oracle, data["qc"], data["qm"], data["cs"], data["ms"], 16384)
        ps = PlainScan(dm, ce, me, c, dc, N_Q, N_DB, 16384)
        cands = ps.candidates()
        assert {p for p, _, _ in cands} == {"split", "pair", "fused"}
        # every candidate (one chunk at this DB size), then several chunks
        # with a ragged last one on each path (2000 = 3 x 640 + 80, 3 x 512 + 464)
        extra = [("split", 256, 640), ("pair", 256, 512), ("fused", 128, 640), ("split", 128, 512)]
        for cand in cands + extra:
            ps.configure(cand)
            dc.reset()
            ps.scan()
            dm.synchronize()
            got = irisb200.bitmap_get(dc.fetch_bitmap(N_Q, N_DB), N_Q, N_DB)
            assert np.array_equal(got, exp), f"candidate {cand}"
        # per-chunk timing of the configured path: one entry per timed pass
        for cand in (("pair", 256, 512), ("fused", 128, 640)):
            ps.configure(cand)
            ps.set_timing(2)
            for _ in range(3):  # the third pass is past the timing capacity
                dc.reset()
                ps.scan()
            g, t, whole = ps.timings()
            assert len(g) == len(t) == len(whole) == 2
            for x, y, z in zip(g, t, whole):
                assert x > 0 and z >= x + y - 1e-3
                # the fused launch is the chunk's whole work: nothing between its two later events
                assert y < 0.1 if cand[0] == "fused" else y > 0
            got = irisb200.bitmap_get(dc.fetch_bitmap(N_Q, N_DB), N_Q, N_DB)
            assert np.array_equal(got, exp), f"timed {cand}"
        # the tuner: every candidate once, the three fastest re-timed, the best
        # finalist mean configured; results unchanged afterwards
        best = ps.tune()
        n = len(cands)
        assert best in cands and len(ps.tune_log) == n + min(3, n) and ps.cand == best
        first = sorted(ps.tune_log[:n], key=lambda x: x[1])
        finals = ps.tune_log[n:]
        assert [cd for cd, _ in finals] == [cd for cd, _ in first[:3]]
        assert best == min(finals, key=lambda x: x[1])[0]
        dc.reset()
        ps.scan()
        dm.synchronize()
        got = irisb200.bitmap_get(dc.fetch_bitmap(N_Q, N_DB), N_Q, N_DB)
        assert np.array_equal(got, exp), f"tuned {best}"
        # restricted to one path: only that path's candidates are timed
        only = ps.tune(only_path="fused")
        assert only[0] == "fused" and {cd[0] for cd, _ in ps.tune_log} == {"fused"}
        ps.restore()
        ps.close()
    finally:
        _close([dc, c] + ce + me)
