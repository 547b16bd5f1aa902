"""Error paths of the C ABI: every call validates its arguments on the host
and returns a status (never aborts, never launches on bad input); the device
stays usable afterwards.  Inputs here are rejected before any GPU work."""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
import workload as W

pytestmark = pytest.mark.gpu


def _raises(fn, code=-1, text=None):
    with pytest.raises(irisb200.IrisError) as ei:
        fn()
    assert ei.value.code == code, str(ei.value)
    if text:
        assert text in str(ei.value)


def test_rejected_inputs_leave_the_device_usable(dm):
    e = irisb200.ShareDB(0, dm, 256, 64, 12800, W.SEEDS[0])
    m = irisb200.ShareDB(0, dm, 256, 64, 6400, W.SEEDS[0])
    dc = irisb200.DistanceComparator(dm, 2, 256)
    plain = irisb200.ShareDB(0, dm, 256, 64, 12800, W.SEEDS[0], is_remote=False)
    plain.alloc_db(256)
    try:
        # dot before alloc_db / query upload
        _raises(lambda: e.dot(0, 64), -4)
        e.alloc_db(256)
        m.alloc_db(256)
        _raises(lambda: e.dot(0, 64), -4, "no query")
        # records beyond the capacity; random fill beyond the capacity
        _raises(lambda: e.load_records(250, np.zeros((10, 12800), np.uint16)), -1, "capacity")
        _raises(lambda: e.fill_random(1, 300), -1)
        # row descriptors: source query out of range, rotation out of range
        base = np.zeros((2, 12800), np.uint16)
        _raises(lambda: e.query_upload_rows(base, np.array([(2 << 8) | 0], np.uint32)), -1, "descriptor")
        _raises(lambda: e.query_upload_rows(base, np.array([(0 << 8) | 31], np.uint32)), -1, "descriptor")
        # the resident pool: writes past the staging
        _raises(lambda: e.query_put_base(64, base), -1, "pool")
        # gathers: ids out of range, mismatched engines
        sub = irisb200.ShareDB(0, dm, 4, 64, 12800, W.SEEDS[0])
        sub.alloc_db(4)
        _raises(lambda: sub.gather_records(e, np.array([300], np.uint32)), -1, "out of range")
        _raises(lambda: sub.gather_records(m, np.array([0], np.uint32)), -1, "same party")
        # (the capacity is rounded up to whole 128-entry tiles)
        _raises(lambda: sub.gather_records(e, np.arange(129, dtype=np.uint32) % 256), -1, "capacity")
        sub.close()
        # comparator: rows out of range, captures not enabled, bad segment tables
        _raises(lambda: dc.take_rows(np.array([2], np.uint32), 10), -1, "out of range")
        _raises(lambda: dc.fetch_distances(), -4, "not enabled")
        _raises(lambda: dc.set_segments(np.array([1, 2], np.uint32), np.array([0], np.uint32),
                                        np.array([1], np.uint32)), -1, "seg_start[0]")
        _raises(lambda: dc.set_segments(np.array([0, 1], np.uint32), np.array([7], np.uint32),
                                        np.array([1], np.uint32)), -1, "query")
        _raises(lambda: dc.clear_rows(1, 5), -1)
        # tile widths and batch ids
        _raises(lambda: e.set_tile(96), -1, "tile width")
        _raises(lambda: e.set_batch(1 << 24), -1, "2^24")
        _raises(lambda: dm.set_batch_counter(1 << 24), -1, "2^24")
        # the device still runs a correct pass afterwards (engine without the
        # zero-share mask: results are the plain dots mod 2^16)
        rows = np.random.default_rng(1).integers(0, 65536, (64, 12800), dtype=np.uint16)
        db = np.random.default_rng(2).integers(0, 65536, (256, 12800), dtype=np.uint16)
        plain.query_upload(rows)
        plain.load_records(0, db)
        plain.dot(0, 256)
        got = plain.fetch_results(256)
        assert dm.error_code() == 0
        ref = (rows.astype(np.uint64) @ db.T.astype(np.uint64)) % 65536
        assert np.array_equal(got.astype(np.uint64), ref)
    finally:
        dc.close()
        for x in (e, m, plain):
            x.close()


def test_empty_inputs_are_no_ops(dm):
    """Zero-length work is accepted and changes nothing: a dot and a
    comparison over no entries, a compaction of no rows, an empty subset
    gather, and the final results of a batch that matched nothing."""
    ce = [irisb200.ShareDB(p, dm, 128, 64, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, 128, 64, 6400, W.SEEDS[p]) for p in range(3)]
    c = irisb200.Circuits(dm, W.SEEDS)
    dc = irisb200.DistanceComparator(dm, 2, 128)
    try:
        slots = [(0, 0, 31, 0), (0, 0, 31, 1)]
        for p in range(3):
            ce[p].alloc_db(128)
            me[p].alloc_db(128)
            ce[p].query_upload_slots(np.zeros((1, 12800), np.uint16), slots)
            me[p].query_upload_slots(np.zeros((1, 6400), np.uint16), slots)
        irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, 0)
        dc.compare_threshold_open(c, ce, me, 0, 0, 2, 16384)
        counts, ids = dc.take_rows(np.zeros(0, np.uint32), 0)
        assert counts.size == 0 and ids.shape[0] == 0
        sub = irisb200.ShareDB(0, dm, 4, 64, 12800, W.SEEDS[0])
        sub.alloc_db(4)
        sub.gather_records(ce[0], np.zeros(0, np.uint32))
        assert sub.db_len() == 0
        sub.close()
        dc.join_db_matches(2, 0)
        final, counters, _ = dc.fetch_final_results(2)
        assert (final == 0xFFFFFFFF).all() and (counters == 0).all()
        assert dm.error_code() == 0
    finally:
        dc.close()
        c.close()
        for e in ce + me:
            e.close()


def test_party_seed_ring_and_batch_counter(dm):
    """Cross-party consistency: the circuits refuse seeds that do not form the
    3-party ring (party p's second seed = party p-1's own seed); the device
    batch counter reads back for checkpoints and advances on the stream."""
    bad = [([0] * 8, [2] * 8), ([1] * 8, [9] * 8), ([2] * 8, [1] * 8)]
    _raises(lambda: irisb200.Circuits(dm, bad), -1, "seed1 of party 1")
    dm.set_batch_counter(123)
    assert dm.batch_counter() == 123
    dm.advance_batch_counter()
    dm.advance_batch_counter()
    assert dm.batch_counter() == 125
    dm.set_batch_counter((1 << 24) - 1)
    dm.advance_batch_counter()
    assert dm.batch_counter() == 1  # wraps past 2^24 - 1 to 1 (0 is never used)


def test_stage_timers(dm):
    """Debug stage timers: with timing on, each dot and threshold launch is
    timed on its stream; the sums read back per label and reset."""
    ce = [irisb200.ShareDB(p, dm, 256, 64, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, 256, 64, 6400, W.SEEDS[p]) for p in range(3)]
    c = irisb200.Circuits(dm, W.SEEDS)
    dc = irisb200.DistanceComparator(dm, 2, 256)
    try:
        slots = [(0, 0, 31, 0), (0, 0, 31, 1)]
        for p in range(3):
            ce[p].alloc_db(256)
            me[p].alloc_db(256)
            ce[p].fill_random(p, 256)
            me[p].fill_random(10 + p, 256)
            ce[p].query_upload_slots(np.ones((1, 12800), np.uint16), slots)
            me[p].query_upload_slots(np.ones((1, 6400), np.uint16), slots)
        dm.timings(reset=True)
        dm.set_timing(True)
        for _ in range(3):
            irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, 256)
            dc.compare_threshold_open(c, ce, me, 0, 256, 2, 16384)
        t = dm.timings(reset=True)
        assert t["dot"][1] == 3 and t["threshold_open"][1] == 3
        assert t["dot"][0] > 0 and t["threshold_open"][0] > 0
        dm.set_timing(False)
        irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, 256)
        assert dm.timings() == {}
    finally:
        dm.set_timing(False)
        dc.close()
        c.close()
        for e in ce + me:
            e.close()


def test_expired_bounded_wait_reports_and_device_recovers(dm, oracle):
    """The GEMM's bounded waits end in an error status, not a hang: with the
    test hook armed, the first CTA of the next dot issues no loads, so its MMA's
    stage wait runs out after 1 ms.  The kernel records
    DEV_ERR_TIMEOUT_FULL and returns; the next synchronising call fails with
    IRS_ERR_DEVICE (the reference panics on a stuck wait instead,
    iris-mpc-gpu/src/helpers/device_manager.rs:25-26,330-343); after
    clear_error the same engine's next dot equals the oracle."""
    rng = np.random.default_rng(11)
    n, q_len = 1024, 32
    db = rng.integers(0, 65535, (n, 12800)).astype(np.uint16)
    q = rng.integers(0, 65535, (q_len, 12800)).astype(np.uint16)
    e = irisb200.ShareDB(0, dm, n, q_len, 12800, W.SEEDS[0], is_remote=False)
    try:
        e.alloc_db(n)
        e.load_records(0, db)
        e.query_upload(q)
        dm.synchronize()
        assert dm.error_code() == 0
        dm.test_stall_next_dot(1_000_000)
        e.dot(0, n, 1)  # the launch itself succeeds
        with pytest.raises(irisb200.IrisError) as ei:
            dm.synchronize()
        assert ei.value.code == irisb200.IRS_ERR_DEVICE, str(ei.value)
        assert dm.error_code() == irisb200.DEV_ERR_TIMEOUT_FULL
        dm.clear_error()
        assert dm.error_code() == 0
        # the hook is one-shot: the next dot runs normally and is exact
        e.dot(0, n, 1)
        got = e.fetch_results(n)
        assert np.array_equal(got, oracle.dot_u16(q, db))
        dm.synchronize()
        # out-of-range limits are refused on the host
        _raises(lambda: dm.test_stall_next_dot(0), -1)
    finally:
        dm.clear_error()
        e.close()
