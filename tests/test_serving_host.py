"""Host-side logic of the continuous-batching server (no GPU): first-fit row
placement inside 32-row words, the row/segment tables it produces, and the
record split used by appends."""
from __future__ import annotations

import collections

import numpy as np

from irisb200.batched import centred_rotations
from irisb200.serving import ContinuousServer, _first_run, _Variant, split_record_i8


def test_first_run():
    assert _first_run(0, 32) == 0
    assert _first_run(0xFFFFFFFF, 1) == -1
    assert _first_run(0x7FFFFFFF, 1) == 31
    assert _first_run(0x7FFFFFFF, 2) == -1
    assert _first_run(0x0000FFFF, 16) == 16
    assert _first_run(0x00FF00FF, 8) == 8
    assert _first_run(0x00FF00FF, 9) == -1
    rng = np.random.default_rng(3)
    for _ in range(2000):
        occ = int(rng.integers(0, 1 << 32))
        n = int(rng.integers(1, 33))
        f = _first_run(occ, n)
        runs = [s for s in range(33 - n) if all(not (occ >> (s + k)) & 1 for k in range(n))]
        assert f == (runs[0] if runs else -1)


def _placer(n_slots):
    s = ContinuousServer.__new__(ContinuousServer)
    s.n_slot_cap = n_slots
    s.row_capacity = 32 * n_slots
    s.slot_occ = [0] * n_slots
    s.slot_vars = [[] for _ in range(n_slots)]
    return s


def test_placement_and_tables():
    s = _placer(4)
    vs = []
    for vid, n in enumerate([31, 16, 16, 1, 1, 31, 20]):
        where = s._place(n)
        assert where is not None
        v = _Variant(vid, False, list(centred_rotations(n)))
        s._occupy(v, *where)
        vs.append(v)
    assert [(v.slot, v.first) for v in vs] == [(0, 0), (1, 0), (1, 16), (0, 31), (2, 0), (2, 1), (3, 0)]
    assert s._place(13) is None and s._place(12) == (3, 20)
    row_desc, seg_start, seg_query, seg_mask = s._layout()
    assert row_desc.size == 128
    # every variant's rows carry its id and its centred rotations, and its segment mask covers exactly them
    for v in vs:
        rows = row_desc[v.slot * 32 + v.first: v.slot * 32 + v.first + len(v.rots)]
        assert ((rows >> 8) == v.vid).all() and ((rows & 0xFF) == np.array(v.rots)).all()
        segs = range(seg_start[v.slot], seg_start[v.slot + 1])
        k = [j for j in segs if seg_query[j] == v.vid]
        assert len(k) == 1 and seg_mask[k[0]] == (((1 << len(v.rots)) - 1) << v.first) & 0xFFFFFFFF
    used = np.zeros(128, bool)
    for v in vs:
        used[v.slot * 32 + v.first: v.slot * 32 + v.first + len(v.rots)] = True
    assert (row_desc[~used] == 0xFFFFFFFF).all()
    # releasing frees exactly the rows; the segment table shrinks to the last used
    # word while the row table stays padded towards the 256-row GEMM tile
    s._release(vs[6])
    assert s.slot_occ[3] == 0
    rd, st, _, _ = s._layout()
    assert st.size - 1 == 3 and rd.size == 128 and (rd[96:] == 0xFFFFFFFF).all()
    assert s._place(31) == (3, 0)


def test_admission_is_exact():
    s = _placer(2)
    s.free_variants = collections.deque(range(8))

    class R:
        kind = "uniqueness"
        n_rot = 31
        mirrored = True
    assert s.can_admit(R())
    R.n_rot = 17
    assert s.can_admit(R())  # one word each
    v = _Variant(0, False, list(range(17)))
    s._occupy(v, 0, 0)
    assert not s.can_admit(R())  # 15 rows left in word 0, one variant fits in word 1 only
    R.mirrored = False
    assert s.can_admit(R())
    assert s.slot_occ == [(1 << 17) - 1, 0]  # the probe left no trace


def test_split_record_i8_roundtrip():
    rng = np.random.default_rng(5)
    r = rng.integers(0, 65536, (2, 64)).astype(np.uint16)
    lo, hi = split_record_i8(r)
    assert lo.dtype == np.int8 and hi.dtype == np.int8
    back = ((lo.view(np.uint8) ^ 0x80).astype(np.uint16) | ((hi.view(np.uint8) ^ 0x80).astype(np.uint16) << 8))
    assert np.array_equal(back, r)


class _Fake:
    """Stands in for the device objects: records calls, returns empty matches."""

    def __init__(self):
        self.calls = collections.Counter()

    def __getattr__(self, name):
        def f(*a, **k):
            self.calls[name] += 1
        return f


class _FakeDC(_Fake):
    def take_rows_into(self, rows, db_len, counts, ids, clear=True):
        self.calls["take_rows"] += 1
        counts[: rows.size] = 0


class _Buf:
    def __init__(self, shape, dtype):
        self.array = np.zeros(shape, dtype)


def _fake_server(monkeypatch, db_len=1000, chunk=256, rows=128, max_variants=16):
    import irisb200.serving as S
    monkeypatch.setattr(S, "dot_many", lambda *a, **k: None)
    s = ContinuousServer.__new__(ContinuousServer)
    s.dm, s.c = _Fake(), _Fake()
    s.ce, s.me = [_Fake() for _ in range(3)], [_Fake() for _ in range(3)]
    s.dc = _FakeDC()
    s.A, s.chunk = 16384, chunk
    s.row_capacity = rows
    s.n_slot_cap = rows // 32
    s.slot_occ = [0] * s.n_slot_cap
    s.slot_vars = [[] for _ in range(s.n_slot_cap)]
    s.max_variants = max_variants
    s.db_len, s.db_capacity = db_len, db_len + 10
    s.free_variants = list(range(max_variants))
    s.pending_bases = set()
    s.max_reauth = 4
    monkeypatch.setattr(S, "PinnedArray", _Buf)
    monkeypatch.setattr(S, "Event", _Fake)
    s._alloc_host(2 * s.max_reauth)
    s.flight, s.layout_dirty, s.next_chunk, s.steps, s.rows_active = [], False, 0, 0, 0
    s.stats = collections.Counter()
    appended = []
    s.append = lambda code, mask: appended.append(s.db_len) or setattr(s, "db_len", s.db_len + 1)
    s._launch_reauth = lambda items: (lambda now: [S.Completion(i, a, now, S.Result(reauth_match=False))
                                                   for i, a, _ in items])
    return s, appended


def test_serve_loop_admission_and_append_barrier(monkeypatch):
    from irisb200.batched import Request
    s, appended = _fake_server(monkeypatch)
    zc, zm = np.zeros((3, 12800), np.uint16), np.zeros((3, 6400), np.uint16)
    reqs = [Request(code=zc, mask=zm, n_rot=31, mirrored=True) for _ in range(3)]        # 2 words each
    reqs += [Request(code=zc, mask=zm, n_rot=1), Request(code=None, mask=None, kind="append"),
             Request(code=zc, mask=zm, n_rot=1), Request(code=zc, mask=zm, kind="reauth", target=3)]
    admitted_at = {}
    orig_admit = ContinuousServer.admit

    def admit(self, r, idx, arrival):
        admitted_at[idx] = (self.steps, self.db_len)
        return orig_admit(self, r, idx, arrival)
    monkeypatch.setattr(ContinuousServer, "admit", admit)
    comps = s.serve([0.0] * len(reqs), reqs, appends={4: (None, None)})
    assert sorted(c.idx for c in comps) == list(range(len(reqs)))
    # 4 words: requests 0 and 1 fit, 2 waits; the 1-row request 3 passes it (bypass) ...
    assert admitted_at[0][0] == 0 and admitted_at[1][0] == 0 and admitted_at[3][0] == 0
    assert admitted_at[2][0] > 0
    # ... but the append waits behind request 2, and request 5 behind the append
    assert appended == [1000]
    assert admitted_at[2][1] == 1000 and admitted_at[5][1] == 1001
    # every uniqueness request visited all 4 chunks of its DB snapshot
    assert s.steps >= 8 and not s.flight and sorted(s.free_variants) == list(range(16))
    assert s.slot_occ == [0, 0, 0, 0]


def test_full_face_mirror_attack_rule():
    from irisb200.batched import Request, Result, full_face_mirror_attack
    u = Request(code=None, mask=None, mirrored=True)
    assert full_face_mirror_attack(u, Result(matches=[], mirror_matches=[7]))
    assert not full_face_mirror_attack(u, Result(matches=[3], mirror_matches=[7]))   # both matched
    assert not full_face_mirror_attack(u, Result(matches=[], mirror_matches=[]))
    r = Request(code=None, mask=None, mirrored=True, kind="reauth", target=1)
    assert not full_face_mirror_attack(r, Result(matches=[], mirror_matches=[7]))
    assert not full_face_mirror_attack(Request(code=None, mask=None), Result(matches=[], mirror_matches=[7]))


def test_async_host_mode_refuses_temporaries():
    """With host synchronisation off the library reads host buffers after the
    call returns: a list or a converted copy would be freed too early, so the
    bindings refuse it; with it on they convert as usual."""
    import pytest

    from irisb200 import _host_arg

    class _Dm:
        host_sync = True

    dm = _Dm()
    a = np.arange(8, dtype=np.uint32)
    assert _host_arg(dm, a, np.uint32) is a
    assert _host_arg(dm, [1, 2, 3], np.uint32).dtype == np.uint32
    assert _host_arg(dm, a.astype(np.int64), np.uint32).dtype == np.uint32
    dm.host_sync = False
    assert _host_arg(dm, a, np.uint32) is a
    assert _host_arg(dm, a[2:6], np.uint32).base is a
    for bad in ([1, 2, 3], a.astype(np.int64), a[::2]):
        with pytest.raises(ValueError):
            _host_arg(dm, bad, np.uint32)
