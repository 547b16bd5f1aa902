"""Host-side mirror of the iris-mpc GPU engines over the irisb200 C ABI.

The classes follow the reference's Rust call surface for the uniqueness hot
path -- ``ShareDB`` (iris-mpc-gpu/src/dot/share_db.rs), ``Circuits``
(iris-mpc-gpu/src/threshold_ring/protocol.rs) and ``DistanceComparator``
(iris-mpc-gpu/src/dot/distance_comparator.rs) -- with the three parties
co-resident on one B200.  Every call goes through ``libirisb200.so``; there is
no CPU fallback: importing this package on a machine without the built library
raises, and constructing a device manager without a B200 raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libirisb200.so")

IRIS_CODE_LENGTH = 12800
MASK_CODE_LENGTH = 6400
ROTATIONS = 31
SLOT_ROWS = 32
MAX_MATCHES_LEN = 256
THRESHOLD_A = 20316          # ratio 0.345 (iris-mpc-gpu/src/dot/mod.rs:12)
THRESHOLD_ANON_STATS_A = 16384  # ratio 0.375 (iris-mpc-gpu/src/dot/mod.rs:14)

IRS_OK = 0
IRS_ERR_OVERFLOW = -6
IRS_ERR_DEVICE = -5
# device error word codes (include/irisb200.h IRS_DEV_ERR_*)
DEV_ERR_TIMEOUT_FULL = 1
DEV_ERR_TIMEOUT_EMPTY = 2
DEV_ERR_TIMEOUT_ACC_FULL = 3
DEV_ERR_TIMEOUT_ACC_EMPTY = 4
DEV_ERR_TIMEOUT_DRAIN = 5


class IrisError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"irisb200 error {code}: {msg}")
        self.code = code


class QuerySlot(C.Structure):
    _fields_ = [("src", C.c_uint32), ("rot_lo", C.c_uint32), ("n_rot", C.c_uint32), ("query", C.c_uint32)]


SCAN_PATHS = ("split", "pair", "fused")  # IRS_SCAN_SPLIT, IRS_SCAN_PAIR, IRS_SCAN_FUSED


class ScanCandidate(C.Structure):
    _fields_ = [("path", C.c_int32), ("tile", C.c_int32), ("chunk", C.c_uint64)]


class ScanTiming(C.Structure):
    _fields_ = [("cand", ScanCandidate), ("ms", C.c_double), ("finalist", C.c_int32), ("reserved", C.c_int32)]


_vp = C.c_void_p
_sz = C.c_size_t
_u32 = C.c_uint32
_u64 = C.c_uint64
_i = C.c_int

# name -> argtypes (all return int status unless listed in _RESTYPES)
_SIGS = {
    "irs_last_error": [],
    "irs_version": [],
    "irs_device_manager_init": [_i, C.POINTER(_vp)],
    "irs_device_manager_destroy": [_vp],
    "irs_device_manager_stream": [_vp, _i, C.POINTER(_vp)],
    "irs_device_manager_synchronize": [_vp],
    "irs_device_manager_error": [_vp, C.POINTER(_i)],
    "irs_device_manager_clear_error": [_vp],
    "irs_device_manager_test_stall_next_dot": [_vp, _u64],
    "irs_device_manager_sm_count": [_vp, C.POINTER(_i)],
    "irs_device_manager_mem_info": [_vp, C.POINTER(_sz), C.POINTER(_sz)],
    "irs_device_manager_set_host_sync": [_vp, _i],
    "irs_event_create": [C.POINTER(_vp)],
    "irs_event_record": [_vp, _vp],
    "irs_event_synchronize": [_vp],
    "irs_event_query": [_vp, C.POINTER(_i)],
    "irs_event_destroy": [_vp],
    "irs_dc_clear_rows": [_vp, _sz, _sz, _vp],
    "irs_dc_take_rows": [_vp, _vp, _sz, _sz, _i, _vp, _vp],
    "irs_dc_enable_distance_capture": [_vp, _sz],
    "irs_dc_set_forced_distances": [_vp, _vp, _vp, _sz],
    "irs_dc_fetch_distances": [_vp, _sz, _vp, _vp, _vp, _vp, C.POINTER(_sz), _i],
    "irs_dc_fetch_rows": [_vp, _sz, _sz, _vp, _sz, C.POINTER(_sz)],
    "irs_device_alloc": [_vp, _sz, C.POINTER(_vp)],
    "irs_device_free": [_vp, _vp],
    "irs_host_alloc_pinned": [_sz, C.POINTER(_vp)],
    "irs_host_free_pinned": [_vp],
    "irs_preprocess_query_share": [_i, _vp, _sz],
    "irs_synth_queries": [_u64, _u64, _sz, _vp, _vp, _i, _vp, _vp],
    "irs_encode_iris": [_vp, _vp, _u64, _i, _vp, _vp],
    "irs_copy_h2d": [_vp, _vp, _sz, _vp],
    "irs_copy_d2h": [_vp, _vp, _sz, _vp],
    "irs_stream_synchronize": [_vp],
    "irs_sharedb_init": [_vp, _i, _sz, _sz, _sz, _vp, _vp, _i, C.POINTER(_vp)],
    "irs_sharedb_destroy": [_vp],
    "irs_sharedb_alloc_db": [_vp, _sz],
    "irs_sharedb_load_records": [_vp, _sz, _sz, _vp],
    "irs_sharedb_load_records_i8": [_vp, _sz, _sz, _vp, _vp],
    "irs_sharedb_fetch_records": [_vp, _sz, _sz, _vp],
    "irs_sharedb_set_db_len": [_vp, _sz],
    "irs_sharedb_db_len": [_vp, C.POINTER(_sz)],
    "irs_sharedb_synth_db": [_vp, _vp, _u64, _sz, _sz],
    "irs_sharedb_query_upload": [_vp, _vp, _sz],
    "irs_sharedb_query_upload_slots": [_vp, _vp, _sz, _vp, _sz],
    "irs_sharedb_set_batch": [_vp, _u64],
    "irs_sharedb_set_tile": [_vp, _i],
    "irs_sharedb_set_pair": [_vp, _i],
    "irs_sharedb_use_batch_counter": [_vp, _i],
    "irs_circuits_use_batch_counter": [_vp, _i],
    "irs_device_manager_set_batch_counter": [_vp, _u64, _vp],
    "irs_device_manager_advance_batch_counter": [_vp, _vp],
    "irs_device_manager_get_batch_counter": [_vp, C.POINTER(_u64)],
    "irs_device_manager_set_timing": [_vp, _i],
    "irs_device_manager_timings": [_vp, _vp, _sz, _i],
    "irs_sharedb_query_upload_rows": [_vp, _vp, _sz, _vp, _sz],
    "irs_sharedb_gather_records": [_vp, _vp, _vp, _sz],
    "irs_sharedb_fill_random": [_vp, _u64, _sz],
    "irs_device_fill_random": [_vp, _sz, _u64, _vp],
    "irs_sharedb_query_put_base": [_vp, _sz, _sz, _vp],
    "irs_sharedb_query_expand_rows": [_vp, _sz, _vp, _sz],
    "irs_mirror_query_share": [_vp, _sz, _i],
    "irs_dc_set_segments": [_vp, _sz, _vp, _vp, _vp],
    "irs_dc_compare_threshold_open_prepared": [_vp, _vp, _vp, _vp, _sz, _sz, _u32, _i, _vp],
    "irs_dc_scan_fused": [_vp, _vp, _vp, _vp, _sz, _sz, _sz, _u32, _i, _vp],
    "irs_scan_init": [_vp, _vp, _vp, _vp, _vp, _sz, _sz, _u32, C.POINTER(_vp)],
    "irs_scan_destroy": [_vp],
    "irs_scan_candidates": [_vp, C.POINTER(ScanCandidate), _sz, C.POINTER(_sz)],
    "irs_scan_set_rows": [_vp, _sz, _i],
    "irs_scan_configure": [_vp, _i, _i, _sz],
    "irs_scan_current": [_vp, C.POINTER(ScanCandidate)],
    "irs_scan_run": [_vp, _vp],
    "irs_scan_set_timing": [_vp, _sz],
    "irs_scan_timings": [_vp, _vp, _vp, _vp, _sz, C.POINTER(_sz), _i],
    "irs_scan_tune": [_vp, _i, _i, _i, _i, C.POINTER(ScanCandidate), C.POINTER(ScanTiming), _sz, C.POINTER(_sz)],
    "irs_scan_restore": [_vp],
    "irs_graph_begin_capture": [_vp],
    "irs_graph_end_capture": [_vp, C.POINTER(_vp)],
    "irs_graph_launch": [_vp, _vp],
    "irs_graph_destroy": [_vp],
    "irs_sharedb_dot": [_vp, _sz, _sz, C.c_uint16, _vp],
    "irs_sharedb_dot_many": [_vp, _vp, _i, _sz, _sz, _vp],
    "irs_sharedb_fetch_results": [_vp, _vp, _sz],
    "irs_sharedb_result_view": [_vp, C.POINTER(_vp), C.POINTER(_sz)],
    "irs_circuits_new": [_vp, _vp, C.POINTER(_vp)],
    "irs_circuits_destroy": [_vp],
    "irs_circuits_set_batch": [_vp, _u64],
    "irs_circuits_compare_threshold_masked_many": [_vp, _vp, _vp, _sz, _u32, _vp, _vp, _vp, _vp],
    "irs_circuits_compare_threshold_masked_many_noalloc": [_vp, _vp, _vp, _sz, _u32, _vp, _vp, _vp, _vp],
    "irs_circuits_extract_msb_of_code": [_vp, _vp, _sz, _vp, _vp, _vp, _vp],
    "irs_circuits_lift_mpc": [_vp, _vp, _sz, _vp, _vp],
    "irs_circuits_or_reduce": [_vp, _vp, _sz, _vp, _vp],
    "irs_circuits_compare_threshold_masked_many_with_or_tree": [_vp, _vp, _vp, _sz, _u32, _vp, _vp],
    "irs_dc_init": [_vp, _sz, _sz, _sz, C.POINTER(_vp)],
    "irs_dc_destroy": [_vp],
    "irs_dc_reset": [_vp, _vp],
    "irs_dc_compare_threshold_open": [_vp, _vp, _vp, _vp, _sz, _sz, _sz, _vp, _vp, _u32, _i, _vp],
    "irs_dc_fetch_bitmap": [_vp, _sz, _sz, _vp],
    "irs_dc_fetch_matches": [_vp, _vp, _sz, C.POINTER(_sz)],
    "irs_dc_get_partial_results": [_vp, _sz, _sz, _vp, _sz, C.POINTER(_sz)],
    "irs_dc_join_db_matches": [_vp, _vp, _vp, _sz, _sz, _vp],
    "irs_dc_join_batch_matches": [_vp, _vp, _sz, _vp],
    "irs_dc_fetch_final_results": [_vp, _sz, _vp, _vp, _vp],
}
_RESTYPES = {"irs_last_error": C.c_char_p, "irs_version": C.c_char_p}

_LIB = None


def lib() -> C.CDLL:
    """Loads libirisb200.so; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run iris-mpc_b200/build.py (the CUDA library is required)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, C.c_int)
        _LIB = L
    return _LIB


def exported_symbols() -> list[str]:
    return list(_SIGS.keys())


def _check(rc: int, allow=()) -> int:
    if rc != IRS_OK and rc not in allow:
        raise IrisError(rc, lib().irs_last_error().decode(errors="replace"))
    return rc


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _host_arg(dm, a, dtype) -> np.ndarray:
    """A host buffer for a call that may only enqueue its copy: with the
    device manager's host synchronisation off the library reads the buffer
    after the call returns, so a converted temporary copy would be freed too
    early -- such calls take the caller's own C-contiguous array or fail."""
    if getattr(dm, "host_sync", True):
        return np.ascontiguousarray(a, dtype)
    if not isinstance(a, np.ndarray) or a.dtype != np.dtype(dtype) or not a.flags.c_contiguous:
        raise ValueError("with host synchronisation off, pass a C-contiguous %s array that stays alive and "
                         "unchanged until the work has run (page-locked memory: PinnedArray)" % np.dtype(dtype))
    return a


def _seed(s) -> np.ndarray:
    return np.ascontiguousarray(np.array(s, dtype=np.uint32).reshape(8))


class DeviceBuffer:
    """A plain device allocation (for callers staging their own shares)."""

    def __init__(self, dm: "DeviceManager", nbytes: int):
        self.dm = dm
        self.nbytes = nbytes
        p = _vp()
        _check(lib().irs_device_alloc(dm.h, nbytes, C.byref(p)))
        self.ptr = p.value

    @classmethod
    def from_array(cls, dm: "DeviceManager", a: np.ndarray) -> "DeviceBuffer":
        a = np.ascontiguousarray(a)
        b = cls(dm, a.nbytes)
        b.upload(a)
        return b

    def upload(self, a: np.ndarray, stream=None) -> None:
        a = np.ascontiguousarray(a)
        assert a.nbytes <= self.nbytes
        _check(lib().irs_copy_h2d(self.ptr, _ptr(a), a.nbytes, stream))
        _check(lib().irs_stream_synchronize(stream))

    def download(self, dtype, count: int, stream=None) -> np.ndarray:
        out = np.zeros(count, dtype)
        _check(lib().irs_copy_d2h(_ptr(out), self.ptr, out.nbytes, stream))
        _check(lib().irs_stream_synchronize(stream))
        return out

    def fill_random(self, seed: int, stream=None) -> None:
        _check(lib().irs_device_fill_random(self.ptr, self.nbytes // 8 * 8, seed, stream))

    def free(self) -> None:
        if self.ptr:
            lib().irs_device_free(self.dm.h, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PinnedArray:
    """A numpy array over page-locked host memory (cudaMallocHost)."""

    def __init__(self, shape, dtype):
        dtype = np.dtype(dtype)
        n = int(np.prod(shape)) * dtype.itemsize
        p = _vp()
        _check(lib().irs_host_alloc_pinned(n, C.byref(p)))
        self._p = p.value
        buf = (C.c_uint8 * n).from_address(self._p)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self) -> None:
        if self._p:
            self.array = None
            lib().irs_host_free_pinned(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def preprocess_query_share(party: int, coefs: np.ndarray) -> np.ndarray:
    """Lagrange x basis-B preprocessing of a query share (galois_engine.rs:23-40)."""
    out = np.ascontiguousarray(coefs, np.uint16).copy()
    _check(lib().irs_preprocess_query_share(party, _ptr(out), out.size))
    return out


def mirror_query_share(coefs: np.ndarray, flip_imaginary: bool) -> np.ndarray:
    """mirrored_code (flip_imaginary) / mirrored_mask of a query share."""
    out = np.ascontiguousarray(coefs, np.uint16).copy()
    _check(lib().irs_mirror_query_share(_ptr(out), out.size, int(flip_imaginary)))
    return out


class Graph:
    """A captured CUDA graph of device work issued on party 0's stream."""

    def __init__(self, h):
        self.h = h

    @staticmethod
    def capture(dm: "DeviceManager", fn) -> "Graph":
        _check(lib().irs_graph_begin_capture(dm.h))
        try:
            fn()
        finally:
            g = _vp()
            rc = lib().irs_graph_end_capture(dm.h, C.byref(g))
        _check(rc)
        return Graph(g.value)

    def launch(self, stream=None) -> None:
        _check(lib().irs_graph_launch(self.h, stream))

    def close(self) -> None:
        if self.h:
            lib().irs_graph_destroy(self.h)
            self.h = None


def encode_iris(code_bits: np.ndarray, mask_bits: np.ndarray, seed: int, preprocess: bool = False):
    """The three parties' shares of one iris (irs_encode_iris): code_bits /
    mask_bits are u64 [200] (12800 bits).  Returns (code [3][12800], mask
    [3][6400]) u16: DB records, or query shares when preprocess."""
    c = np.ascontiguousarray(code_bits, np.uint64).reshape(200)
    m = np.ascontiguousarray(mask_bits, np.uint64).reshape(200)
    code = np.zeros((3, IRIS_CODE_LENGTH), np.uint16)
    mask = np.zeros((3, MASK_CODE_LENGTH), np.uint16)
    _check(lib().irs_encode_iris(_ptr(c), _ptr(m), seed, int(preprocess), _ptr(code), _ptr(mask)))
    return code, mask


def deletion_record(seed: int = 0):
    """Shares of the default iris (all-zero code, full mask) that a deletion
    writes over a DB record (get_dummy_shares_for_deletion,
    iris-mpc-common/src/iris_db/mod.rs:10-23): it matches no real query."""
    return encode_iris(np.zeros(200, np.uint64), np.full(200, 0xFFFFFFFFFFFFFFFF, np.uint64), seed)


def delete_records(code_engines, mask_engines, indices, seed: int = 0) -> None:
    """Deletions (actor.rs:2641-2680): the deletion record over each index of
    the six engines (party p code at code_engines[p], mask at mask_engines[p])."""
    code, mask = deletion_record(seed)
    for idx in indices:
        for p in range(3):
            code_engines[p].load_records(int(idx), code[p][None])
            mask_engines[p].load_records(int(idx), mask[p][None])


def synth_queries(db_seed: int, q_seed: int, n_queries: int, planted: dict, preprocess: bool = True,
                  code_out: np.ndarray = None, mask_out: np.ndarray = None):
    """Seeded synthetic query shares; planted = {query: (db entry, rotation)}.
    Returns (code [3][n][12800], mask [3][n][6400]) u16."""
    pe = np.full(n_queries, -1, np.int64)
    pr = np.zeros(n_queries, np.int32)
    for j, (e, r) in planted.items():
        pe[j] = e
        pr[j] = r
    code = code_out if code_out is not None else np.zeros((3, n_queries, IRIS_CODE_LENGTH), np.uint16)
    mask = mask_out if mask_out is not None else np.zeros((3, n_queries, MASK_CODE_LENGTH), np.uint16)
    assert code.shape == (3, n_queries, IRIS_CODE_LENGTH) and code.flags.c_contiguous
    assert mask.shape == (3, n_queries, MASK_CODE_LENGTH) and mask.flags.c_contiguous
    _check(lib().irs_synth_queries(db_seed, q_seed, n_queries, _ptr(pe), _ptr(pr), int(preprocess), _ptr(code),
                                   _ptr(mask)))
    return code, mask


class Event:
    """A CUDA event (no timing) for the asynchronous host mode."""

    def __init__(self):
        p = _vp()
        _check(lib().irs_event_create(C.byref(p)))
        self.h = p.value

    def record(self, stream=None) -> None:
        _check(lib().irs_event_record(self.h, stream))

    def synchronize(self) -> None:
        _check(lib().irs_event_synchronize(self.h))

    def done(self) -> bool:
        d = _i()
        _check(lib().irs_event_query(self.h, C.byref(d)))
        return bool(d.value)

    def close(self) -> None:
        if self.h:
            lib().irs_event_destroy(self.h)
            self.h = None


class DeviceManager:
    """DeviceManager (iris-mpc-gpu/src/helpers/device_manager.rs) for one GPU
    hosting the three parties, each with its own stream and memory pool."""

    def __init__(self, device: int = 0):
        h = _vp()
        _check(lib().irs_device_manager_init(device, C.byref(h)))
        self.h = h.value
        self.device = device
        self.host_sync = True

    def stream(self, party: int):
        s = _vp()
        _check(lib().irs_device_manager_stream(self.h, party, C.byref(s)))
        return s.value

    def synchronize(self) -> None:
        _check(lib().irs_device_manager_synchronize(self.h))

    def error_code(self) -> int:
        c = C.c_int()
        _check(lib().irs_device_manager_error(self.h, C.byref(c)))
        return c.value

    def clear_error(self) -> None:
        _check(lib().irs_device_manager_clear_error(self.h))

    def test_stall_next_dot(self, wait_limit_ns: int) -> None:
        """Test hook: the next dot launch runs with this bounded-wait limit and
        its first CTA loads nothing, so that CTA's stage wait runs out and the
        kernel records DEV_ERR_TIMEOUT_FULL (irs_device_manager_test_stall_next_dot)."""
        _check(lib().irs_device_manager_test_stall_next_dot(self.h, int(wait_limit_ns)))

    def set_batch_counter(self, batch_id: int, stream=None) -> None:
        _check(lib().irs_device_manager_set_batch_counter(self.h, batch_id, stream))

    def set_timing(self, on: bool) -> None:
        """Stage timers on the dot and threshold launches (debug timing)."""
        _check(lib().irs_device_manager_set_timing(self.h, int(on)))

    def timings(self, reset: bool = True) -> dict:
        """{label: (total ms, launches)} of the stage timers."""
        buf = C.create_string_buffer(4096)
        _check(lib().irs_device_manager_timings(self.h, buf, len(buf), int(reset)))
        out = {}
        for item in filter(None, buf.value.decode().split(";")):
            name, v = item.split("=")
            ms, n = v.split("/")
            out[name] = (float(ms), int(n))
        return out

    def batch_counter(self) -> int:
        v = _u64()
        _check(lib().irs_device_manager_get_batch_counter(self.h, C.byref(v)))
        return v.value

    def advance_batch_counter(self, stream=None) -> None:
        _check(lib().irs_device_manager_advance_batch_counter(self.h, stream))

    def set_host_sync(self, on: bool) -> None:
        """See irs_device_manager_set_host_sync: off = enqueue-only calls on pinned host buffers."""
        _check(lib().irs_device_manager_set_host_sync(self.h, int(on)))
        self.host_sync = bool(on)

    def mem_info(self):
        f, t = _sz(), _sz()
        _check(lib().irs_device_manager_mem_info(self.h, C.byref(f), C.byref(t)))
        return f.value, t.value

    def sm_count(self) -> int:
        c = C.c_int()
        _check(lib().irs_device_manager_sm_count(self.h, C.byref(c)))
        return c.value

    def close(self) -> None:
        if self.h:
            lib().irs_device_manager_destroy(self.h)
            self.h = None


class ShareDB:
    """ShareDB (iris-mpc-gpu/src/dot/share_db.rs:448-1070) of one party."""

    def __init__(self, peer_id: int, dm: DeviceManager, max_db_length: int, query_length: int, code_length: int,
                 chacha_seeds, is_remote: bool = True):
        h = _vp()
        s0, s1 = _seed(chacha_seeds[0]), _seed(chacha_seeds[1])
        _check(lib().irs_sharedb_init(dm.h, peer_id, max_db_length, query_length, code_length, _ptr(s0), _ptr(s1),
                                      int(is_remote), C.byref(h)))
        self.h = h.value
        self.dm = dm
        self.peer_id = peer_id
        self.query_length = query_length
        self.code_length = code_length

    def alloc_db(self, max_db_length: int) -> None:
        _check(lib().irs_sharedb_alloc_db(self.h, max_db_length))

    def load_records(self, first: int, records: np.ndarray) -> None:
        r = np.ascontiguousarray(records, np.uint16).reshape(-1, self.code_length)
        _check(lib().irs_sharedb_load_records(self.h, first, r.shape[0], _ptr(r)))

    def load_records_i8(self, first: int, limb0: np.ndarray, limb1: np.ndarray) -> None:
        a = np.ascontiguousarray(limb0).view(np.uint8).reshape(-1, self.code_length)
        b = np.ascontiguousarray(limb1).view(np.uint8).reshape(-1, self.code_length)
        _check(lib().irs_sharedb_load_records_i8(self.h, first, a.shape[0], _ptr(a), _ptr(b)))

    def fetch_records(self, first: int, n: int) -> np.ndarray:
        out = np.zeros((n, self.code_length), np.uint16)
        _check(lib().irs_sharedb_fetch_records(self.h, first, n, _ptr(out)))
        return out

    def set_db_len(self, n: int) -> None:
        _check(lib().irs_sharedb_set_db_len(self.h, n))

    def db_len(self) -> int:
        n = _sz()
        _check(lib().irs_sharedb_db_len(self.h, C.byref(n)))
        return n.value

    def query_upload(self, rows: np.ndarray) -> None:
        r = np.ascontiguousarray(rows, np.uint16).reshape(-1, self.code_length)
        _check(lib().irs_sharedb_query_upload(self.h, _ptr(r), r.shape[0]))

    def query_upload_slots(self, base: np.ndarray, slots) -> None:
        b = np.ascontiguousarray(base, np.uint16).reshape(-1, self.code_length)
        arr = (QuerySlot * len(slots))(*[QuerySlot(*s) for s in slots])
        _check(lib().irs_sharedb_query_upload_slots(self.h, _ptr(b), b.shape[0], C.cast(arr, _vp), len(slots)))

    def set_batch(self, batch_id: int) -> None:
        _check(lib().irs_sharedb_set_batch(self.h, batch_id))

    def set_pair(self, on: bool) -> None:
        """Two-SM GEMM for the 256-row tile (irs_sharedb_set_pair)."""
        _check(lib().irs_sharedb_set_pair(self.h, int(on)))

    def set_tile(self, block_n: int) -> None:
        _check(lib().irs_sharedb_set_tile(self.h, block_n))

    def use_batch_counter(self, on: bool = True) -> None:
        _check(lib().irs_sharedb_use_batch_counter(self.h, int(on)))

    def query_upload_rows(self, base: np.ndarray, row_desc) -> None:
        """Rows row_desc[r] = (src << 8) | rotation, 0xFFFFFFFF = empty."""
        b = _host_arg(self.dm, base, np.uint16).reshape(-1, self.code_length)
        rd = _host_arg(self.dm, row_desc, np.uint32)
        _check(lib().irs_sharedb_query_upload_rows(self.h, _ptr(b), b.shape[0], _ptr(rd), rd.size))

    def query_put_base(self, first: int, base: np.ndarray) -> None:
        """Writes base queries [first, first + len(base)) of the resident pool."""
        b = _host_arg(self.dm, base, np.uint16).reshape(-1, self.code_length)
        _check(lib().irs_sharedb_query_put_base(self.h, first, b.shape[0], _ptr(b)))

    def query_expand_rows(self, n_base: int, row_desc) -> None:
        """query_upload_rows over the resident pool [0, n_base)."""
        rd = _host_arg(self.dm, row_desc, np.uint32)
        _check(lib().irs_sharedb_query_expand_rows(self.h, n_base, _ptr(rd), rd.size))

    def fill_random(self, seed: int, n: int) -> None:
        """Records 0..n-1 filled with seeded uniform limb bytes (benchmark DB)."""
        _check(lib().irs_sharedb_fill_random(self.h, seed, n))

    def gather_records(self, src: "ShareDB", ids) -> None:
        """prefetch_subset: records ids[k] of src become records k of this engine."""
        i = _host_arg(self.dm, ids, np.uint32)
        _check(lib().irs_sharedb_gather_records(self.h, src.h, _ptr(i), i.size))

    def dot(self, offset: int, length: int, multiplier: int = 1, stream=None) -> None:
        """dot + dot_reduce_and_multiply (share_db.rs:800-905), fused."""
        _check(lib().irs_sharedb_dot(self.h, offset, length, multiplier, stream))

    def fetch_results(self, length: int) -> np.ndarray:
        out = np.zeros((self.query_length, length), np.uint16)
        _check(lib().irs_sharedb_fetch_results(self.h, _ptr(out), length))
        return out

    def result_view(self):
        p = _vp()
        s = _sz()
        _check(lib().irs_sharedb_result_view(self.h, C.byref(p), C.byref(s)))
        return p.value, s.value

    def close(self) -> None:
        if self.h:
            lib().irs_sharedb_destroy(self.h)
            self.h = None


def dot_many(engines, multipliers, offset: int, length: int, stream=None) -> None:
    """One tcgen05 launch for several engines (e.g. 3 parties x code/mask)."""
    hs = (_vp * len(engines))(*[e.h for e in engines])
    ms = (C.c_uint16 * len(engines))(*multipliers)
    _check(lib().irs_sharedb_dot_many(C.cast(hs, _vp), C.cast(ms, _vp), len(engines), offset, length, stream))


def synth_db(code_engines, mask_engines, seed: int, first: int, n: int) -> None:
    hc = (_vp * 3)(*[e.h for e in code_engines])
    hm = (_vp * 3)(*[e.h for e in mask_engines])
    _check(lib().irs_sharedb_synth_db(C.cast(hc, _vp), C.cast(hm, _vp), seed, first, n))


def _ptr3(xs):
    return C.cast((_vp * 3)(*[x if isinstance(x, int) else x.ptr for x in xs]), _vp)


class Circuits:
    """Circuits (iris-mpc-gpu/src/threshold_ring/protocol.rs:433-2611) of the
    three co-resident parties.  seeds[p] = party p's (seed0, seed1)."""

    def __init__(self, dm: DeviceManager, seeds):
        arr = np.ascontiguousarray(np.array(seeds, dtype=np.uint32).reshape(3, 2, 8))
        h = _vp()
        _check(lib().irs_circuits_new(dm.h, _ptr(arr), C.byref(h)))
        self.h = h.value
        self.dm = dm

    def set_batch(self, batch_id: int) -> None:
        _check(lib().irs_circuits_set_batch(self.h, batch_id))

    def use_batch_counter(self, on: bool = True) -> None:
        _check(lib().irs_circuits_use_batch_counter(self.h, int(on)))

    def compare_threshold_masked_many(self, code_a, mask_a, n: int, threshold_a: int, res_a=None, res_b=None,
                                      opened=None, stream=None) -> None:
        _check(lib().irs_circuits_compare_threshold_masked_many(
            self.h, _ptr3(code_a), _ptr3(mask_a), n, threshold_a,
            _ptr3(res_a) if res_a else None, _ptr3(res_b) if res_b else None,
            opened.ptr if opened else None, stream))

    def extract_msb_of_code(self, code_a, n: int, res_a=None, res_b=None, opened=None, stream=None) -> None:
        _check(lib().irs_circuits_extract_msb_of_code(
            self.h, _ptr3(code_a), n, _ptr3(res_a) if res_a else None, _ptr3(res_b) if res_b else None,
            opened.ptr if opened else None, stream))

    def or_reduce(self, res_a, n: int, stream=None):
        """(party a-shares [3] of the OR bit, opened bit) of n result bits."""
        out = np.zeros(4, np.uint32)
        _check(lib().irs_circuits_or_reduce(self.h, _ptr3(res_a), n, _ptr(out), stream))
        return out[:3].copy(), int(out[3])

    def compare_threshold_masked_many_with_or_tree(self, code_a, mask_a, n: int, threshold_a: int, stream=None):
        out = np.zeros(4, np.uint32)
        _check(lib().irs_circuits_compare_threshold_masked_many_with_or_tree(
            self.h, _ptr3(code_a), _ptr3(mask_a), n, threshold_a, _ptr(out), stream))
        return out[:3].copy(), int(out[3])

    def lift_mpc(self, mask_a, n: int, corr, stream=None) -> None:
        _check(lib().irs_circuits_lift_mpc(self.h, _ptr3(mask_a), n, _ptr3(corr), stream))

    def close(self) -> None:
        if self.h:
            lib().irs_circuits_destroy(self.h)
            self.h = None


class DistanceComparator:
    """DistanceComparator (iris-mpc-gpu/src/dot/distance_comparator.rs)."""

    def __init__(self, dm: DeviceManager, max_queries: int, max_db_length: int, match_list_cap: int = 1 << 20):
        h = _vp()
        _check(lib().irs_dc_init(dm.h, max_queries, max_db_length, match_list_cap, C.byref(h)))
        self.h = h.value
        self.dm = dm
        self.max_queries = max_queries

    def reset(self, stream=None) -> None:
        _check(lib().irs_dc_reset(self.h, stream))

    def compare_threshold_open(self, circuits: Circuits, code_engines, mask_engines, offset: int, length: int,
                               n_slots: int, threshold_a: int, slot_valid=None, slot_query=None,
                               self_check: bool = False, stream=None) -> None:
        hc = (_vp * 3)(*[e.h for e in code_engines])
        hm = (_vp * 3)(*[e.h for e in mask_engines])
        sv = np.ascontiguousarray(slot_valid, np.uint32) if slot_valid is not None else None
        sq = np.ascontiguousarray(slot_query, np.uint32) if slot_query is not None else None
        _check(lib().irs_dc_compare_threshold_open(
            self.h, circuits.h, C.cast(hc, _vp), C.cast(hm, _vp), offset, length, n_slots,
            _ptr(sv) if sv is not None else None, _ptr(sq) if sq is not None else None, threshold_a,
            int(self_check), stream))

    def set_segments(self, seg_start, seg_query, seg_mask) -> None:
        st = _host_arg(self.dm, seg_start, np.uint32)
        sq = _host_arg(self.dm, seg_query, np.uint32)
        sm = _host_arg(self.dm, seg_mask, np.uint32)
        _check(lib().irs_dc_set_segments(self.h, st.size - 1, _ptr(st), _ptr(sq) if sq.size else None,
                                         _ptr(sm) if sm.size else None))

    def compare_threshold_open_prepared(self, circuits: Circuits, code_engines, mask_engines, offset: int,
                                        length: int, threshold_a: int, self_check: bool = False,
                                        stream=None) -> None:
        hc = (_vp * 3)(*[e.h for e in code_engines])
        hm = (_vp * 3)(*[e.h for e in mask_engines])
        _check(lib().irs_dc_compare_threshold_open_prepared(self.h, circuits.h, C.cast(hc, _vp), C.cast(hm, _vp),
                                                            offset, length, threshold_a, int(self_check), stream))

    def scan_fused(self, circuits: Circuits, code_engines, mask_engines, offset: int, length: int,
                   threshold_a: int, n_slots: int = 0, use_segments: bool = False, stream=None) -> None:
        """The six limb GEMMs and the threshold/open/rotation OR of entries
        [offset, offset + length) in one persistent kernel (irs_dc_scan_fused):
        plain 32-row slots 0..n_slots-1, or the stored segment table."""
        hc = (_vp * 3)(*[e.h for e in code_engines])
        hm = (_vp * 3)(*[e.h for e in mask_engines])
        _check(lib().irs_dc_scan_fused(self.h, circuits.h, C.cast(hc, _vp), C.cast(hm, _vp), offset, length, n_slots,
                                       threshold_a, int(use_segments), stream))

    def take_rows(self, rows, db_len: int, clear: bool = True):
        """(counts [n], ids [n][256]) of the listed bitmap rows; see irs_dc_take_rows."""
        r = np.ascontiguousarray(rows, np.uint32)
        counts = np.zeros(max(r.size, 1), np.uint32)
        ids = np.zeros((max(r.size, 1), MAX_MATCHES_LEN), np.uint32)
        _check(lib().irs_dc_take_rows(self.h, _ptr(r) if r.size else None, r.size, db_len, int(clear), _ptr(counts),
                                      _ptr(ids)))
        return counts[: r.size], ids[: r.size]

    def enable_distance_capture(self, cap: int) -> None:
        _check(lib().irs_dc_enable_distance_capture(self.h, cap))

    def set_forced_distances(self, pairs) -> None:
        """(query, entry) pairs captured on every valid row, match or not."""
        q = np.ascontiguousarray([p[0] for p in pairs], np.uint32)
        e = np.ascontiguousarray([p[1] for p in pairs], np.uint32)
        _check(lib().irs_dc_set_forced_distances(self.h, _ptr(q) if q.size else None, _ptr(e) if e.size else None,
                                                 q.size))

    def fetch_distances(self, cap: int = 1 << 16, reset: bool = True):
        """(entry [n], row [n], code [3][n], mask [3][n], total captured)."""
        entry = np.zeros(cap, np.uint32)
        row = np.zeros(cap, np.uint32)
        code = np.zeros((3, cap), np.uint16)
        mask = np.zeros((3, cap), np.uint16)
        n = _sz()
        _check(lib().irs_dc_fetch_distances(self.h, cap, _ptr(entry), _ptr(row), _ptr(code), _ptr(mask), C.byref(n),
                                            int(reset)))
        k = min(n.value, cap)
        return entry[:k], row[:k], code[:, :k], mask[:, :k], n.value

    def take_rows_into(self, rows: np.ndarray, db_len: int, counts: np.ndarray, ids: np.ndarray,
                       clear: bool = True) -> None:
        """irs_dc_take_rows into caller-owned arrays (page-locked, and read only
        after the stream has passed the call, in the asynchronous host mode)."""
        for a, dt in ((rows, np.uint32), (counts, np.uint32), (ids, np.uint32)):
            if a.dtype != dt or not a.flags.c_contiguous:
                raise ValueError("take_rows_into needs contiguous uint32 arrays")
        if counts.size < rows.size or ids.shape[0] < rows.size or ids.shape[1] != MAX_MATCHES_LEN:
            raise ValueError("output arrays too small")
        _check(lib().irs_dc_take_rows(self.h, _ptr(rows), rows.size, db_len, int(clear), _ptr(counts), _ptr(ids)))

    def clear_rows(self, first: int, n: int, stream=None) -> None:
        _check(lib().irs_dc_clear_rows(self.h, first, n, stream))

    def row_words(self) -> int:
        """u32 words per bitmap row (the stride of fetch_rows_into)."""
        stride = _sz()
        probe = np.zeros(1, np.uint32)
        _check(lib().irs_dc_fetch_rows(self.h, 0, 0, _ptr(probe), 0, C.byref(stride)))
        return stride.value

    def fetch_rows_into(self, first: int, n: int, out: np.ndarray) -> None:
        """Raw bitmap rows [first, first + n) into out [n][row_words()] u32
        (page-locked, and read only after the stream has passed the call, in
        the asynchronous host mode)."""
        stride = _sz()
        if out.dtype != np.uint32 or not out.flags.c_contiguous:
            raise ValueError("fetch_rows_into needs a contiguous uint32 array")
        _check(lib().irs_dc_fetch_rows(self.h, first, n, _ptr(out), out.size, C.byref(stride)))

    def fetch_rows(self, first: int, n: int, db_len: int) -> np.ndarray:
        """Bitmap rows [first, first+n) unpacked to [n][db_len] uint8."""
        stride = _sz()
        probe = np.zeros(1, np.uint32)
        _check(lib().irs_dc_fetch_rows(self.h, first, 0, _ptr(probe), 0, C.byref(stride)))
        cap = max(n * stride.value, 1)
        buf = np.zeros(cap, np.uint32)
        _check(lib().irs_dc_fetch_rows(self.h, first, n, _ptr(buf), cap, C.byref(stride)))
        rows = buf[: n * stride.value].reshape(n, stride.value)
        bits = np.unpackbits(rows.view(np.uint8), axis=1, bitorder="little")
        return bits[:, :db_len]

    def fetch_bitmap(self, n_queries: int, db_len: int) -> np.ndarray:
        """Reference layout: bit (q * db_len + e), u64 words."""
        out = np.zeros((n_queries * db_len + 63) // 64, np.uint64)
        _check(lib().irs_dc_fetch_bitmap(self.h, n_queries, db_len, _ptr(out)))
        return out

    def fetch_matches(self, cap: int = 1 << 20) -> np.ndarray:
        out = np.zeros(2 * cap, np.uint32)
        n = _sz()
        _check(lib().irs_dc_fetch_matches(self.h, _ptr(out), cap, C.byref(n)))
        return out[: 2 * min(n.value, cap)].reshape(-1, 2)

    def get_partial_results(self, n_queries: int, db_len: int, cap: int = 1 << 20) -> np.ndarray:
        out = np.zeros(cap, np.uint32)
        n = _sz()
        _check(lib().irs_dc_get_partial_results(self.h, n_queries, db_len, _ptr(out), cap, C.byref(n)))
        return out[: min(n.value, cap)]

    def join_db_matches(self, n_queries: int, db_len: int, right: "DistanceComparator" = None,
                        or_policy=None, stream=None) -> None:
        _check(lib().irs_dc_join_db_matches(self.h, right.h if right else None, or_policy, n_queries, db_len,
                                            stream))

    def join_batch_matches(self, n_queries: int, right: "DistanceComparator" = None, stream=None) -> None:
        _check(lib().irs_dc_join_batch_matches(self.h, right.h if right else None, n_queries, stream))

    def fetch_final_results(self, n_queries: int):
        f = np.zeros(n_queries, np.uint32)
        c = np.zeros(n_queries, np.uint32)
        a = np.zeros((n_queries, MAX_MATCHES_LEN), np.uint32)
        _check(lib().irs_dc_fetch_final_results(self.h, n_queries, _ptr(f), _ptr(c), _ptr(a)))
        return f, c, a

    def fetch_final_results_into(self, n_queries: int, final: np.ndarray, counters: np.ndarray,
                                 matches: np.ndarray) -> None:
        """irs_dc_fetch_final_results into caller-owned arrays (page-locked,
        and read only after the stream has passed the call, in the
        asynchronous host mode)."""
        for a in (final, counters, matches):
            if a.dtype != np.uint32 or not a.flags.c_contiguous:
                raise ValueError("fetch_final_results_into needs contiguous uint32 arrays")
        if final.size < n_queries or counters.size < n_queries or matches.shape[0] < n_queries or \
                matches.shape[1] != MAX_MATCHES_LEN:
            raise ValueError("output arrays too small")
        _check(lib().irs_dc_fetch_final_results(self.h, n_queries, _ptr(final), _ptr(counters), _ptr(matches)))

    def close(self) -> None:
        if self.h:
            lib().irs_dc_destroy(self.h)
            self.h = None


def bitmap_get(bitmap: np.ndarray, n_queries: int, db_len: int) -> np.ndarray:
    """Unpacks a reference-layout bitmap into [n_queries][db_len] uint8."""
    bits = np.unpackbits(bitmap.view(np.uint8), bitorder="little")[: n_queries * db_len]
    return bits.reshape(n_queries, db_len)
