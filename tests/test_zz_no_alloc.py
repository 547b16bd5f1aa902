"""The no-allocation threshold entry point against the regular one.

irs_circuits_compare_threshold_masked_many_noalloc serves callers that cannot
allocate device memory once running (a server that reserved all of HBM for
the share database, or a host runtime whose own allocator owns the device):
its scratch is a static device array instead of a pool allocation.  This test
calls it through the C ABI twice in a row, with different inputs, and checks
every output word against irs_circuits_compare_threshold_masked_many on the
same inputs (integer work: bit-exact).  It also checks the size limit.  The
file is named to be collected last, so a failure here never hides another
test's result.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import irisb200

pytestmark = pytest.mark.gpu

SEEDS = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]


def _shares(rng, v):
    a = rng.integers(0, 65536, v.size).astype(np.uint16)
    b = rng.integers(0, 65536, v.size).astype(np.uint16)
    return [a, b, ((v.astype(np.int64) - a - b) % 65536).astype(np.uint16)]


def _ptr3(bufs):
    return C.cast((C.c_void_p * 3)(*[b.ptr for b in bufs]), C.c_void_p)


def _run(lib, fn, circuits, code, mask, n, a, res_a, res_b, opened):
    return getattr(lib, fn)(circuits.h, _ptr3(code), _ptr3(mask), n, a, _ptr3(res_a), _ptr3(res_b), opened.ptr, None)


def test_noalloc_matches_regular_entry_point_twice():
    lib = irisb200.lib()
    dm = irisb200.DeviceManager(0)
    c = irisb200.Circuits(dm, SEEDS)
    try:
        for call, (n, a, seed) in enumerate(((64 * 4096, 16384, 1), (64 * 1500, 20316, 2))):
            rng = np.random.default_rng(seed)
            code = rng.integers(0, 12801, n)
            code = np.where(rng.integers(0, 2, n) == 1, (65536 - code) % 65536, code).astype(np.uint16)
            mask = rng.integers(0, 12801, n).astype(np.uint16)
            dcode = [irisb200.DeviceBuffer.from_array(dm, x) for x in _shares(rng, code)]
            dmask = [irisb200.DeviceBuffer.from_array(dm, x) for x in _shares(rng, mask)]
            outs = {}
            for fn in ("irs_circuits_compare_threshold_masked_many_noalloc",
                       "irs_circuits_compare_threshold_masked_many"):
                ra = [irisb200.DeviceBuffer(dm, n // 8) for _ in range(3)]
                rb = [irisb200.DeviceBuffer(dm, n // 8) for _ in range(3)]
                op = irisb200.DeviceBuffer(dm, n // 8)
                rc = _run(lib, fn, c, dcode, dmask, n, a, ra, rb, op)
                assert rc == 0, lib.irs_last_error()
                dm.synchronize()
                outs[fn] = ([x.download(np.uint64, n // 64) for x in ra], [x.download(np.uint64, n // 64) for x in rb],
                            op.download(np.uint64, n // 64))
            na, nb, nop = outs["irs_circuits_compare_threshold_masked_many_noalloc"]
            ra_, rb_, rop = outs["irs_circuits_compare_threshold_masked_many"]
            assert np.array_equal(nop, rop), f"call {call}: opened bits differ"
            for p in range(3):
                assert np.array_equal(na[p], ra_[p]) and np.array_equal(nb[p], rb_[p]), f"call {call}: party {p}"
            # and the opened bits are the plaintext predicate (threshold.rs:110-124)
            r = (mask.astype(np.uint64) * np.uint64(a) - (code.astype(np.uint64) << np.uint64(16)) - np.uint64(1))
            bits = ((r & np.uint64(0xFFFFFFFF)) >> np.uint64(31)).astype(np.uint8)
            assert np.array_equal(np.unpackbits(nop.view(np.uint8), bitorder="little"), bits)
    finally:
        c.close()
        dm.close()


def test_noalloc_rejects_sizes_beyond_the_limit():
    lib = irisb200.lib()
    dm = irisb200.DeviceManager(0)
    c = irisb200.Circuits(dm, SEEDS)
    try:
        buf = [irisb200.DeviceBuffer(dm, 256) for _ in range(3)]
        n = (1 << 22) + 64
        rc = _run(lib, "irs_circuits_compare_threshold_masked_many_noalloc", c, buf, buf, n, 16384, buf, buf, buf[0])
        assert rc == -1  # IRS_ERR_INVALID
        assert b"no-allocation limit" in lib.irs_last_error()
    finally:
        c.close()
        dm.close()
