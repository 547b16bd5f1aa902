"""CPU-side checks of the product boundary (no GPU needed).

- the C-ABI library loads and exports every function include/irisb200.h
  declares, and the Python mirror binds exactly those;
- the bit-sliced circuit header (the code the threshold kernels run) matches
  the oracle bit-for-bit when compiled for the host by a test harness.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "irisb200.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(irs_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_header_symbols():
    import irisb200
    lib = irisb200.lib()
    names = header_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), f"{n} declared in irisb200.h but not exported"
    assert sorted(irisb200.exported_symbols()) == names
    out = subprocess.run(["nm", "-D", irisb200.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (irs_\w+)", out))
    assert exported == set(names)


def test_rust_binding_declares_every_header_function():
    """The Rust `extern` block of include/irisb200.rs declares exactly the
    functions of include/irisb200.h."""
    text = open(os.path.join(ROOT, "include", "irisb200.rs")).read()
    declared = set(re.findall(r"pub fn (irs_[a-z0-9_]+)\(", text))
    assert declared == set(header_functions())


def test_version_and_errors_without_gpu():
    import irisb200
    lib = irisb200.lib()
    assert b"sm_100a" in lib.irs_version()
    h = C.c_void_p()
    rc = lib.irs_device_manager_init(-1, C.byref(h))
    assert rc != 0 and h.value is None
    assert len(lib.irs_last_error()) > 0


@pytest.fixture(scope="module")
def harness():
    out = os.path.join(ROOT, "tests", "native", "_build")
    os.makedirs(out, exist_ok=True)
    so = os.path.join(out, "libcircuit_harness.so")
    src = os.path.join(ROOT, "tests", "native", "circuit_harness.cu")
    deps = [src] + [os.path.join(ROOT, "iris-mpc_b200", "csrc", f) for f in ("circuit.cuh", "common.cuh")]
    if not os.path.exists(so) or any(os.path.getmtime(d) > os.path.getmtime(so) for d in deps):
        subprocess.run(["nvcc", "-x", "cu", "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
                        "-Wno-deprecated-gpu-targets", "-o", so, src], check=True)
    return C.CDLL(so)


def _shares(rng, v):
    a = rng.integers(0, 65536, v.size).astype(np.uint16)
    b = rng.integers(0, 65536, v.size).astype(np.uint16)
    return [a, b, ((v.astype(np.int64) - a - b) % 65536).astype(np.uint16)]


@pytest.mark.parametrize("stage", [0, 1])
def test_circuit_header_matches_oracle(oracle, harness, stage):
    rng = np.random.default_rng(11 + stage)
    W = 96
    n = 32 * W
    code = rng.integers(0, 12801, n)
    code = np.where(rng.integers(0, 2, n) == 1, (65536 - code) % 65536, code).astype(np.uint16)
    mask = rng.integers(0, 12801, n).astype(np.uint16)
    cs, ms = _shares(rng, code), _shares(rng, mask)
    keys = [[3] * 8, [4] * 8, [5] * 8]
    A = 20316
    o = oracle.threshold_words(cs, ms, A, keys, dev=0, batch=9, word_base=777, stage=stage)
    rev = np.zeros(W, np.uint32)
    comp = np.zeros(3 * W, np.uint32)
    P = C.c_void_p * 3
    karr = np.ascontiguousarray(np.array(keys, np.uint32).reshape(24))
    harness.harness_threshold_words(P(*[x.ctypes.data for x in cs]), P(*[x.ctypes.data for x in ms]), C.c_long(W),
                                    C.c_uint32(A), C.c_void_p(karr.ctypes.data), C.c_uint32(0), C.c_uint64(9),
                                    C.c_uint64(777), C.c_int(stage), C.c_void_p(rev.ctypes.data),
                                    C.c_void_p(comp.ctypes.data))
    comp = comp.reshape(3, W)
    assert np.array_equal(rev, o["revealed"])
    for p in range(3):
        assert np.array_equal(comp[p], o["res_a"][p])
        assert np.array_equal(comp[(p + 2) % 3], o["res_b"][p])


def test_chacha12_and_packed_math(oracle, harness):
    key = np.arange(8, dtype=np.uint32) + 99
    for rounds in (12, 20):
        out = np.zeros(16, np.uint32)
        harness.harness_chacha_block(C.c_void_p(key.ctypes.data), C.c_uint64(1 << 41), C.c_uint64(7), C.c_int(rounds),
                                     C.c_void_p(out.ctypes.data))
        assert np.array_equal(out, oracle.chacha_block(key, 1 << 41, 7, rounds))
    rng = np.random.default_rng(2)
    a = rng.integers(0, 2 ** 32, 4096, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 2 ** 32, 4096, dtype=np.uint64).astype(np.uint32)
    a[:4] = [0, 0xFFFFFFFF, 0x80008000, 0x7FFF7FFF]
    b[:4] = [0xFFFFFFFF, 1, 0x80008000, 0x80018001]
    ad = np.zeros_like(a)
    sb = np.zeros_like(a)
    harness.harness_packed16(C.c_void_p(a.ctypes.data), C.c_void_p(b.ctypes.data), C.c_void_p(ad.ctypes.data),
                             C.c_void_p(sb.ctypes.data), C.c_long(a.size))
    assert np.array_equal(ad.view(np.uint16), a.view(np.uint16) + b.view(np.uint16))
    assert np.array_equal(sb.view(np.uint16), a.view(np.uint16) - b.view(np.uint16))


def test_bit_transposes(harness):
    rng = np.random.default_rng(3)
    v = rng.integers(0, 65536, 32).astype(np.uint16)
    w = np.ascontiguousarray(v.view(np.uint32))
    planes = np.zeros(16, np.uint32)
    harness.harness_slice16(C.c_void_p(w.ctypes.data), C.c_void_p(planes.ctypes.data))
    for k in range(16):
        exp = sum(((int(v[j]) >> k) & 1) << j for j in range(32))
        assert int(planes[k]) == exp
    a = rng.integers(0, 2 ** 32, 32, dtype=np.uint64).astype(np.uint32)
    t = a.copy()
    harness.harness_transpose32(C.c_void_p(t.ctypes.data))
    for r in range(32):
        exp = sum(((int(a[c]) >> r) & 1) << c for c in range(32))
        assert int(t[r]) == exp


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the header's structs have the C sizes and field
    offsets (compiled against include/irisb200.h with the host compiler)."""
    import irisb200
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stddef.h>
#include <stdio.h>
#include "irisb200.h"
#define F(T, m) printf(#T "." #m " %zu\\n", offsetof(T, m))
int main(void) {
  printf("irs_query_slot %zu\\n", sizeof(irs_query_slot));
  F(irs_query_slot, src); F(irs_query_slot, rot_lo); F(irs_query_slot, n_rot); F(irs_query_slot, query);
  printf("irs_scan_candidate %zu\\n", sizeof(irs_scan_candidate));
  F(irs_scan_candidate, path); F(irs_scan_candidate, tile); F(irs_scan_candidate, chunk);
  printf("irs_scan_timing %zu\\n", sizeof(irs_scan_timing));
  F(irs_scan_timing, cand); F(irs_scan_timing, ms); F(irs_scan_timing, finalist); F(irs_scan_timing, reserved);
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.split("\n") if line)
    mirrors = {"irs_query_slot": irisb200.QuerySlot, "irs_scan_candidate": irisb200.ScanCandidate,
               "irs_scan_timing": irisb200.ScanTiming}
    for cname, cls in mirrors.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert int(got[f"{cname}.{field}"]) == getattr(cls, field).offset, f"{cname}.{field}"
