"""Phase 1 against the reference's own arithmetic, run on the GPU.

The reference computes a party's u16 dot shares as three int8 cuBLAS GEMMs on
signed limbs (byte - 128) combined as A0.B0 + 256 (A0.B1 + A1.B0) in wrapping
i32 (iris-mpc-gpu/src/dot/share_db.rs:62-112,800-845; the limbs of
preprocess_query, share_db.rs:45-59), then corrects with the limb sums and
reduces mod 2^16 in `matmul_correct_and_reduce` (iris-mpc-gpu/src/dot/
kernel.cu:16-28).  Here the same GEMMs run through cuBLAS (torch._int_mm) and
the reference's kernel, compiled unmodified into oracle/_ref/dot_ref.cubin,
runs on their output; the library's single-pass unsigned-limb tcgen05 GEMM
must produce the identical u16 results (codes x1 and masks x2)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest
import torch

import irisb200
import workload as W

pytestmark = pytest.mark.gpu

Q, M = 64, 384


def _cuda():
    lib = C.CDLL("libcuda.so.1")
    for name in ("cuModuleLoad", "cuModuleGetFunction", "cuLaunchKernel", "cuCtxSynchronize", "cuModuleUnload"):
        getattr(lib, name).restype = C.c_int
    return lib


def _limbs(x):
    """u16 -> the reference's signed limbs (byte - 128) as int8."""
    lo = ((x & 0xFF).astype(np.int16) - 128).astype(np.int8)
    hi = ((x >> 8).astype(np.int16) - 128).astype(np.int8)
    return lo, hi


def _reference_dot(cu, fn, db, q, multiplier):
    dev = torch.device("cuda", 0)
    a0, a1 = (torch.from_numpy(x).to(dev) for x in _limbs(db))  # [M][K]
    b0, b1 = (torch.from_numpy(x).to(dev) for x in _limbs(q))   # [Q][K]
    c = torch._int_mm(b0, a0.t()) + 256 * (torch._int_mm(b0, a1.t()) +
                                                          torch._int_mm(b1, a0.t()))
    c = c.contiguous()  # [Q][M] i32, wrapping
    sums = [x.to(torch.int32).sum(dim=1).to(torch.int32).contiguous() for x in (a0, a1, b0, b1)]
    out = torch.zeros(Q * M, dtype=torch.int16, device=dev)
    zeros = torch.zeros(Q * M, dtype=torch.int16, device=dev)
    torch.cuda.synchronize()
    args = [C.c_void_p(c.data_ptr()), C.c_void_p(out.data_ptr())] + [C.c_void_p(s.data_ptr()) for s in sums] + \
        [C.c_size_t(M), C.c_size_t(Q * M), C.c_size_t(0), C.c_uint16(multiplier), C.c_void_p(zeros.data_ptr()),
         C.c_void_p(zeros.data_ptr())]
    params = (C.c_void_p * len(args))(*[C.cast(C.byref(x), C.c_void_p) for x in args])
    assert cu.cuLaunchKernel(fn, (Q * M + 255) // 256, 1, 1, 256, 1, 1, 0, None, params, None) == 0
    assert cu.cuCtxSynchronize() == 0
    return out.cpu().numpy().view(np.uint16).reshape(Q, M)


def test_reference_phase1_equals_library_gemm(dm, oracle):
    cubin = oracle.REF_DOT_CUBIN
    if not os.path.exists(cubin):
        pytest.skip("oracle/_ref/dot_ref.cubin not built (make -C oracle ref, needs the reference tree)")
    cu = _cuda()
    mod = C.c_void_p()
    assert cu.cuModuleLoad(C.byref(mod), cubin.encode()) == 0
    fn = C.c_void_p()
    assert cu.cuModuleGetFunction(C.byref(fn), mod, b"matmul_correct_and_reduce") == 0
    rng = np.random.default_rng(77)
    try:
        for k, mult in ((12800, 1), (6400, 2)):
            db = rng.integers(0, 65536, (M, k), dtype=np.uint16)
            q = rng.integers(0, 65536, (Q, k), dtype=np.uint16)
            db[0], q[0] = 0xFFFF, 0xFFFF  # extreme limbs
            ref = _reference_dot(cu, fn, db, q, mult)
            e = irisb200.ShareDB(0, dm, M, Q, k, W.SEEDS[0], is_remote=False)
            e.alloc_db(M)
            e.load_records(0, db)
            e.query_upload(q)
            e.dot(0, M, mult)
            got = e.fetch_results(M)
            e.close()
            assert np.array_equal(got, ref), f"K={k}"
            # and both are the plain dot mod 2^16 (times the multiplier)
            plain = (q[:8].astype(np.uint64) @ db.T.astype(np.uint64) * mult) % 65536
            assert np.array_equal(ref[:8].astype(np.uint64), plain)
    finally:
        cu.cuModuleUnload(mod)
