"""Pins the ChaCha12 keystream to the reference's own kernel.

`chacha12` of iris-mpc-gpu/src/rng/chacha.cu, compiled unmodified from the
reference tree by `make -C oracle ref` into oracle/_ref/chacha_ref.cubin, is
loaded with the CUDA driver API and launched as ChachaCommon::fill_rng_into
does (iris-mpc-gpu/src/rng/chacha.rs:38-79: state = constants | seed |
counter | nonce, one 16-word block per thread at counter + thread index, 256
threads per block).  Its output must equal the oracle's 12-round keystream
bit for bit -- the oracle whose 20-round variant equals Python's ChaCha20 and
whose 12-round layout the library's kernels are tested against."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

import irisb200

pytestmark = pytest.mark.gpu

CONST = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574]


def _cuda():
    lib = C.CDLL("libcuda.so.1")
    for name in ("cuModuleLoad", "cuModuleGetFunction", "cuLaunchKernel", "cuCtxSynchronize", "cuModuleUnload"):
        getattr(lib, name).restype = C.c_int
    return lib


def test_reference_chacha12_kernel_equals_oracle(dm, oracle):
    cubin = oracle.REF_CHACHA_CUBIN
    if not os.path.exists(cubin):
        pytest.skip("oracle/_ref/chacha_ref.cubin not built (make -C oracle ref, needs the reference tree)")
    cu = _cuda()
    mod = C.c_void_p()
    assert cu.cuModuleLoad(C.byref(mod), cubin.encode()) == 0
    fn = C.c_void_p()
    assert cu.cuModuleGetFunction(C.byref(fn), mod, b"chacha12") == 0
    rng = np.random.default_rng(12)
    try:
        for key, counter, nonce, n_blocks in (
                ([0] * 8, 0, 0, 1),
                ([1] * 8, 7, 3, 300),
                (rng.integers(0, 2 ** 32, 8).tolist(), (5 << 40) | 123, (2 << 32) | 0, 1000),
                (rng.integers(0, 2 ** 32, 8).tolist(), 0xFFFFFFFF - 10, 1, 64)):  # counter carries into word 13
            state = np.array(CONST + [int(k) for k in key] + [counter & 0xFFFFFFFF, counter >> 32,
                                                                 nonce & 0xFFFFFFFF, nonce >> 32], np.uint32)
            d_state = irisb200.DeviceBuffer.from_array(dm, state)
            n = 16 * n_blocks
            d_out = irisb200.DeviceBuffer(dm, 4 * n)
            a_out, a_state = C.c_void_p(d_out.ptr), C.c_void_p(d_state.ptr)
            s12, s13, ln = C.c_uint32(int(state[12])), C.c_uint32(int(state[13])), C.c_size_t(n)
            params = (C.c_void_p * 5)(*[C.cast(C.byref(x), C.c_void_p) for x in (a_out, a_state, s12, s13, ln)])
            grid = (n_blocks + 255) // 256
            assert cu.cuLaunchKernel(fn, grid, 1, 1, 256, 1, 1, 0, None, params, None) == 0
            assert cu.cuCtxSynchronize() == 0
            got = d_out.download(np.uint32, n)
            exp = oracle.chacha_fill(key, counter, nonce, n_blocks, rounds=12)
            assert np.array_equal(got, exp), f"counter {counter:#x} nonce {nonce:#x}"
            d_state.free()
            d_out.free()
    finally:
        cu.cuModuleUnload(mod)
