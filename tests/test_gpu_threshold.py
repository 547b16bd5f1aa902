"""GPU parity of the fused 3-party threshold protocol (Circuits).

Mirrors iris-mpc-gpu/tests/threshold.rs (compare_threshold_masked_many against
real_result_msb, seeds ([0;8],[2;8]) / ([1;8],[0;8]) / ([2;8],[1;8]),
DB_RNG_SEED 0xdeadbeef), tests/extract_msb_mod.rs (msb of -code*2^16 - 1) and
tests/lift.rs (lifted shares minus injected corrections reconstruct the mask).
Opened bits must equal the plaintext predicate; every party's replicated share
must equal the oracle's.
"""
from __future__ import annotations

import numpy as np
import pytest

import irisb200

pytestmark = pytest.mark.gpu

SEEDS = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
KEYS = [SEEDS[p][0] for p in range(3)]
DB_RNG_SEED = 0xDEADBEEF


def sample_code_dots(rng, n):
    x = rng.integers(0, 12801, n)
    neg = rng.integers(0, 2, n) == 1
    return np.where(neg, (65536 - x) % 65536, x).astype(np.uint16)


def sample_mask_dots(rng, n):
    return rng.integers(0, 12801, n).astype(np.uint16)


def rep_share(rng, v):
    a = rng.integers(0, 65536, v.size).astype(np.uint16)
    b = rng.integers(0, 65536, v.size).astype(np.uint16)
    return [a, b, ((v.astype(np.int64) - a - b) % 65536).astype(np.uint16)]


def to_gpu(dm, parts):
    return [irisb200.DeviceBuffer.from_array(dm, x) for x in parts]


def _u32_words(u64_words):
    return np.ascontiguousarray(u64_words).view(np.uint32)


# 12,507,136 = INPUTS_PER_GPU_SIZE of iris-mpc-gpu/tests/threshold.rs:24, the
# reference test's own size.
@pytest.mark.parametrize("n,threshold_a", [(64 * 1024, 20316), (64 * 4096, 16384), (64, 20316),
                                           (12_507_136, 16384)])
def test_threshold(dm, oracle, n, threshold_a):
    rng = np.random.default_rng(DB_RNG_SEED)
    code = sample_code_dots(rng, n)
    mask = sample_mask_dots(rng, n)
    code[:3] = [0, 12800, 65536 - 12800]
    mask[:3] = [0, 0, 12800]
    cs, ms = rep_share(rng, code), rep_share(rng, mask)
    c = irisb200.Circuits(dm, SEEDS)
    c.set_batch(3)
    dc = to_gpu(dm, cs)
    dmk = to_gpu(dm, ms)
    ra = [irisb200.DeviceBuffer(dm, n // 8) for _ in range(3)]
    rb = [irisb200.DeviceBuffer(dm, n // 8) for _ in range(3)]
    op = irisb200.DeviceBuffer(dm, n // 8)
    c.compare_threshold_masked_many(dc, dmk, n, threshold_a, res_a=ra, res_b=rb, opened=op)
    dm.synchronize()
    opened = op.download(np.uint64, n // 64)
    real = oracle.pack_bits_u32(oracle.match_predicate(code, mask, threshold_a))
    assert np.array_equal(_u32_words(opened), real)
    o = oracle.threshold_words(cs, ms, threshold_a, KEYS, dev=0, batch=3, word_base=0)
    for p in range(3):
        assert np.array_equal(_u32_words(ra[p].download(np.uint64, n // 64)), o["res_a"][p]), f"party {p} a"
        assert np.array_equal(_u32_words(rb[p].download(np.uint64, n // 64)), o["res_b"][p]), f"party {p} b"
    c.close()


def test_extract_msb_mod(dm, oracle):
    rng = np.random.default_rng(DB_RNG_SEED + 1)
    n = 64 * 2048
    code = sample_code_dots(rng, n)
    cs = rep_share(rng, code)
    c = irisb200.Circuits(dm, SEEDS)
    op = irisb200.DeviceBuffer(dm, n // 8)
    c.extract_msb_of_code(to_gpu(dm, cs), n, opened=op)
    dm.synchronize()
    # real_result_msb of extract_msb_mod.rs:111-120: msb of (2^64-1 - code<<16) mod 2^32
    exp = ((((0xFFFFFFFF - (code.astype(np.uint64) << np.uint64(16))) & np.uint64(0xFFFFFFFF)) >> np.uint64(31))
           .astype(np.uint8))
    assert np.array_equal(_u32_words(op.download(np.uint64, n // 64)), oracle.pack_bits_u32(exp))
    c.close()


def test_lift(dm, oracle):
    rng = np.random.default_rng(DB_RNG_SEED + 2)
    n = 64 * 1024
    mask = sample_mask_dots(rng, n)
    ms = rep_share(rng, mask)
    c = irisb200.Circuits(dm, SEEDS)
    corr = [irisb200.DeviceBuffer(dm, 4 * n) for _ in range(3)]
    c.lift_mpc(to_gpu(dm, ms), n, corr)
    dm.synchronize()
    cr = [x.download(np.uint16, 2 * n).reshape(2, n) for x in corr]
    c1 = sum(x[0].astype(np.uint64) for x in cr) % 65536
    c2 = sum(x[1].astype(np.uint64) for x in cr) % 65536
    assert set(np.unique(c1)) <= {0, 1} and set(np.unique(c2)) <= {0, 1}
    lifted = sum(x.astype(np.uint64) for x in ms)
    assert np.array_equal((lifted - (c1 << 16) - (c2 << 17)) % (1 << 32), mask.astype(np.uint64))
    o = oracle.threshold_words(ms, ms, 16384, KEYS, want_lift=True)
    for p in range(3):
        assert np.array_equal(cr[p][0], o["corr"][p][0]) and np.array_equal(cr[p][1], o["corr"][p][1])
    c.close()


def test_rejects_bad_shapes(dm):
    c = irisb200.Circuits(dm, SEEDS)
    buf = [irisb200.DeviceBuffer(dm, 256) for _ in range(3)]
    with pytest.raises(irisb200.IrisError):
        c.compare_threshold_masked_many(buf, buf, 96, 20316)  # not a multiple of 64
    bad = [([0] * 8, [1] * 8)] * 3
    with pytest.raises(irisb200.IrisError):
        irisb200.Circuits(dm, bad)
    c.close()
