"""MPC OR tree (or_reduce_result, iris-mpc-gpu/src/threshold_ring/
protocol.rs:2363-2515; compare_threshold_masked_many_with_or_tree, 2594-2610;
tests/threshold_and_or_tree.rs): the comparison of n elements reduced to one
shared bit.  The opened bit must be the OR of the plaintext predicate
(real_result_msb_reduce), and every party's share of it must equal the
oracle's OR tree run on the oracle's threshold shares."""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
import workload as W

pytestmark = pytest.mark.gpu

A = 16384
KEYS = [W.SEEDS[p][0] for p in range(3)]


def _shares(rng, v):
    a = rng.integers(0, 65536, v.size).astype(np.uint16)
    b = rng.integers(0, 65536, v.size).astype(np.uint16)
    return [a, b, ((v.astype(np.int64) - a - b) % 65536).astype(np.uint16)]


@pytest.mark.parametrize("n,planted", [(64 * 1000, []), (64 * 1000, [12345]), (64 * 3, [191]),
                                       (64 * 777, [0, 40000]), (1 << 22, [(1 << 22) - 1])])
def test_or_tree_matches_plaintext_and_oracle(dm, oracle, n, planted):
    rng = np.random.default_rng(n + len(planted))
    code = np.full(n, 65536 - 100, np.uint16)  # -100: no match against mask 1000
    mask = np.full(n, 1000, np.uint16)
    for i in planted:
        code[i], mask[i] = 12800, 100
    exp = bool(oracle.match_predicate(code, mask, A).any())
    cs, ms = _shares(rng, code), _shares(rng, mask)
    dcode = [irisb200.DeviceBuffer.from_array(dm, x) for x in cs]
    dmask = [irisb200.DeviceBuffer.from_array(dm, x) for x in ms]
    c = irisb200.Circuits(dm, W.SEEDS)
    try:
        comps, opened = c.compare_threshold_masked_many_with_or_tree(dcode, dmask, n, A)
        assert opened == int(exp)
        assert int(comps[0] ^ comps[1] ^ comps[2]) == opened
        ref = oracle.threshold_words(cs, ms, A, KEYS)
        ocomps, oopened = oracle.or_tree([ref["res_a"][p] for p in range(3)], KEYS)
        assert oopened == opened and np.array_equal(ocomps, comps)
        # the same tree from the parties' a-shares written by the plain comparison
        ra = [irisb200.DeviceBuffer(dm, n // 8) for _ in range(3)]
        c.compare_threshold_masked_many(dcode, dmask, n, A, res_a=ra)
        comps2, opened2 = c.or_reduce(ra, n)
        assert opened2 == opened and np.array_equal(comps2, comps)
        for b in ra:
            b.free()
    finally:
        c.close()
        for b in dcode + dmask:
            b.free()
