"""Pins the CPU oracle to the reference's own known-answer tests.

Mirrors: symmetric-gr-shamir_sage.sage:301-339 (test_gr_inv / test_gr_prod /
test_lagrange), gr4_encoding_example.sage:40 (S64 mod 2^16 == S16),
galois_engine.rs:713-765 (galois_dot_trick, rotation_aware_dot_trick),
galois_engine.rs:784-867 (hamming_distance_galois, random_codes.txt),
galois_engine.rs:938-996 and iris.rs:742-766 (mirrored codes,
flipped_codes.txt), iris.rs:726-741 (decode_from_string, all_rotations.txt),
galois_engine.rs:998-1013 (check_remap), threshold.rs:110-124 (real_result_msb).
The example-data vectors come from tests/golden/reference_kats.json, written
from the reference's example-data files by tests/golden/make_golden.py.
"""
from __future__ import annotations

import numpy as np
import pytest

import hashlib
import json
import os

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kats.json")))

S64 = [
    [1, 0, 0, 0],
    [3721680401061044962, 1, 0, 0],
    [8289148916157705379, 3107565179763450474, 1, 0],
    [11432970333055501229, 7744929693175761652, 17484058852862123699, 1],
]


def test_gr_inv(oracle):
    assert list(oracle.gr4_inv([1, 1, 0, 0])) == [2, 65535, 1, 65535]


def test_gr_prod(oracle):
    assert list(oracle.gr4_mul([7, 0, 3, 0], [1, 1, 0, 1])) == [7, 10, 6, 10]


def test_gr_inverse_roundtrip(oracle):
    rng = np.random.default_rng(3)
    for _ in range(20):
        a = rng.integers(0, 65536, 4)
        a[0] |= 1
        inv = oracle.gr4_inv(a)
        assert list(oracle.gr4_mul(a, inv)) == [1, 0, 0, 0]


def test_basis_matrices(oracle):
    s, b, lag = oracle.basis_mats()
    assert np.array_equal(s, (np.array(S64, dtype=object) % 65536).astype(np.uint16))
    # (S S^T) B == I mod 2^16
    sst = (s.astype(np.int64) @ s.T.astype(np.int64)) % 65536
    assert np.array_equal((sst @ b.astype(np.int64)) % 65536, np.eye(4, dtype=np.int64))


def test_lagrange_interpolates_degree_two(oracle):
    """sage test_lagrange: a degree-2 polynomial is recovered at 0 from its
    values at the three base points 1, x, 1+x."""
    _, _, lag = oracle.basis_mats()
    rng = np.random.default_rng(4)
    pts = [[1, 0, 0, 0], [0, 1, 0, 0], [1, 1, 0, 0]]
    for _ in range(10):
        c = [rng.integers(0, 65536, 4) for _ in range(3)]

        def ev(x):
            x2 = oracle.gr4_mul(x, x)
            return (c[0].astype(np.int64) + oracle.gr4_mul(c[1], x) + oracle.gr4_mul(c[2], x2)) % 65536

        acc = np.zeros(4, np.int64)
        for p in range(3):
            acc = (acc + oracle.gr4_mul(lag[p], ev(pts[p]))) % 65536
        assert np.array_equal(acc, c[0] % 65536)


def test_galois_dot_trick(oracle):
    rng = np.random.default_rng(5)
    for t in range(5):
        a = rng.integers(0, 2 ** 63, 200, dtype=np.uint64)
        b = rng.integers(0, 2 ** 63, 200, dtype=np.uint64)
        sd = oracle.encode_mask_code(a, 100 + t, trimmed=False)
        sq = oracle.encode_mask_code(b, 200 + t, trimmed=False)
        dot = sum(oracle.trick_dot(sd[p], oracle.preprocess_query(p, sq[p])) for p in range(3)) % 65536
        assert dot == sum(bin(int(x)).count("1") for x in (a & b))


def test_rotation_aware_dot_trick(oracle):
    """Rotating the share rows by whole 4-coefficient blocks equals rotating
    the plaintext iris by whole columns."""
    code, mask = oracle.iris_random(7, 1)
    q_code, q_mask = oracle.iris_random(7, 2)
    db = oracle.encode_iris_code(code, mask, 11)
    for r in (0, 7, 15, 22, 30):
        shares = oracle.encode_iris_code(q_code, q_mask, 12)
        rot = [oracle.rotate_share(shares[p], r) for p in range(3)]
        dot = sum(oracle.trick_dot(db[p], oracle.preprocess_query(p, rot[p])) for p in range(3)) % 65536
        # plaintext: rotation r = net left rotation by 15 - r columns
        pc = oracle.iris_rotate(q_code, -(15 - r))
        pm = oracle.iris_rotate(q_mask, -(15 - r))
        m = mask & pm
        hd = sum(bin(int(x)).count("1") for x in ((code ^ pc) & m))
        mc = sum(bin(int(x)).count("1") for x in m)
        assert dot == (mc - 2 * hd) % 65536


def _calc_distance(oracle, code_sh, mask_sh, q_code_sh, q_mask_sh):
    """calculate_distance (galois_engine.rs:869-913)."""
    cd = sum(oracle.trick_dot(code_sh[p], oracle.preprocess_query(p, q_code_sh[p])) for p in range(3)) % 65536
    md = sum(2 * oracle.trick_dot(mask_sh[p], oracle.preprocess_query(p, q_mask_sh[p])) for p in range(3)) % 65536
    cd = cd - 65536 if cd >= 32768 else cd
    return 0.5 - cd / (2.0 * md)


def test_hamming_distance_galois(oracle):
    g = GOLDEN["random_codes"]
    c1, m1, c2, m2 = (oracle.iris_from_base64(g[k]) for k in ("code1", "mask1", "code2", "mask2"))
    d0, d15 = g["distance_rot0"], g["distance_min_rot"]
    assert abs(oracle.fractional_distance(c1, m1, c2, m2) - d0) <= 1e-6
    t1c = oracle.encode_iris_code(c1, m1, 21)
    t1m = oracle.encode_mask_code(m1, 22)
    t2c = oracle.encode_iris_code(c2, m2, 23)
    t2m = oracle.encode_mask_code(m2, 24)
    dists = []
    for r in range(31):
        qc = [oracle.rotate_share(t2c[p], r) for p in range(3)]
        qm = [oracle.rotate_share(t2m[p], r) for p in range(3)]
        dists.append(_calc_distance(oracle, t1c, t1m, qc, qm))
    assert abs(dists[15] - d0) <= 1e-6
    assert abs(min(dists) - d15) <= 1e-6


def test_match_mirrored_codes(oracle):
    g = GOLDEN["flipped_codes"]
    code, mask, fcode, fmask = (oracle.iris_from_base64(g[k]) for k in ("code", "mask", "flipped_code",
                                                                         "flipped_mask"))
    mask_both = mask & fmask
    plain = oracle.fractional_distance(code, mask_both, fcode, fmask)
    cs = oracle.encode_iris_code(code, mask_both, 31)
    ms = oracle.encode_mask_code(mask_both, 32)
    ics = oracle.encode_iris_code(fcode, fmask, 33)
    ims = oracle.encode_mask_code(fmask, 34, trimmed=False)
    d = _calc_distance(oracle, cs, ms, ics, [x[:6400] for x in ims])
    assert abs(d - plain) <= 1e-6 and abs(d - 0.5) <= 0.1
    mc = [oracle.mirror_share(ics[p], True) for p in range(3)]
    mm = [oracle.mirror_share(ims[p], False)[:6400] for p in range(3)]
    assert abs(_calc_distance(oracle, cs, ms, mc, mm)) <= 1e-6
    # plaintext mirror (iris.rs:742-766)
    mcode, mmask = oracle.iris_mirror(fcode, fmask)
    assert oracle.fractional_distance(code, mask, mcode, mmask) <= 1e-6


def test_decode_and_rotations(oracle):
    g = GOLDEN["all_rotations"]
    code = oracle.iris_from_base64(g["code"])
    assert oracle.iris_to_base64(code) == g["code"]
    rots = {int(k): v for k, v in g["rotation_bits_sha256"].items()}
    assert sorted(rots) == list(range(-15, 16))
    for r, expect in rots.items():
        got = "".join(str(b) for b in oracle.bits_of(oracle.iris_rotate(code, r)))
        assert hashlib.sha256(got.encode()).hexdigest() == expect, f"rotation {r}"


def test_remap_roundtrip(oracle):
    for i in (0, 1, 5, 799, 800, 6399, 6400, 12799):
        assert oracle.remap_old_to_new(oracle.remap_new_to_old(i)) == i
        assert oracle.remap_new_to_old(oracle.remap_old_to_new(i)) == i


def test_chacha20_matches_cryptography(oracle):
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    key = (np.arange(8, dtype=np.uint32) * 0x01020304 + 7).astype(np.uint32)
    for ctr, nonce in ((0, 0), (5, 0x1122334455667788), (1000, 3)):
        ks = oracle.chacha_fill(key, ctr, nonce, 4, rounds=20)
        iv = int(ctr).to_bytes(8, "little") + int(nonce).to_bytes(8, "little")
        enc = Cipher(algorithms.ChaCha20(key.tobytes(), iv), mode=None).encryptor().update(b"\0" * 256)
        assert np.array_equal(np.frombuffer(enc, np.uint32), ks)


def test_chacha_correlation(oracle):
    """chacha_corr.rs:102-125: the three correlated streams XOR to zero."""
    seeds = [[0] * 8, [1] * 8, [2] * 8]
    ks = [oracle.chacha_fill(s, 0, 0, 64) for s in seeds]
    corr = [ks[p] ^ ks[(p + 2) % 3] for p in range(3)]
    assert not np.any(corr[0] ^ corr[1] ^ corr[2])
    assert np.count_nonzero(corr[0] == 0) <= 1


def _sample_dots(rng, n):
    code = rng.integers(0, 12801, n)
    neg = rng.integers(0, 2, n) == 1
    code = np.where(neg, (65536 - code) % 65536, code).astype(np.uint16)
    mask = rng.integers(0, 12801, n).astype(np.uint16)
    return code, mask


def _rep_share(rng, v):
    a = rng.integers(0, 65536, v.size).astype(np.uint16)
    b = rng.integers(0, 65536, v.size).astype(np.uint16)
    c = ((v.astype(np.int64) - a - b) % 65536).astype(np.uint16)
    return [a, b, c]


@pytest.mark.parametrize("threshold_a", [16384, 20316])
def test_threshold_oracle_matches_predicate(oracle, threshold_a):
    rng = np.random.default_rng(0xDEADBEEF)
    code, mask = _sample_dots(rng, 64 * 40)
    # edge cases: mask = code = 0 (match), extremes
    code[:4] = [0, 12800, 65536 - 12800, 0]
    mask[:4] = [0, 12800, 12800, 1]
    out = oracle.threshold_words(_rep_share(rng, code), _rep_share(rng, mask), threshold_a,
                                 [[0] * 8, [1] * 8, [2] * 8])
    exp = oracle.pack_bits_u32(oracle.match_predicate(code, mask, threshold_a))
    assert np.array_equal(out["revealed"], exp)
    assert int(oracle.match_predicate(np.array([0]), np.array([0]), threshold_a)[0]) == 1
    # replicated views are consistent: party p's b is party p-1's a
    for p in range(3):
        assert np.array_equal(out["res_b"][p], out["res_a"][(p + 2) % 3])


def test_lift_oracle(oracle):
    """tests/lift.rs:84-86: lifted shares minus the injected corrections
    reconstruct the mask in Z_2^32, corrections in {0, 1}."""
    rng = np.random.default_rng(8)
    _, mask = _sample_dots(rng, 64 * 8)
    sh = _rep_share(rng, mask)
    out = oracle.threshold_words(sh, sh, 16384, [[0] * 8, [1] * 8, [2] * 8], want_lift=True)
    lx = out["lift_x"].astype(np.uint64).sum(axis=0)
    c1 = out["corr"][:, 0].astype(np.uint64).sum(axis=0) % 65536
    c2 = out["corr"][:, 1].astype(np.uint64).sum(axis=0) % 65536
    assert set(np.unique(c1)) <= {0, 1} and set(np.unique(c2)) <= {0, 1}
    rec = (lx - (c1 << 16) - (c2 << 17)) % (1 << 32)
    assert np.array_equal(rec, mask.astype(np.uint64))


def test_or_tree_oracle(oracle):
    """The oracle's MPC OR tree opens to the OR of the shared bits, for odd and
    even word counts and a single set bit anywhere (threshold_and_or_tree.rs)."""
    rng = np.random.default_rng(9)
    keys = [[0] * 8, [1] * 8, [2] * 8]
    for n in (1, 2, 3, 7, 64, 101):
        for bit in (None, 0, 32 * n - 1, int(rng.integers(0, 32 * n))):
            plain = np.zeros(n, np.uint32)
            if bit is not None:
                plain[bit // 32] = np.uint32(1 << (bit % 32))
            a = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
            b = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
            comps, opened = oracle.or_tree([a, b, a ^ b ^ plain], keys)
            assert opened == int(bit is not None), (n, bit)
            assert int(comps[0] ^ comps[1] ^ comps[2]) == opened
