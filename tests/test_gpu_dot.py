"""GPU parity of the tcgen05 limb GEMM (ShareDB::dot + dot_reduce_and_multiply).

Mirrors the reference's share_db.rs tests: check_matmul (1132-1198, random u16
matrices against a plain mod-2^16 product), check_shared_matmul (1202-1284,
the three parties' dots of mask shares sum to the mask popcount) and
check_shared_distances (1288-1465, reconstructed code/mask dots give the
plaintext fractional distances) -- plus per-party parity of the zero-share
masked results against the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WIDTH = 12800
QUERY_SIZE = 32
SEEDS = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]


def _engine(dm, party, db_size, q_len, width, remote):
    import irisb200
    e = irisb200.ShareDB(party, dm, db_size, q_len, width, SEEDS[party], is_remote=remote)
    e.alloc_db(db_size)
    return e


@pytest.mark.parametrize("db_size,q_len", [(8000, 32), (1000, 256), (544, 1984), (4096, 2048)])
def test_check_matmul(dm, oracle, db_size, q_len):
    rng = np.random.default_rng(42)
    db = rng.integers(0, 65535, (db_size, WIDTH)).astype(np.uint16)
    q = rng.integers(0, 65535, (q_len, WIDTH)).astype(np.uint16)
    e = _engine(dm, 0, db_size, q_len, WIDTH, remote=False)
    try:
        e.load_records(0, db)
        e.query_upload(q)
        e.dot(0, db_size, 1)
        got = e.fetch_results(db_size)
        exp = oracle.dot_u16(q, db)
        assert np.array_equal(got, exp)
    finally:
        e.close()


def test_check_matmul_offset_chunk_and_mask_width(dm, oracle):
    """Chunked dots (offset, len) and the 6400-wide mask engine with multiplier 2."""
    rng = np.random.default_rng(7)
    n, width = 3000, 6400
    db = rng.integers(0, 65535, (n, width)).astype(np.uint16)
    q = rng.integers(0, 65535, (96, width)).astype(np.uint16)
    e = _engine(dm, 1, n, 96, width, remote=False)
    try:
        e.load_records(0, db)
        e.query_upload(q)
        full = (oracle.dot_u16(q, db).astype(np.uint32) * 2 % 65536).astype(np.uint16)
        for off, ln in ((0, 1024), (1024, 1000), (2048, 952)):
            e.dot(off, ln, 2)
            assert np.array_equal(e.fetch_results(ln), full[:, off:off + ln])
    finally:
        e.close()


def test_s3_i8_limbs_load(dm, oracle):
    """load_single_record_from_s3: stored limbs are byte - 128 as i8."""
    rng = np.random.default_rng(9)
    db = rng.integers(0, 65535, (256, WIDTH)).astype(np.uint16)
    q = rng.integers(0, 65535, (32, WIDTH)).astype(np.uint16)
    limb0 = ((db & 0xFF).astype(np.int16) - 128).astype(np.int8)
    limb1 = ((db >> 8).astype(np.int16) - 128).astype(np.int8)
    e = _engine(dm, 2, 256, 32, WIDTH, remote=False)
    try:
        e.load_records_i8(0, limb0, limb1)
        e.query_upload(q)
        e.dot(0, 256, 1)
        assert np.array_equal(e.fetch_results(256), oracle.dot_u16(q, db))
    finally:
        e.close()


def test_masked_dot_shares_per_party(dm, oracle):
    """With the zero-share mask on, each party's share equals the oracle's and
    the three shares sum to the plain dot."""
    rng = np.random.default_rng(12)
    n, q_len = 640, 64
    dbs = [rng.integers(0, 65535, (n, WIDTH)).astype(np.uint16) for _ in range(3)]
    qs = [rng.integers(0, 65535, (q_len, WIDTH)).astype(np.uint16) for _ in range(3)]
    engines = [_engine(dm, p, n, q_len, WIDTH, remote=True) for p in range(3)]
    try:
        total = np.zeros((q_len, n), np.uint64)
        for p, e in enumerate(engines):
            e.load_records(0, dbs[p])
            e.query_upload(qs[p])
            e.set_batch(5)
            e.dot(0, n, 1)
            got = e.fetch_results(n)
            plain = oracle.dot_u16(qs[p], dbs[p])
            exp = oracle.mask_dot_shares(plain.T, 0, 64, 1, SEEDS[p][0], SEEDS[p][1], oracle.DOM_CODE_DOT, 0, 5).T
            assert np.array_equal(got, exp), f"party {p}"
            total += got
        plain_sum = sum(oracle.dot_u16(qs[p], dbs[p]).astype(np.uint64) for p in range(3))
        assert np.array_equal(total % 65536, plain_sum % 65536)
    finally:
        for e in engines:
            e.close()


def _iris_db(oracle, n, seed):
    codes, masks = [], []
    for i in range(n):
        c, m = oracle.iris_random(seed, i)
        codes.append(c)
        masks.append(m)
    return codes, masks


def test_check_shared_matmul_and_distances(dm, oracle):
    """check_shared_matmul / check_shared_distances on encoded irises."""
    import irisb200
    n, nq = 512, 32
    codes, masks = _iris_db(oracle, n, 0xABC)
    code_sh = [oracle.encode_iris_code(codes[i], masks[i], 1000 + i) for i in range(n)]
    mask_sh = [oracle.encode_mask_code(masks[i], 5000 + i) for i in range(n)]
    res_code, res_mask = [], []
    for p in range(3):
        ce = _engine(dm, p, n, nq, 12800, remote=True)
        me = _engine(dm, p, n, nq, 6400, remote=True)
        try:
            ce.load_records(0, np.stack([code_sh[i][p] for i in range(n)]))
            me.load_records(0, np.stack([mask_sh[i][p] for i in range(n)]))
            ce.query_upload(np.stack([oracle.preprocess_query(p, code_sh[i][p]) for i in range(nq)]))
            me.query_upload(np.stack([oracle.preprocess_query(p, mask_sh[i][p]) for i in range(nq)]))
            irisb200.dot_many([ce, me], [1, 2], 0, n)
            res_code.append(ce.fetch_results(n).astype(np.uint64))
            res_mask.append(me.fetch_results(n).astype(np.uint64))
        finally:
            ce.close()
            me.close()
    code_dot = (sum(res_code) % 65536).astype(np.uint16)
    mask_dot = (sum(res_mask) % 65536).astype(np.uint16)
    for qi in range(nq):
        for j in range(0, n, 37):
            m = masks[qi] & masks[j]
            mc = sum(bin(int(x)).count("1") for x in m)
            hd = sum(bin(int(x)).count("1") for x in ((codes[qi] ^ codes[j]) & m))
            assert int(mask_dot[qi, j]) == mc
            dist = 0.5 - (int(code_dot[qi, j]) - 65536 * (int(code_dot[qi, j]) >= 32768)) / (2.0 * mc)
            assert abs(dist - hd / mc) <= 1e-6
