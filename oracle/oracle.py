"""CPU oracle (test infrastructure only).

ctypes/numpy wrapper around ``oracle.c``, the plain-C restatement of the
reference algorithm for the iris uniqueness hot path.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import this
module, and only as the checker.  The product library never calls it.

Reference files restated here are cited per function in ``oracle.c``.
"""
from __future__ import annotations

import base64
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
IRIS_CODE_LENGTH = 12800
MASK_CODE_LENGTH = 6400
ROTATIONS = 31
CODE_COLS = 200

# Thresholds (iris-mpc-gpu/src/dot/mod.rs:10-15).
THRESHOLD_B = 1 << 16
THRESHOLD_A = int((1.0 - 2.0 * 0.345) * THRESHOLD_B)  # 20316
THRESHOLD_ANON_STATS_A = int((1.0 - 2.0 * 0.375) * THRESHOLD_B)  # 16384

DOM_CODE_DOT = 1
DOM_MASK_DOT = 2
DOM_CIRCUIT = 3

STAGE_FULL = 0
STAGE_MSB_ONLY = 1

_u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def _cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = line.split()
                    return "avx512bw" in flags and "avx512f" in flags
    except OSError:
        pass
    return False


def lib_paths():
    return os.path.join(HERE, "liboracle.so"), os.path.join(HERE, "liboracle_avx512.so")


def build(force: bool = False) -> None:
    """Compile the oracle with the Makefile next to this file."""
    base, wide = lib_paths()
    if force or not (os.path.exists(base) and os.path.exists(wide)) or \
            os.path.getmtime(base) < os.path.getmtime(os.path.join(HERE, "oracle.c")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def build_ref(ref_root: str | None = None) -> bool:
    """Compile the reference's ChaCha12 and Phase-1 kernels into _ref/ from a
    worldcoin/iris-mpc checkout at `ref_root` (default: the IRIS_REFERENCE
    environment variable).  One of the two is required: without a checkout
    there is nothing to compile, and the prebuilt cubins, if any, are used as
    they are.  Returns whether both cubins exist."""
    ref = ref_root or os.environ.get("IRIS_REFERENCE")
    if not ref:
        raise ValueError("build_ref needs the path of a worldcoin/iris-mpc checkout: pass ref_root or set "
                         "IRIS_REFERENCE")
    if not os.path.isdir(ref):
        raise ValueError(f"build_ref: {ref} is not a directory (expected a worldcoin/iris-mpc checkout)")
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={ref}"], check=True)
    return os.path.exists(REF_CHACHA_CUBIN) and os.path.exists(REF_DOT_CUBIN)


REF_CHACHA_CUBIN = os.path.join(HERE, "_ref", "chacha_ref.cubin")
REF_DOT_CUBIN = os.path.join(HERE, "_ref", "dot_ref.cubin")
_LIB = None


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    base, wide = lib_paths()
    if not os.path.exists(base):
        build()
    path = wide if (_cpu_has_avx512() and os.path.exists(wide)) else base
    L = C.CDLL(path)
    L.orc_gr4_mul.argtypes = [_u16p, _u16p, _u16p]
    L.orc_gr4_inv.argtypes = [_u16p, _u16p]
    L.orc_gr4_inv.restype = C.c_int
    L.orc_lagrange_at_zero.argtypes = [_u16p]
    L.orc_basis_mats.argtypes = [_u16p, _u16p, _u16p]
    L.orc_rng64.argtypes = [C.c_uint64, C.c_uint64]
    L.orc_rng64.restype = C.c_uint64
    L.orc_iris_random.argtypes = [C.c_uint64, C.c_uint64, _u64p, _u64p]
    L.orc_iris_flip.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, _u64p]
    L.orc_iris_rotate.argtypes = [_u64p, C.c_int]
    L.orc_iris_mirror.argtypes = [_u64p, _u64p, _u64p, _u64p]
    for f in ("orc_remap_new_to_old", "orc_remap_old_to_new", "orc_remap_new_to_mirrored"):
        getattr(L, f).argtypes = [C.c_int]
        getattr(L, f).restype = C.c_int
    L.orc_encode_iris_code.argtypes = [_u64p, _u64p, C.c_uint64, _u16p]
    L.orc_encode_mask_code.argtypes = [_u64p, C.c_uint64, _u16p]
    L.orc_preprocess_query.argtypes = [C.c_int, _u16p, C.c_int]
    L.orc_rotate_share.argtypes = [_u16p, _u16p, C.c_int, C.c_int]
    L.orc_mirror_share.argtypes = [_u16p, _u16p, C.c_int, C.c_int]
    L.orc_dot_u16.argtypes = [_u16p, C.c_int, _u16p, C.c_long, C.c_int, _u16p]
    L.orc_chacha_block.argtypes = [_u32p, C.c_uint64, C.c_uint64, C.c_int, _u32p]
    L.orc_chacha_fill.argtypes = [_u32p, C.c_uint64, C.c_uint64, C.c_int, _u32p, C.c_long]
    L.orc_or_tree.argtypes = [_u32p, C.c_long, _u32p, C.c_uint32, C.c_uint64, _u32p]
    L.orc_mask_dot_shares.argtypes = [_u16p, C.c_long, C.c_long, C.c_int, C.c_uint16, _u32p, _u32p,
                                      C.c_uint32, C.c_uint32, C.c_uint64]
    P = C.POINTER(C.c_void_p)
    L.orc_threshold_words.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.c_uint32, _u32p, C.c_uint32,
                                      C.c_uint64, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_match_predicate.argtypes = [C.c_uint16, C.c_uint16, C.c_uint32]
    L.orc_match_predicate.restype = C.c_int
    L.orc_cpu_plain_match.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_long,
                                      C.c_uint32, C.c_void_p, C.c_int]
    L.orc_cpu_plain_match.restype = C.c_long
    del P
    _LIB = L
    return L


def _ptrs(arrs):
    a = (C.c_void_p * len(arrs))(*[x.ctypes.data for x in arrs])
    return a


# --------------------------------------------------------------------------
# GR4 ring
# --------------------------------------------------------------------------
def gr4_mul(a, b):
    out = np.zeros(4, np.uint16)
    lib().orc_gr4_mul(np.asarray(a, np.uint16) if False else (np.array(a, dtype=np.int64) % 65536).astype(np.uint16),
                      (np.array(b, dtype=np.int64) % 65536).astype(np.uint16), out)
    return out


def gr4_inv(a):
    out = np.zeros(4, np.uint16)
    rc = lib().orc_gr4_inv((np.array(a, dtype=np.int64) % 65536).astype(np.uint16), out)
    if rc != 0:
        raise ZeroDivisionError(f"{a} is not a unit")
    return out


def lagrange_at_zero():
    out = np.zeros(12, np.uint16)
    lib().orc_lagrange_at_zero(out)
    return out.reshape(3, 4)


def basis_mats():
    s = np.zeros(16, np.uint16)
    b = np.zeros(16, np.uint16)
    lg = np.zeros(12, np.uint16)
    lib().orc_basis_mats(s, b, lg)
    return s.reshape(4, 4), b.reshape(4, 4), lg.reshape(3, 4)


# --------------------------------------------------------------------------
# Plaintext irises
# --------------------------------------------------------------------------
def iris_from_base64(s: str) -> np.ndarray:
    """IrisCodeArray::from_base64 (iris.rs:111-131): u64 from big-endian bytes, bit-reversed."""
    raw = base64.b64decode(s)
    assert len(raw) % 8 == 0
    words = np.frombuffer(raw, dtype=">u8").astype(np.uint64)
    out = np.zeros(len(words), np.uint64)
    for i, w in enumerate(words):
        out[i] = int(f"{int(w):064b}"[::-1], 2)
    return out


def iris_to_base64(words: np.ndarray) -> str:
    b = bytearray()
    for w in words:
        b += int(f"{int(w):064b}"[::-1], 2).to_bytes(8, "big")
    return base64.b64encode(bytes(b)).decode()


def bits_of(words: np.ndarray) -> np.ndarray:
    """Bit i of the iris = word i/64 bit i%64, as a uint8 array of 12800."""
    return np.unpackbits(words.astype("<u8").view(np.uint8), bitorder="little")[:IRIS_CODE_LENGTH]


def words_of(bits: np.ndarray) -> np.ndarray:
    return np.packbits(bits.astype(np.uint8), bitorder="little").view("<u8").astype(np.uint64)


def iris_random(seed: int, idx: int):
    code = np.zeros(200, np.uint64)
    mask = np.zeros(200, np.uint64)
    lib().orc_iris_random(seed, idx, code, mask)
    return code, mask


def iris_flip(seed: int, idx: int, p: float, code: np.ndarray) -> np.ndarray:
    out = code.copy()
    lib().orc_iris_flip(seed, idx, int(p * 2 ** 32), out)
    return out


def iris_rotate(bits_words: np.ndarray, by: int) -> np.ndarray:
    out = bits_words.copy()
    lib().orc_iris_rotate(out, int(by))
    return out


def iris_mirror(code, mask):
    oc = np.zeros(200, np.uint64)
    om = np.zeros(200, np.uint64)
    lib().orc_iris_mirror(np.ascontiguousarray(code), np.ascontiguousarray(mask), oc, om)
    return oc, om


def fractional_distance(c1, m1, c2, m2) -> float:
    """get_distance (iris.rs:534-548)."""
    m = np.bitwise_and(m1, m2)
    d = np.bitwise_and(np.bitwise_xor(c1, c2), m)
    return float(sum(bin(int(x)).count("1") for x in d)) / float(sum(bin(int(x)).count("1") for x in m))


def remap_new_to_old(i):
    return lib().orc_remap_new_to_old(int(i))


def remap_old_to_new(i):
    return lib().orc_remap_old_to_new(int(i))


def remap_new_to_mirrored(i):
    return lib().orc_remap_new_to_mirrored(int(i))


# --------------------------------------------------------------------------
# Shares
# --------------------------------------------------------------------------
def encode_iris_code(code, mask, seed: int) -> np.ndarray:
    out = np.zeros(3 * IRIS_CODE_LENGTH, np.uint16)
    lib().orc_encode_iris_code(np.ascontiguousarray(code), np.ascontiguousarray(mask), seed, out)
    return out.reshape(3, IRIS_CODE_LENGTH)


def encode_mask_code(mask, seed: int, trimmed: bool = True) -> np.ndarray:
    out = np.zeros(3 * IRIS_CODE_LENGTH, np.uint16)
    lib().orc_encode_mask_code(np.ascontiguousarray(mask), seed, out)
    out = out.reshape(3, IRIS_CODE_LENGTH)
    return np.ascontiguousarray(out[:, :MASK_CODE_LENGTH]) if trimmed else out


def preprocess_query(party: int, coefs: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(coefs, dtype=np.uint16).copy()
    lib().orc_preprocess_query(int(party), out, out.size)
    return out


def rotate_share(coefs: np.ndarray, r: int) -> np.ndarray:
    c = np.ascontiguousarray(coefs, dtype=np.uint16)
    out = np.zeros_like(c)
    lib().orc_rotate_share(c, out, c.size, int(r))
    return out


def all_rotations(coefs: np.ndarray) -> np.ndarray:
    return np.stack([rotate_share(coefs, r) for r in range(ROTATIONS)])


def mirror_share(coefs: np.ndarray, flip_imaginary: bool) -> np.ndarray:
    c = np.ascontiguousarray(coefs, dtype=np.uint16)
    out = np.zeros_like(c)
    lib().orc_mirror_share(c, out, c.size, int(flip_imaginary))
    return out


def trick_dot(a: np.ndarray, b: np.ndarray) -> int:
    return int((a.astype(np.uint64) * b.astype(np.uint64)).sum() % 65536)


def dot_u16(q: np.ndarray, d: np.ndarray) -> np.ndarray:
    """out[i][j] = sum_k q[i,k] d[j,k] mod 2^16."""
    q = np.ascontiguousarray(q, np.uint16)
    d = np.ascontiguousarray(d, np.uint16)
    nq, K = q.shape
    nd = d.shape[0]
    out = np.zeros((nq, nd), np.uint16)
    lib().orc_dot_u16(q, nq, d, nd, K, out)
    return out


# --------------------------------------------------------------------------
# ChaCha
# --------------------------------------------------------------------------
def seed_words(seed) -> np.ndarray:
    return np.ascontiguousarray(np.array(seed, dtype=np.uint32).reshape(8))


def chacha_block(key, counter: int, nonce: int, rounds: int = 12) -> np.ndarray:
    out = np.zeros(16, np.uint32)
    lib().orc_chacha_block(seed_words(key), counter, nonce, rounds, out)
    return out


def chacha_fill(key, counter: int, nonce: int, n_blocks: int, rounds: int = 12) -> np.ndarray:
    out = np.zeros(16 * n_blocks, np.uint32)
    lib().orc_chacha_fill(seed_words(key), counter, nonce, rounds, out, n_blocks)
    return out


def nonce_of(domain: int, dev: int) -> int:
    return (domain << 32) | dev


def counter_of(batch: int, blk: int) -> int:
    return (batch << 40) | blk


def mask_dot_shares(dots: np.ndarray, m0: int, q_pad: int, mult: int, key_own, key_prev,
                    domain: int, dev: int, batch: int) -> np.ndarray:
    """dots: [n_entries][q_pad] u16, returns masked copy."""
    d = np.ascontiguousarray(dots, np.uint16).copy()
    lib().orc_mask_dot_shares(d, m0, d.shape[0], q_pad, mult, seed_words(key_own), seed_words(key_prev),
                              domain, dev, batch)
    return d


# --------------------------------------------------------------------------
# Threshold protocol
# --------------------------------------------------------------------------
def threshold_words(code_parts, mask_parts, threshold_a: int, keys, dev: int = 0, batch: int = 0,
                    word_base: int = 0, stage: int = STAGE_FULL, want_lift: bool = False):
    """Run the 3-party circuit on additive components.

    code_parts/mask_parts: three u16 arrays (component p = party p's a share),
    length a multiple of 32.  keys: three 8-word seeds (stream p = party p's
    own seed).  Returns dict with res_a [3][W], res_b [3][W], revealed [W]
    (u32 words, bit j = element 32*w + j) and optionally lift outputs.
    """
    code_parts = [np.ascontiguousarray(x, np.uint16) for x in code_parts]
    mask_parts = [np.ascontiguousarray(x, np.uint16) for x in mask_parts]
    n = code_parts[0].size
    assert n % 32 == 0
    W = n // 32
    keys_arr = np.ascontiguousarray(np.stack([seed_words(k) for k in keys]).reshape(24))
    res_a = np.zeros((3, W), np.uint32)
    res_b = np.zeros((3, W), np.uint32)
    rev = np.zeros(W, np.uint32)
    lift_x = np.zeros((3, n), np.uint32) if want_lift else None
    corr = np.zeros((3, 2, n), np.uint16) if want_lift else None
    lib().orc_threshold_words(_ptrs(code_parts), _ptrs(mask_parts), W, threshold_a, keys_arr, dev, batch,
                              word_base, stage, res_a.ctypes.data, res_b.ctypes.data, rev.ctypes.data,
                              lift_x.ctypes.data if want_lift else None,
                              corr.ctypes.data if want_lift else None)
    out = {"res_a": res_a, "res_b": res_b, "revealed": rev}
    if want_lift:
        out["lift_x"] = lift_x
        out["corr"] = corr
    return out


def or_tree(comp, keys, dev: int = 0, batch: int = 0):
    """MPC OR of all bits of a shared u32 word vector (orc_or_tree): comp =
    three u32 arrays (component p = party p's a-share).  Returns (components
    [3] of the OR bit, opened bit)."""
    c = np.ascontiguousarray(np.stack([np.asarray(x, np.uint32) for x in comp]))
    keys_arr = np.ascontiguousarray(np.array(keys, np.uint32).reshape(3, 8))
    out = np.zeros(4, np.uint32)
    lib().orc_or_tree(c.reshape(-1), c.shape[1], keys_arr.reshape(-1), dev, batch, out)
    return out[:3].copy(), int(out[3])


def match_predicate(code, mask, threshold_a: int) -> np.ndarray:
    """bit31((mask*A - code*2^16 - 1) mod 2^32), vectorised (threshold.rs:110-124)."""
    code = np.asarray(code, np.uint64)
    mask = np.asarray(mask, np.uint64)
    r = (mask * np.uint64(threshold_a) - (code << np.uint64(16)) - np.uint64(1)) & np.uint64(0xFFFFFFFF)
    return ((r >> np.uint64(31)) & np.uint64(1)).astype(np.uint8)


def pack_bits_u32(bits: np.ndarray) -> np.ndarray:
    bits = np.asarray(bits, np.uint8).reshape(-1, 32)
    return (bits.astype(np.uint64) << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)


def cpu_plain_match(q_code, q_mask, n_query, db_code, db_mask, threshold_a, n_threads=0):
    """q_code[p]: [n_query*31][12800]; db_code[p]: [n_db][12800] ... -> bitmap [n_query][n_db] u8."""
    q_code = [np.ascontiguousarray(x, np.uint16) for x in q_code]
    q_mask = [np.ascontiguousarray(x, np.uint16) for x in q_mask]
    db_code = [np.ascontiguousarray(x, np.uint16) for x in db_code]
    db_mask = [np.ascontiguousarray(x, np.uint16) for x in db_mask]
    n_db = db_code[0].shape[0]
    bm = np.zeros((n_query, n_db), np.uint8)
    lib().orc_cpu_plain_match(_ptrs(q_code), _ptrs(q_mask), n_query, _ptrs(db_code), _ptrs(db_mask), n_db,
                              threshold_a, bm.ctypes.data, n_threads)
    return bm
