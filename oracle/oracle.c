/*
 * CPU oracle for the iris uniqueness hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is a plain-C restatement of the reference algorithm.  It is used
 * by tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of
 * bench.py as the checker; nothing in the product library links or calls it.
 *
 * What it restates (file:line in worldcoin/iris-mpc):
 *   - GR4 = Z_2^16[x]/(x^4 - x - 1): prod_monom, inv_monom, Lagrange
 *     coefficients at 0 over the base points {1, x, 1+x}, the basis-A ->
 *     monomial matrix S16 and monomial -> basis-B matrix (S S^T)^-1
 *       iris-mpc-common/src/sage/symmetric-gr-shamir_sage.sage:136-242,255-269
 *       iris-mpc-common/src/sage/gr4_encoding_example.sage:1-137
 *   - share encoding of iris code / mask bits, index remaps, mirroring,
 *     Lagrange preprocessing, rotations
 *       iris-mpc-common/src/galois_engine.rs:23-52,256-300,319-397,438-488,520-543
 *   - plaintext iris bits, rotations, mirror, fractional distance
 *       iris-mpc-common/src/iris_db/iris.rs:44-160,534-568,630-650
 *   - wrapping u16 dot products (trick_dot) and the row-major rotation-aware
 *     CPU kernel used as the timed CPU baseline
 *       iris-mpc-common/src/galois_engine.rs:54-97
 *       iris-mpc-cpu/src/protocol/ops.rs:238-341
 *   - ChaCha with 12 (or 20) rounds, 64-bit counter in words 12-13 and
 *     64-bit nonce in words 14-15
 *       iris-mpc-gpu/src/rng/chacha.cu:74-138, iris-mpc-gpu/src/rng/chacha.rs:205-250
 *   - the 3-party replicated-share threshold protocol: lift (3-input adder
 *     with two carries), bit injection, lift_mul_sub, extract_msb (32-bit
 *     3-input adder), open
 *       iris-mpc-gpu/src/threshold_ring/protocol.rs:610-661,1302-1643,
 *       1673-1872,2041-2074,2137-2359,2519-2546
 *       iris-mpc-gpu/src/threshold_ring/cuda/kernel.cu:12-270,334-426,526-629
 *   - the zero-share mask of the dot shares
 *       iris-mpc-gpu/src/dot/share_db.rs:815-821, iris-mpc-gpu/src/dot/kernel.cu:16-28
 *
 * The share-generation randomness (the external ampc-secret-sharing crate's
 * encode_3_mat and its StdRng stream) and the order in which the reference
 * consumes ChaCha keystream are not reproduced: this oracle and the CUDA path
 * share the position-addressable layout documented with each function below,
 * so per-party shares agree between them; revealed bits, bitmaps and indices
 * do not depend on the randomness at all.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint16_t u16;
typedef uint32_t u32;
typedef uint64_t u64;

#define IRIS_CODE_LENGTH 12800
#define MASK_CODE_LENGTH 6400
#define CODE_COLS 200
#define ROW_LEN 800
#define ROTATIONS 31

/* ------------------------------------------------------------------------ */
/* GR4 ring, monomial basis (symmetric-gr-shamir_sage.sage:150-166)          */
/* ------------------------------------------------------------------------ */
void orc_gr4_mul(const u16 *a, const u16 *b, u16 *out) {
    u32 a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3];
    u32 b0 = b[0], b1 = b[1], b2 = b[2], b3 = b[3];
    u32 d4 = a1 * b3 + a2 * b2 + a3 * b1; /* x^4 = 1 + x */
    u32 d5 = a2 * b3 + a3 * b2;           /* x^5 = x + x^2 */
    u32 d6 = a3 * b3;                     /* x^6 = x^2 + x^3 */
    out[0] = (u16)(a0 * b0 + d4);
    out[1] = (u16)(a0 * b1 + a1 * b0 + d4 + d5);
    out[2] = (u16)(a0 * b2 + a1 * b1 + a2 * b0 + d5 + d6);
    out[3] = (u16)(a0 * b3 + a1 * b2 + a2 * b1 + a3 * b0 + d6);
}

/* Inverse of a unit: a^(|GR*| - 1) with |GR(2^16,4)*| = 15 * 2^60. */
int orc_gr4_inv(const u16 *a, u16 *out) {
    if (!((a[0] | a[1] | a[2] | a[3]) & 1)) return -1; /* all even: not a unit */
    u64 e = 15ull * (1ull << 60) - 1ull;
    u16 r[4] = {1, 0, 0, 0}, base[4] = {a[0], a[1], a[2], a[3]}, t[4];
    while (e) {
        if (e & 1) { orc_gr4_mul(r, base, t); memcpy(r, t, sizeof t); }
        orc_gr4_mul(base, base, t); memcpy(base, t, sizeof t);
        e >>= 1;
    }
    /* check: a * r == 1 */
    orc_gr4_mul(a, r, t);
    if (t[0] != 1 || t[1] || t[2] || t[3]) return -2;
    memcpy(out, r, sizeof r);
    return 0;
}

/* Base points of the three parties: 1, x, 1+x. */
static const u16 BASE_POINTS[3][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {1, 1, 0, 0}};

/* Lagrange coefficients at 0 for degree-2 polynomials over the base points
 * (deg_2_lagrange_polys_at_zero; sage legrange_coeffs at z = 0). */
void orc_lagrange_at_zero(u16 *out /* [3][4] */) {
    for (int i = 0; i < 3; i++) {
        u16 c[4] = {1, 0, 0, 0}, t[4], d[4], inv[4];
        for (int j = 0; j < 3; j++) {
            if (j == i) continue;
            u16 negq[4], pq[4];
            for (int k = 0; k < 4; k++) {
                negq[k] = (u16)(0 - BASE_POINTS[j][k]);
                pq[k] = (u16)(BASE_POINTS[i][k] - BASE_POINTS[j][k]);
            }
            orc_gr4_mul(c, negq, t);
            orc_gr4_inv(pq, inv);
            orc_gr4_mul(t, inv, d);
            memcpy(c, d, sizeof c);
        }
        memcpy(out + 4 * i, c, sizeof c);
    }
}

/* S16: basis A -> monomial (gr4_encoding_example.sage:5-10). */
static const u16 S16[4][4] = {
    {1, 0, 0, 0}, {58082, 1, 0, 0}, {60579, 25194, 1, 0}, {17325, 51956, 57011, 1}};
static u16 BMAT[4][4]; /* (S S^T)^-1: monomial -> basis B */
static u16 LAGRANGE[3][4];
static int g_init = 0;

static void mat_inv_lower_unit(const u16 L[4][4], u16 out[4][4]) {
    /* forward substitution mod 2^16 for a unit lower-triangular matrix */
    memset(out, 0, sizeof(u16) * 16);
    for (int c = 0; c < 4; c++) {
        for (int r = 0; r < 4; r++) {
            u32 v = (r == c) ? 1u : 0u;
            for (int k = 0; k < r; k++) v -= (u32)L[r][k] * out[k][c];
            out[r][c] = (u16)v;
        }
    }
}

void orc_init(void) {
    if (g_init) return;
    u16 Sinv[4][4];
    mat_inv_lower_unit(S16, Sinv);
    /* (S S^T)^-1 = (S^-1)^T S^-1 */
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            u32 v = 0;
            for (int k = 0; k < 4; k++) v += (u32)Sinv[k][i] * Sinv[k][j];
            BMAT[i][j] = (u16)v;
        }
    orc_lagrange_at_zero(&LAGRANGE[0][0]);
    g_init = 1;
}

void orc_basis_mats(u16 *s_out, u16 *b_out, u16 *lagrange_out) {
    orc_init();
    memcpy(s_out, S16, sizeof S16);
    memcpy(b_out, BMAT, sizeof BMAT);
    memcpy(lagrange_out, LAGRANGE, sizeof LAGRANGE);
}

static void matvec(const u16 M[4][4], const u16 *v, u16 *out) {
    for (int i = 0; i < 4; i++) {
        u32 s = 0;
        for (int j = 0; j < 4; j++) s += (u32)M[i][j] * v[j];
        out[i] = (u16)s;
    }
}

/* ------------------------------------------------------------------------ */
/* Position-addressable generator shared (as a definition) with the CUDA     */
/* synthetic-data kernels: splitmix64 of seed + counter * golden ratio.      */
/* ------------------------------------------------------------------------ */
static inline u64 mix64(u64 z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
u64 orc_rng64(u64 seed, u64 ctr) { return mix64(seed + (ctr + 1) * 0x9E3779B97F4A7C15ull); }

/* ------------------------------------------------------------------------ */
/* Plaintext iris codes: 200 u64 words, bit i = word i/64 bit i%64           */
/* (iris.rs:44-90).                                                          */
/* ------------------------------------------------------------------------ */
static inline int get_bit(const u64 *w, int i) { return (int)((w[i >> 6] >> (i & 63)) & 1); }
static inline void set_bit(u64 *w, int i, int v) {
    if (v) w[i >> 6] |= 1ull << (i & 63); else w[i >> 6] &= ~(1ull << (i & 63));
}

/* Synthetic iris number `idx` of stream `seed`: code bits uniform, mask kept
 * per real/imaginary pair (bits 2i, 2i+1) with probability 0.9
 * (iris.rs:244-260 keeps mask pairs equal; the keep rate is the workload's). */
#define MASK_KEEP_THRESHOLD 3865470566u /* 0.9 * 2^32 */
void orc_iris_random(u64 seed, u64 idx, u64 *code, u64 *mask) {
    u64 s = mix64(seed ^ (idx * 0xD1B54A32D192ED03ull));
    for (int w = 0; w < 200; w++) code[w] = orc_rng64(s, (u64)w);
    memset(mask, 0, 200 * sizeof(u64));
    for (int p = 0; p < IRIS_CODE_LENGTH / 2; p++) {
        u64 r = orc_rng64(s ^ 0x5bd1e995ull, (u64)(p >> 1));
        u32 v = (p & 1) ? (u32)(r >> 32) : (u32)r;
        if (v < MASK_KEEP_THRESHOLD) mask[(2 * p) >> 6] |= 3ull << ((2 * p) & 63);
    }
}

/* Flip every code bit independently with probability p_num / 2^32. */
void orc_iris_flip(u64 seed, u64 idx, u32 p_num, u64 *code) {
    u64 s = mix64(seed ^ (idx * 0x9FB21C651E98DF25ull) ^ 0x1234567ull);
    for (int i = 0; i < IRIS_CODE_LENGTH; i++) {
        u64 r = orc_rng64(s, (u64)(i >> 1));
        u32 v = (i & 1) ? (u32)(r >> 32) : (u32)r;
        if (v < p_num) code[i >> 6] ^= 1ull << (i & 63);
    }
}

/* Rotate the bits of every 800-bit row by 4*by (by > 0: right, by < 0: left)
 * (IrisCodeArray::rotate_right / rotate_left, iris.rs:140-152). */
void orc_iris_rotate(u64 *bits, int by) {
    u64 tmp[200];
    memset(tmp, 0, sizeof tmp);
    int sh = ((by % CODE_COLS) + CODE_COLS) % CODE_COLS * 4;
    for (int i = 0; i < IRIS_CODE_LENGTH; i++) {
        int row = i / ROW_LEN, col = i % ROW_LEN;
        int dst = row * ROW_LEN + (col + sh) % ROW_LEN;
        set_bit(tmp, dst, get_bit(bits, i));
    }
    memcpy(bits, tmp, sizeof tmp);
}

/* Index remaps (galois_engine.rs:256-285). */
int orc_remap_new_to_old(int i) {
    int b = i / 6400, w = i % 6400 / 3200, r1 = i % 3200 / 800, c = i % 800 / 4, r2 = i % 4;
    int r = r2 * 4 + r1;
    return 800 * r + c * 4 + w * 2 + b;
}
int orc_remap_old_to_new(int i) {
    int r = i / 800, c = i % 800 / 4, w = i % 4 / 2, b = i % 2;
    int r1 = r % 4, r2 = r / 4;
    return b * 6400 + w * 3200 + r1 * 800 + c * 4 + r2;
}
int orc_remap_new_to_mirrored(int i) {
    int b = i / 6400, w = i % 6400 / 3200, r1 = i % 3200 / 800, c = i % 800 / 4, r2 = i % 4;
    int fc = (c < 100) ? (100 - 1 - c) : (199 - (c - 100));
    return b * 6400 + w * 3200 + r1 * 800 + fc * 4 + r2;
}

/* IrisCode::mirrored (iris.rs:630-650). */
void orc_iris_mirror(const u64 *code, const u64 *mask, u64 *out_code, u64 *out_mask) {
    memset(out_code, 0, 200 * 8);
    memset(out_mask, 0, 200 * 8);
    for (int i = 0; i < IRIS_CODE_LENGTH; i++) {
        int mi = orc_remap_new_to_old(orc_remap_new_to_mirrored(orc_remap_old_to_new(i)));
        set_bit(out_mask, mi, get_bit(mask, i));
        int cb = get_bit(code, i);
        set_bit(out_code, mi, (i % 2 == 0) ? cb : !cb);
    }
}

/* ------------------------------------------------------------------------ */
/* Share encoding (galois_engine.rs:319-397).  A block of 4 coefficients is  */
/* one GR4 element in basis A, converted to the monomial basis, then shared  */
/* with a degree-1 Shamir polynomial s + r*X evaluated at 1, x, 1+x (the     */
/* product of two such sharings has degree 2, reconstructed by the degree-2  */
/* Lagrange coefficients).  r comes from orc_rng64(seed, block).             */
/* ------------------------------------------------------------------------ */
static void share_block(const u16 *a_basis, u64 seed, u64 block, u16 out[3][4]) {
    u16 s[4];
    matvec(S16, a_basis, s);
    u64 rr = orc_rng64(seed, block);
    u16 r[4] = {(u16)rr, (u16)(rr >> 16), (u16)(rr >> 32), (u16)(rr >> 48)};
    for (int p = 0; p < 3; p++) {
        u16 t[4];
        orc_gr4_mul(r, BASE_POINTS[p], t);
        for (int k = 0; k < 4; k++) out[p][k] = (u16)(s[k] + t[k]);
    }
}

/* shares: [3][12800] */
void orc_encode_iris_code(const u64 *code, const u64 *mask, u64 seed, u16 *shares) {
    orc_init();
    for (int i = 0; i < IRIS_CODE_LENGTH; i += 4) {
        u16 v[4], sh[3][4];
        for (int k = 0; k < 4; k++) {
            int o = orc_remap_new_to_old(i + k);
            u16 m = (u16)get_bit(mask, o), c = (u16)get_bit(code, o);
            v[k] = (u16)(m - 2 * (c & m));
        }
        share_block(v, seed, (u64)(i / 4), sh);
        for (int p = 0; p < 3; p++)
            for (int k = 0; k < 4; k++) shares[p * IRIS_CODE_LENGTH + i + k] = sh[p][k];
    }
}

void orc_encode_mask_code(const u64 *mask, u64 seed, u16 *shares) {
    orc_init();
    for (int i = 0; i < IRIS_CODE_LENGTH; i += 4) {
        u16 v[4], sh[3][4];
        for (int k = 0; k < 4; k++) v[k] = (u16)get_bit(mask, orc_remap_new_to_old(i + k));
        share_block(v, seed ^ 0xabcdef12345ull, (u64)(i / 4), sh);
        for (int p = 0; p < 3; p++)
            for (int k = 0; k < 4; k++) shares[p * IRIS_CODE_LENGTH + i + k] = sh[p][k];
    }
}

/* preprocess_coefs (galois_engine.rs:23-40): x Lagrange(id), to basis B. */
void orc_preprocess_query(int party, u16 *coefs, int n) {
    orc_init();
    for (int i = 0; i < n; i += 4) {
        u16 t[4], b[4];
        orc_gr4_mul(coefs + i, LAGRANGE[party], t);
        matvec(BMAT, t, b);
        memcpy(coefs + i, b, sizeof b);
    }
}

/* Rotation index r in 0..30 of all_rotations(): net rotate_left by 15 - r
 * coefficient blocks of each 800-coef row (galois_engine.rs:42-52,197-206). */
void orc_rotate_share(const u16 *in, u16 *out, int n, int r) {
    int left = (15 - r) * 4; /* may be negative = right rotation */
    for (int row = 0; row < n / ROW_LEN; row++)
        for (int j = 0; j < ROW_LEN; j++) {
            int src = ((j + left) % ROW_LEN + ROW_LEN) % ROW_LEN;
            out[row * ROW_LEN + j] = in[row * ROW_LEN + src];
        }
}

/* mirrored_code / mirrored_mask (galois_engine.rs:218-225,520-543).  The
 * imaginary-half flip subtracts from a sharing of zero; this oracle uses the
 * all-zero sharing (the reference draws a fixed one from StdRng(0)). */
void orc_mirror_share(const u16 *in, u16 *out, int n, int flip_imaginary) {
    u16 tmp[IRIS_CODE_LENGTH];
    memcpy(tmp, in, (size_t)n * 2);
    if (flip_imaginary)
        for (int i = IRIS_CODE_LENGTH / 2; i < n; i++) tmp[i] = (u16)(0 - tmp[i]);
    for (int i = 0; i < n; i++) out[orc_remap_new_to_mirrored(i)] = tmp[i];
}

/* ------------------------------------------------------------------------ */
/* Wrapping u16 dot products (trick_dot, galois_engine.rs:54-60).            */
/* out[q][d] = sum_k q[q][k] * d[d][k] mod 2^16                              */
/* ------------------------------------------------------------------------ */
void orc_dot_u16(const u16 *q, int nq, const u16 *d, long nd, int K, u16 *out) {
#pragma omp parallel for schedule(static)
    for (long j = 0; j < nd; j++)
        for (int i = 0; i < nq; i++) {
            const u16 *a = q + (long)i * K, *b = d + j * K;
            u32 s = 0;
            for (int k = 0; k < K; k++) s += (u32)a[k] * b[k];
            out[(long)i * nd + j] = (u16)s;
        }
}

/* ------------------------------------------------------------------------ */
/* ChaCha block (chacha.cu:74-138): state = constants | key | counter | nonce */
/* ------------------------------------------------------------------------ */
#define ROTL(v, n) (((v) << (n)) | ((v) >> (32 - (n))))
#define QR(x, a, b, c, d)                                                        \
    x[a] += x[b]; x[d] ^= x[a]; x[d] = ROTL(x[d], 16);                           \
    x[c] += x[d]; x[b] ^= x[c]; x[b] = ROTL(x[b], 12);                           \
    x[a] += x[b]; x[d] ^= x[a]; x[d] = ROTL(x[d], 8);                            \
    x[c] += x[d]; x[b] ^= x[c]; x[b] = ROTL(x[b], 7);

void orc_chacha_block(const u32 *key, u64 counter, u64 nonce, int rounds, u32 *out) {
    u32 s[16] = {0x61707865, 0x3320646e, 0x79622d32, 0x6b206574};
    for (int i = 0; i < 8; i++) s[4 + i] = key[i];
    s[12] = (u32)counter; s[13] = (u32)(counter >> 32);
    s[14] = (u32)nonce; s[15] = (u32)(nonce >> 32);
    u32 x[16];
    memcpy(x, s, sizeof s);
    for (int i = 0; i < rounds / 2; i++) {
        QR(x, 0, 4, 8, 12) QR(x, 1, 5, 9, 13) QR(x, 2, 6, 10, 14) QR(x, 3, 7, 11, 15)
        QR(x, 0, 5, 10, 15) QR(x, 1, 6, 11, 12) QR(x, 2, 7, 8, 13) QR(x, 3, 4, 9, 14)
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

/* Keystream fill: out[16*i + j] = block(counter + i)[j]  (chacha.cu:140-161). */
void orc_chacha_fill(const u32 *key, u64 counter, u64 nonce, int rounds, u32 *out, long n_blocks) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n_blocks; i++) orc_chacha_block(key, counter + (u64)i, nonce, rounds, out + 16 * i);
}

/* Keystream domains (nonce high word) and counter layout shared with the
 * CUDA path:  nonce = (domain << 32) | device_index;
 *             counter = (batch << 40) | block_within_batch.                */
#define DOM_CODE_DOT 1u
#define DOM_MASK_DOT 2u
#define DOM_CIRCUIT 3u
#define CIRCUIT_BLOCKS_PER_WORD 8 /* 128 keystream words per 32-element word */

static inline u64 nonce_of(u32 domain, u32 dev) { return ((u64)domain << 32) | dev; }
static inline u64 counter_of(u64 batch, u64 blk) { return (batch << 40) | blk; }

/* Zero-share mask of one party's dot shares (share_db.rs:815-821 and the
 * reduce kernel, kernel.cu:16-28): out = dot * mult + ks_own - ks_prev, with
 * the u16 keystream index of element (entry m, padded row n) equal to
 * m * q_pad + n (element-major over the whole DB, independent of chunking).
 * dots: [n_entries][q_pad] u16 for entries m0..m0+n_entries-1. */
void orc_mask_dot_shares(u16 *dots, long m0, long n_entries, int q_pad, u16 mult,
                         const u32 *key_own, const u32 *key_prev, u32 domain, u32 dev, u64 batch) {
    u64 nonce = nonce_of(domain, dev);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n_entries; j++) {
        for (int n = 0; n < q_pad; n += 32) {
            u64 e = (u64)(m0 + j) * (u64)q_pad + (u64)n; /* multiple of 32 when q_pad % 32 == 0 */
            u32 k0[16], k1[16];
            orc_chacha_block(key_own, counter_of(batch, e / 32), nonce, 12, k0);
            orc_chacha_block(key_prev, counter_of(batch, e / 32), nonce, 12, k1);
            for (int t = 0; t < 32 && n + t < q_pad; t++) {
                u16 r0 = (u16)(k0[t / 2] >> (16 * (t & 1)));
                u16 r1 = (u16)(k1[t / 2] >> (16 * (t & 1)));
                u16 *v = &dots[j * q_pad + n + t];
                *v = (u16)(*v * mult + r0 - r1);
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* 3-party replicated-share threshold protocol, one 32-element word at a     */
/* time.  Party p holds (a, b) = (component p, component p-1); a gate's      */
/* "send a to next, receive b from prev" is the explicit copy in reshare().  */
/* ------------------------------------------------------------------------ */
typedef struct { u32 a, b; } rs; /* one party's view of one bit plane */

/* Randomness of one word: ks[s][0..127] = stream s (party s's own seed). */
typedef struct { u32 ks[3][128]; } word_rand;

static void fill_word_rand(const u32 *keys /* [3][8] */, u32 dev, u64 batch, u64 word, word_rand *wr) {
    u64 nonce = nonce_of(DOM_CIRCUIT, dev);
    for (int s = 0; s < 3; s++)
        for (int j = 0; j < CIRCUIT_BLOCKS_PER_WORD; j++)
            orc_chacha_block(keys + 8 * s, counter_of(batch, word * CIRCUIT_BLOCKS_PER_WORD + j), nonce, 12,
                             wr->ks[s] + 16 * j);
}

/* and_pre_inner (kernel.cu:37-41) with r = ks_own ^ ks_prev (fill_rng_into,
 * chacha_corr.rs:54-57), followed by the reshare: party p sends its new a to
 * p+1 and receives its new b from p-1. */
static void and_gate(const rs x[3], const rs y[3], rs z[3], const word_rand *wr, int gate) {
    u32 local[3];
    for (int p = 0; p < 3; p++) {
        u32 r = wr->ks[p][gate] ^ wr->ks[(p + 2) % 3][gate];
        local[p] = (x[p].a & y[p].a) ^ (x[p].b & y[p].a) ^ (x[p].a & y[p].b) ^ r;
    }
    for (int p = 0; p < 3; p++) { z[p].a = local[p]; z[p].b = local[(p + 2) % 3]; }
}
static void xor3(const rs x[3], const rs y[3], rs z[3]) {
    for (int p = 0; p < 3; p++) { z[p].a = x[p].a ^ y[p].a; z[p].b = x[p].b ^ y[p].b; }
}

/* split_inner (kernel.cu:204-234): the replicated views of the three additive
 * share components as separate shared values x1, x2, x3. */
static void split(const rs in[3], rs x1[3], rs x2[3], rs x3[3]) {
    memset(x1, 0, sizeof(rs) * 3); memset(x2, 0, sizeof(rs) * 3); memset(x3, 0, sizeof(rs) * 3);
    x1[0].a = in[0].a; x3[0].b = in[0].b;
    x1[1].b = in[1].b; x2[1].a = in[1].a;
    x2[2].b = in[2].b; x3[2].a = in[2].a;
}

/* binary_add_3_get_two_carries (protocol.rs:2137-2241), K = 16.
 * planes[k][p]: party p's view of bit k.  Keystream word of each AND gate:
 * carry-save AND of plane k -> 2k (k < 15) or 30 (k = 15); ripple step k ->
 * 2k + 1; final AND -> 31. */
static void add3_two_carries(rs planes[16][3], rs c1[3], rs c2[3], const word_rand *wr) {
    rs x1[16][3], x2[16][3], x3[16][3], s[16][3], c[16][3];
    for (int k = 0; k < 16; k++) split(planes[k], x1[k], x2[k], x3[k]);
    for (int k = 0; k < 16; k++) {
        xor3(x2[k], x3[k], x2[k]);                 /* x2x3 */
        if (k > 0) xor3(x1[k], x2[k], s[k - 1]);   /* s[k-1] = bit k of the carry-save sum */
        xor3(x1[k], x3[k], x1[k]);                 /* x1x3 */
        and_gate(x1[k], x2[k], c[k], wr, k < 15 ? 2 * k : 30); /* carry-save gates */
        xor3(c[k], x3[k], c[k]);
    }
    rs carry[3], t[3];
    and_gate(s[0], c[0], carry, wr, 1);
    for (int k = 1; k < 15; k++) {
        xor3(s[k], carry, s[k]);
        xor3(c[k], carry, c[k]);
        and_gate(s[k], c[k], t, wr, 2 * k + 1);    /* ripple gates */
        xor3(carry, t, carry);
    }
    and_gate(c[15], carry, c2, wr, 31);
    xor3(carry, c[15], c1);
}

/* binary_add_3_get_msb (protocol.rs:2262-2359), 32 bits.  Keystream word of
 * each AND gate: carry-save AND of plane k -> 32 + 2k; ripple step k -> 33 + 2k. */
static void add3_msb(rs planes[32][3], rs msb[3], const word_rand *wr) {
    rs x1[32][3], x2[32][3], x3[32][3], s[31][3], c[31][3];
    for (int k = 0; k < 32; k++) split(planes[k], x1[k], x2[k], x3[k]);
    for (int k = 0; k < 32; k++) {
        xor3(x2[k], x3[k], x2[k]);
        if (k > 0) xor3(x1[k], x2[k], s[k - 1]);
        if (k < 31) {
            xor3(x1[k], x3[k], x1[k]);
            and_gate(x1[k], x2[k], c[k], wr, 32 + 2 * k);
            xor3(c[k], x3[k], c[k]);
        }
    }
    rs carry[3], t[3];
    and_gate(s[0], c[0], carry, wr, 33);
    for (int k = 1; k < 30; k++) {
        xor3(s[k], carry, s[k]);
        xor3(c[k], carry, c[k]);
        and_gate(s[k], c[k], t, wr, 33 + 2 * k);
        xor3(carry, t, carry);
    }
    xor3(carry, s[30], msb);
    xor3(msb, c[30], msb);
}

/* bit_inject_party_{0,1,2} (protocol.rs:1302-1643, kernel.cu:526-629) for
 * 32 elements.  bits[p]: party p's view of the bit plane.  out[p][j]: party
 * p's arithmetic (a, b) for element j.  Randomness: u16 number j of keystream
 * words [off, off+16) -- r01 from stream 0, r12 from stream 1, r02 from
 * stream 2; off = 96 for the first carry, 112 for the second. */
static void bit_inject(const rs bits[3], u16 out_a[3][32], u16 out_b[3][32], const word_rand *wr, int off) {
    for (int j = 0; j < 32; j++) {
        u16 r01 = (u16)(wr->ks[0][off + j / 2] >> (16 * (j & 1)));
        u16 r12 = (u16)(wr->ks[1][off + j / 2] >> (16 * (j & 1)));
        u16 r02 = (u16)(wr->ks[2][off + j / 2] >> (16 * (j & 1)));
        u16 b0a = (u16)((bits[0].a >> j) & 1), b0b = (u16)((bits[0].b >> j) & 1);
        u16 b1a = (u16)((bits[1].a >> j) & 1), b1b = (u16)((bits[1].b >> j) & 1);
        u16 b2a = (u16)((bits[2].a >> j) & 1);
        (void)b0a;
        /* party 1: x = (a ^ b) - r01, sent to party 2 */
        u16 x = (u16)((b1a ^ b1b) - r01);
        /* party 0: y = b * r01 - r02, sent to party 1 */
        u16 y = (u16)(b0b * r01 - r02);
        /* party 2: z = a * x - r12, sent to party 0 */
        u16 z = (u16)(b2a * x - r12);
        /* party 0 */
        out_a[0][j] = (u16)(r01 - (u16)(y << 1));
        out_b[0][j] = (u16)((u16)(0 - (u16)((u16)(r02 + z) << 1)) + b0b);
        /* party 1 */
        out_a[1][j] = (u16)(x - (u16)(r12 << 1));
        out_b[1][j] = (u16)(r01 - (u16)(y << 1));
        /* party 2 */
        out_a[2][j] = (u16)((u16)(0 - (u16)((u16)(r02 + z) << 1)) + b2a);
        out_b[2][j] = (u16)(x - (u16)(r12 << 1));
    }
}

static void u16_to_planes(const u16 v[32], u32 planes[16]) {
    for (int k = 0; k < 16; k++) {
        u32 w = 0;
        for (int j = 0; j < 32; j++) w |= (u32)((v[j] >> k) & 1) << j;
        planes[k] = w;
    }
}
static void u32_to_planes(const u32 v[32], u32 planes[32]) {
    for (int k = 0; k < 32; k++) {
        u32 w = 0;
        for (int j = 0; j < 32; j++) w |= ((v[j] >> k) & 1u) << j;
        planes[k] = w;
    }
}

/* Mode flags for orc_threshold_words. */
#define ORC_STAGE_FULL 0    /* lift(mask) -> mul_sub -> msb   (compare_threshold_masked_many) */
#define ORC_STAGE_MSB_ONLY 1 /* mask treated as 0 and corrections as 0 (extract_msb test) */

/*
 * compare_threshold_masked_many for n_words words of 32 elements.
 * code[p], mask[p]: party p's additive component (its `a`), [n_words*32] u16;
 * party p's `b` is component p-1.  word_base: index of the first word in the
 * keystream layout.  Outputs (each optional):
 *   res_a[p][w], res_b[p][w]: party p's view of the msb plane;
 *   revealed[w]: a ^ b ^ c (the opened comparison bits).
 *   lift_x[p][e], corr[p][2][e]: party p's (a) lifted mask and injected
 *   corrections (lift_mpc outputs) when non-NULL.
 */
void orc_threshold_words(const u16 *const *code, const u16 *const *mask, long n_words, u32 threshold_a,
                         const u32 *keys, u32 dev, u64 batch, u64 word_base, int stage,
                         u32 *res_a, u32 *res_b, u32 *revealed, u32 *lift_x, u16 *corr) {
#pragma omp parallel for schedule(static)
    for (long w = 0; w < n_words; w++) {
        word_rand wr;
        fill_word_rand(keys, dev, batch, word_base + (u64)w, &wr);
        u16 m[3][32], c[3][32];
        for (int p = 0; p < 3; p++)
            for (int j = 0; j < 32; j++) {
                m[p][j] = stage == ORC_STAGE_MSB_ONLY ? 0 : mask[p][w * 32 + j];
                c[p][j] = code[p][w * 32 + j];
            }
        u16 inj1_a[3][32], inj1_b[3][32], inj2_a[3][32], inj2_b[3][32];
        if (stage == ORC_STAGE_FULL) {
            /* lift_mpc (protocol.rs:2041-2074): transpose, split, adder, inject */
            u32 pl[3][16];
            for (int p = 0; p < 3; p++) u16_to_planes(m[p], pl[p]);
            rs planes[16][3];
            for (int k = 0; k < 16; k++)
                for (int p = 0; p < 3; p++) { planes[k][p].a = pl[p][k]; planes[k][p].b = pl[(p + 2) % 3][k]; }
            rs c1[3], c2[3];
            add3_two_carries(planes, c1, c2, &wr);
            bit_inject(c1, inj1_a, inj1_b, &wr, 96);
            bit_inject(c2, inj2_a, inj2_b, &wr, 112);
        } else {
            memset(inj1_a, 0, sizeof inj1_a); memset(inj1_b, 0, sizeof inj1_b);
            memset(inj2_a, 0, sizeof inj2_a); memset(inj2_b, 0, sizeof inj2_b);
        }
        /* lift_mul_sub (kernel.cu:181-195,407-426) */
        u32 xa[3][32], xb[3][32];
        for (int p = 0; p < 3; p++) {
            int q = (p + 2) % 3;
            for (int j = 0; j < 32; j++) {
                u32 ma = (u32)m[p][j] - ((u32)inj1_a[p][j] << 16) - ((u32)inj2_a[p][j] << 17);
                u32 mb = (u32)m[q][j] - ((u32)inj1_b[p][j] << 16) - ((u32)inj2_b[p][j] << 17);
                if (lift_x) lift_x[(long)p * n_words * 32 + w * 32 + j] = (u32)m[p][j];
                if (corr) {
                    corr[((long)p * 2 + 0) * n_words * 32 + w * 32 + j] = inj1_a[p][j];
                    corr[((long)p * 2 + 1) * n_words * 32 + w * 32 + j] = inj2_a[p][j];
                }
                xa[p][j] = ma * threshold_a - ((u32)c[p][j] << 16);
                xb[p][j] = mb * threshold_a - ((u32)c[q][j] << 16);
                if (p == 0) xa[p][j] -= 1;
                if (p == 1) xb[p][j] -= 1;
            }
        }
        /* extract_msb (protocol.rs:2243-2258) */
        u32 pa[3][32], pb[3][32];
        for (int p = 0; p < 3; p++) { u32_to_planes(xa[p], pa[p]); u32_to_planes(xb[p], pb[p]); }
        rs planes32[32][3];
        for (int k = 0; k < 32; k++)
            for (int p = 0; p < 3; p++) { planes32[k][p].a = pa[p][k]; planes32[k][p].b = pb[p][k]; }
        rs msb[3];
        add3_msb(planes32, msb, &wr);
        for (int p = 0; p < 3; p++) {
            if (res_a) res_a[(long)p * n_words + w] = msb[p].a;
            if (res_b) res_b[(long)p * n_words + w] = msb[p].b;
        }
        /* open (actor.rs:2928-2997): a ^ b ^ (third component from prev) */
        if (revealed) revealed[w] = msb[0].a ^ msb[0].b ^ msb[2].b;
    }
}

/* The match predicate of the plaintext values (threshold.rs:110-124):
 * bit31((mask * A - code * 2^16 - 1) mod 2^32). */
/* MPC OR tree (or_reduce_result / or_tree_on_gpu, protocol.rs:2363-2515):
 * comp [3][n] = the three components (party p's a-shares) of a bit vector in
 * u32 words.  Each level ORs word i with word i + num (num = half, rounded
 * down) and moves an odd last word down; the last word's 32 bits are then
 * collapsed with shifts 16, 8, 4, 2, 1.  OR(x, y) = x ^ y ^ AND(x, y); the AND
 * gate of level L, index i takes word 0 of the ChaCha12 block at counter
 * (batch << 40) | (L << 34) | i of each party's stream (nonce domain 4), party
 * p masking with k_p ^ k_{p-1}.  out[0..2] = components of the OR bit, out[3]
 * = the opened bit.  comp is overwritten. */
#define DOM_OR_TREE 4u
static void or_gate(u32 x[3], const u32 y[3], const u32 *keys, u32 dev, u64 batch, u64 gate) {
    u32 k[3], blk[16], z[3];
    for (int s = 0; s < 3; s++) {
        orc_chacha_block(keys + 8 * s, counter_of(batch, gate), nonce_of(DOM_OR_TREE, dev), 12, blk);
        k[s] = blk[0];
    }
    for (int p = 0; p < 3; p++) {
        int q = (p + 2) % 3;
        z[p] = (x[p] & y[p]) ^ (x[q] & y[p]) ^ (x[p] & y[q]) ^ (k[p] ^ k[q]);
    }
    for (int p = 0; p < 3; p++) x[p] = x[p] ^ y[p] ^ z[p];
}

void orc_or_tree(u32 *comp, long n, const u32 *keys, u32 dev, u64 batch, u32 *out) {
    long num = n;
    u64 level = 1;
    while (num > 1) {
        long odd = num & 1;
        num >>= 1;
        for (long i = 0; i < num; i++) {
            u32 x[3], y[3];
            for (int p = 0; p < 3; p++) { x[p] = comp[p * n + i]; y[p] = comp[p * n + i + num]; }
            or_gate(x, y, keys, dev, batch, (level << 34) | (u64)i);
            for (int p = 0; p < 3; p++) comp[p * n + i] = x[p];
        }
        if (odd)
            for (int p = 0; p < 3; p++) comp[p * n + num] = comp[p * n + 2 * num];
        num += odd;
        level++;
    }
    u32 x[3] = {comp[0], comp[n], comp[2 * n]};
    int j = 0;
    for (int sh = 16; sh >= 1; sh >>= 1, j++) {
        u32 y[3] = {x[0] >> sh, x[1] >> sh, x[2] >> sh};
        or_gate(x, y, keys, dev, batch, (u64)(40 + j) << 34);
    }
    for (int p = 0; p < 3; p++) out[p] = x[p] & 1u;
    out[3] = (x[0] ^ x[1] ^ x[2]) & 1u;
}

int orc_match_predicate(u16 code, u16 mask, u32 threshold_a) {
    u32 r = (u32)mask * threshold_a - ((u32)code << 16) - 1u;
    return (int)(r >> 31);
}

/* ------------------------------------------------------------------------ */
/* CPU baseline: rotation_aware_pairwise_distance_rowmajor (ops.rs:238-331)   */
/* run per party on its shares, summed over parties, thresholded, OR over the */
/* rotations.  q_code[p]: [n_query*31][12800] preprocessed rotated query      */
/* shares; q_mask[p]: [n_query*31][6400]; db_code[p]: [n_db][12800];           */
/* db_mask[p]: [n_db][6400].  bitmap: [n_query][n_db] bytes (0/1).            */
/* Returns the number of (query, entry) matches.                              */
/* ------------------------------------------------------------------------ */
long orc_cpu_plain_match(const u16 *const *q_code, const u16 *const *q_mask, int n_query,
                         const u16 *const *db_code, const u16 *const *db_mask, long n_db,
                         u32 threshold_a, unsigned char *bitmap, int n_threads) {
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    long total = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
    for (long d = 0; d < n_db; d++) {
        for (int q = 0; q < n_query; q++) {
            u16 code_dot[ROTATIONS], mask_dot[ROTATIONS];
            for (int r = 0; r < ROTATIONS; r++) { code_dot[r] = 0; mask_dot[r] = 0; }
            for (int p = 0; p < 3; p++) {
                const u16 *dc = db_code[p] + d * IRIS_CODE_LENGTH;
                const u16 *dm = db_mask[p] + d * MASK_CODE_LENGTH;
                for (int r = 0; r < ROTATIONS; r++) {
                    const u16 *qc = q_code[p] + (long)(q * ROTATIONS + r) * IRIS_CODE_LENGTH;
                    const u16 *qm = q_mask[p] + (long)(q * ROTATIONS + r) * MASK_CODE_LENGTH;
                    u16 sc = 0, sm = 0;
                    for (int k = 0; k < IRIS_CODE_LENGTH; k++) sc = (u16)(sc + (u16)(qc[k] * dc[k]));
                    for (int k = 0; k < MASK_CODE_LENGTH; k++) sm = (u16)(sm + (u16)(qm[k] * dm[k]));
                    code_dot[r] = (u16)(code_dot[r] + sc);
                    mask_dot[r] = (u16)(mask_dot[r] + (u16)(2 * sm));
                }
            }
            int any = 0;
            for (int r = 0; r < ROTATIONS; r++) any |= orc_match_predicate(code_dot[r], mask_dot[r], threshold_a);
            if (bitmap) bitmap[(long)q * n_db + d] = (unsigned char)any;
            total += any;
        }
    }
    return total;
}
