// Host-side share preprocessing and the seeded synthetic query generator.
//
// preprocess (iris-mpc-common/src/galois_engine.rs:23-40): every block of four
// coefficients is a GR4 = Z_2^16[x]/(x^4 - x - 1) element in the monomial
// basis; the query share of party p is multiplied by the Lagrange coefficient
// at 0 of the party's evaluation point (1, x or 1+x) and converted to basis B
// = (S S^T)^-1 (symmetric-gr-shamir_sage.sage:136-269).  Both steps are
// linear, so each party gets one 4x4 matrix over Z_2^16.
//
// The synthetic generator defines the benchmark workload: iris bits from a
// position-addressable splitmix64 stream (code bits uniform, mask pairs kept
// with probability 0.9), planted near-duplicates (code bits flipped with
// p = 0.2, rotated by whole columns), degree-1 Shamir shares s + r*X at the
// three points.  The device-side DB generator (prep.cu) uses the same stream
// definitions, so a planted query is a near-duplicate of the device DB entry.
#include <stdint.h>
#include <string.h>

#include "../../include/irisb200.h"
#include "common.cuh"

namespace {

typedef uint16_t u16;
typedef uint32_t u32;
typedef uint64_t u64;

void gr_mul(const u16* a, const u16* b, u16* o) {
  const u32 d4 = (u32)a[1] * b[3] + (u32)a[2] * b[2] + (u32)a[3] * b[1];
  const u32 d5 = (u32)a[2] * b[3] + (u32)a[3] * b[2];
  const u32 d6 = (u32)a[3] * b[3];
  o[0] = (u16)((u32)a[0] * b[0] + d4);
  o[1] = (u16)((u32)a[0] * b[1] + (u32)a[1] * b[0] + d4 + d5);
  o[2] = (u16)((u32)a[0] * b[2] + (u32)a[1] * b[1] + (u32)a[2] * b[0] + d5 + d6);
  o[3] = (u16)((u32)a[0] * b[3] + (u32)a[1] * b[2] + (u32)a[2] * b[1] + (u32)a[3] * b[0] + d6);
}

// Units of GR(2^16, 4) form a group of order 15 * 2^60.
void gr_inv(const u16* a, u16* o) {
  u16 r[4] = {1, 0, 0, 0}, b[4] = {a[0], a[1], a[2], a[3]}, t[4];
  for (u64 e = 15ull * (1ull << 60) - 1; e; e >>= 1) {
    if (e & 1) { gr_mul(r, b, t); memcpy(r, t, 8); }
    gr_mul(b, b, t); memcpy(b, t, 8);
  }
  memcpy(o, r, 8);
}

const u16 kPoints[3][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {1, 1, 0, 0}};
const u16 kS[4][4] = {{1, 0, 0, 0}, {58082, 1, 0, 0}, {60579, 25194, 1, 0}, {17325, 51956, 57011, 1}};

struct Tables {
  u16 pre[3][4][4];  // per party: basis_B * (multiply by lambda_p)
  Tables() {
    // S^-1 (unit lower triangular), then B = (S^-1)^T S^-1
    u16 si[4][4] = {};
    for (int c = 0; c < 4; c++)
      for (int r = 0; r < 4; r++) {
        u32 v = r == c;
        for (int k = 0; k < r; k++) v -= (u32)kS[r][k] * si[k][c];
        si[r][c] = (u16)v;
      }
    u16 B[4][4];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        u32 v = 0;
        for (int k = 0; k < 4; k++) v += (u32)si[k][i] * si[k][j];
        B[i][j] = (u16)v;
      }
    for (int p = 0; p < 3; p++) {
      // lambda_p = prod_{q != p} (0 - x_q) / (x_p - x_q)
      u16 lam[4] = {1, 0, 0, 0};
      for (int q = 0; q < 3; q++) {
        if (q == p) continue;
        u16 neg[4], diff[4], inv[4], t[4];
        for (int k = 0; k < 4; k++) {
          neg[k] = (u16)(0 - kPoints[q][k]);
          diff[k] = (u16)(kPoints[p][k] - kPoints[q][k]);
        }
        gr_inv(diff, inv);
        gr_mul(lam, neg, t);
        gr_mul(t, inv, lam);
      }
      u16 L[4][4];
      for (int j = 0; j < 4; j++) {
        u16 e[4] = {0, 0, 0, 0}, col[4];
        e[j] = 1;
        gr_mul(lam, e, col);
        for (int i = 0; i < 4; i++) L[i][j] = col[i];
      }
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
          u32 v = 0;
          for (int k = 0; k < 4; k++) v += (u32)B[i][k] * L[k][j];
          pre[p][i][j] = (u16)v;
        }
    }
  }
};

const Tables& tables() {
  static const Tables t;
  return t;
}

u64 mix64(u64 z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
u64 rng64(u64 seed, u64 ctr) { return mix64(seed + (ctr + 1) * 0x9E3779B97F4A7C15ull); }

inline int bit(const u64* w, int i) { return (int)((w[i >> 6] >> (i & 63)) & 1); }

void iris_random(u64 seed, u64 idx, u64* code, u64* mask) {
  const u64 s = mix64(seed ^ (idx * 0xD1B54A32D192ED03ull));
  for (int w = 0; w < 200; w++) code[w] = rng64(s, (u64)w);
  memset(mask, 0, 200 * 8);
  for (int p = 0; p < 6400; p++) {
    const u64 r = rng64(s ^ 0x5bd1e995ull, (u64)(p >> 1));
    const u32 v = (p & 1) ? (u32)(r >> 32) : (u32)r;
    if (v < 3865470566u) mask[(2 * p) >> 6] |= 3ull << ((2 * p) & 63);
  }
}

void iris_flip(u64 seed, u64 idx, u32 p_num, u64* code) {
  const u64 s = mix64(seed ^ (idx * 0x9FB21C651E98DF25ull) ^ 0x1234567ull);
  for (int i = 0; i < 12800; i++) {
    const u64 r = rng64(s, (u64)(i >> 1));
    const u32 v = (i & 1) ? (u32)(r >> 32) : (u32)r;
    if (v < p_num) code[i >> 6] ^= 1ull << (i & 63);
  }
}

// by > 0 rotates every 800-bit row right by 4*by bits, by < 0 left.
void iris_rotate(u64* w, int by) {
  u64 t[200] = {};
  const int sh = ((by % 200) + 200) % 200 * 4;
  for (int i = 0; i < 12800; i++) {
    const int row = i / 800, col = i % 800;
    const int d = row * 800 + (col + sh) % 800;
    if (bit(w, i)) t[d >> 6] |= 1ull << (d & 63);
  }
  memcpy(w, t, sizeof t);
}

int remap_new_to_old(int i) {
  const int b = i / 6400, w = i % 6400 / 3200, r1 = i % 3200 / 800, c = i % 800 / 4, r2 = i % 4;
  return 800 * (r2 * 4 + r1) + c * 4 + w * 2 + b;
}

// Degree-1 Shamir shares of the iris code (mask = 0) or mask (mask = 1)
// coefficients, preprocessed for party p when `pre`; out[p] = [len] u16.
void encode(const u64* code, const u64* mask, int which, u64 seed, bool pre, u16* out[3], int len) {
  const Tables& T = tables();
  const u64 rseed = which == 0 ? seed : (seed ^ 0xabcdef12345ull);
  for (int i = 0; i < len; i += 4) {
    u16 v[4], s[4];
    for (int k = 0; k < 4; k++) {
      const int o = remap_new_to_old(i + k);
      const u16 m = (u16)bit(mask, o), c = (u16)bit(code, o);
      v[k] = which == 0 ? (u16)(m - 2 * (c & m)) : m;
    }
    for (int r = 0; r < 4; r++) {
      u32 a = 0;
      for (int k = 0; k < 4; k++) a += (u32)kS[r][k] * v[k];
      s[r] = (u16)a;
    }
    const u64 rr = rng64(rseed, (u64)(i / 4));
    const u16 rv[4] = {(u16)rr, (u16)(rr >> 16), (u16)(rr >> 32), (u16)(rr >> 48)};
    for (int p = 0; p < 3; p++) {
      u16 t[4], sh[4];
      gr_mul(rv, kPoints[p], t);
      for (int k = 0; k < 4; k++) sh[k] = (u16)(s[k] + t[k]);
      if (pre) {
        for (int r = 0; r < 4; r++) {
          u32 a = 0;
          for (int k = 0; k < 4; k++) a += (u32)T.pre[p][r][k] * sh[k];
          out[p][i + r] = (u16)a;
        }
      } else {
        memcpy(out[p] + i, sh, 8);
      }
    }
  }
}

}  // namespace

extern "C" {

int irs_preprocess_query_share(int party, uint16_t* coefs, size_t n) {
  if (party < 0 || party > 2 || !coefs || n % 4) return IRS_ERR_INVALID;
  const Tables& T = tables();
  for (size_t i = 0; i < n; i += 4) {
    u16 o[4];
    for (int r = 0; r < 4; r++) {
      u32 a = 0;
      for (int k = 0; k < 4; k++) a += (u32)T.pre[party][r][k] * coefs[i + k];
      o[r] = (u16)a;
    }
    memcpy(coefs + i, o, 8);
  }
  return IRS_OK;
}

int irs_mirror_query_share(uint16_t* coefs, size_t n, int flip_imaginary) {
  if (!coefs || (n != 12800 && n != 6400)) return IRS_ERR_INVALID;
  u16 tmp[12800], out[12800];
  memcpy(tmp, coefs, n * 2);
  // The imaginary half (b = 1) is negated: the reference subtracts it from a
  // sharing of zero; the all-zero sharing gives the same plaintext.
  if (flip_imaginary)
    for (size_t i = 6400; i < n; i++) tmp[i] = (u16)(0 - tmp[i]);
  for (size_t i = 0; i < n; i++) {
    const int b = (int)i / 6400, w = (int)i % 6400 / 3200, r1 = (int)i % 3200 / 800, c = (int)i % 800 / 4,
              r2 = (int)i % 4;
    const int fc = c < 100 ? 99 - c : 199 - (c - 100);
    out[b * 6400 + w * 3200 + r1 * 800 + fc * 4 + r2] = tmp[i];
  }
  memcpy(coefs, out, n * 2);
  return IRS_OK;
}

int irs_encode_iris(const uint64_t* code_bits, const uint64_t* mask_bits, uint64_t seed, int preprocess,
                    uint16_t* code_out, uint16_t* mask_out) {
  if (!code_bits || !mask_bits || !code_out || !mask_out) return IRS_ERR_INVALID;
  u16* co[3];
  u16* mo[3];
  for (int p = 0; p < 3; p++) {
    co[p] = code_out + (size_t)p * 12800;
    mo[p] = mask_out + (size_t)p * 6400;
  }
  encode(code_bits, mask_bits, 0, seed, preprocess != 0, co, 12800);
  encode(code_bits, mask_bits, 1, seed, preprocess != 0, mo, 6400);
  return IRS_OK;
}

int irs_synth_queries(uint64_t db_seed, uint64_t q_seed, size_t n_queries, const int64_t* planted_entry,
                      const int32_t* planted_rot, int preprocess, uint16_t* code_out, uint16_t* mask_out) {
  if (!code_out || !mask_out) return IRS_ERR_INVALID;
  for (size_t j = 0; j < n_queries; j++) {
    u64 code[200], mask[200];
    const int64_t e = planted_entry ? planted_entry[j] : -1;
    if (e >= 0) {
      const int r = planted_rot ? planted_rot[j] : 0;
      if (r < -15 || r > 15) return IRS_ERR_INVALID;
      iris_random(db_seed, (u64)e, code, mask);
      iris_flip(q_seed, j, 858993459u /* 0.2 * 2^32 */, code);
      iris_rotate(code, r);
      iris_rotate(mask, r);
    } else {
      iris_random(q_seed ^ 0x9999ull, j, code, mask);
    }
    const u64 s = rng64(q_seed ^ 0x7777ull, j);
    u16* co[3];
    u16* mo[3];
    for (int p = 0; p < 3; p++) {
      co[p] = code_out + ((size_t)p * n_queries + j) * 12800;
      mo[p] = mask_out + ((size_t)p * n_queries + j) * 6400;
    }
    encode(code, mask, 0, s, preprocess != 0, co, 12800);
    encode(code, mask, 1, s, preprocess != 0, mo, 6400);
  }
  return IRS_OK;
}

}  // extern "C"
