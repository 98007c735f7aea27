/*
 * mg_oracle.c -- CPU oracle (test infrastructure only; see mg_oracle.h).
 *
 * Plain-C restatement of the reference's CPU DPF evaluation and fused scan.
 * Every function cites the reference file:line it follows.  Scalar ChaCha, as
 * in the reference; OpenMP over tiles stands in for the reference's rayon.
 */
#include "mg_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const uint32_t MGO_SIGMA[4] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};

static inline uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

/* chacha_prg.rs:93-109 */
static inline void quarter_round(uint32_t* s, int a, int b, int c, int d) {
  s[a] += s[b]; s[d] ^= s[a]; s[d] = rotl32(s[d], 16);
  s[c] += s[d]; s[b] ^= s[c]; s[b] = rotl32(s[b], 12);
  s[a] += s[b]; s[d] ^= s[a]; s[d] = rotl32(s[d], 8);
  s[c] += s[d]; s[b] ^= s[c]; s[b] = rotl32(s[b], 7);
}

/* chacha_prg.rs:112-144 (RFC 8439 state layout; feed-forward add). */
void mgo_chacha_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3],
                      int double_rounds, uint32_t out[16]) {
  uint32_t s[16], init[16];
  int i;
  for (i = 0; i < 4; i++) s[i] = MGO_SIGMA[i];
  for (i = 0; i < 8; i++) s[4 + i] = key[i];
  s[12] = counter;
  s[13] = nonce[0]; s[14] = nonce[1]; s[15] = nonce[2];
  memcpy(init, s, sizeof s);
  for (i = 0; i < double_rounds; i++) {
    quarter_round(s, 0, 4, 8, 12);
    quarter_round(s, 1, 5, 9, 13);
    quarter_round(s, 2, 6, 10, 14);
    quarter_round(s, 3, 7, 11, 15);
    quarter_round(s, 0, 5, 10, 15);
    quarter_round(s, 1, 6, 11, 12);
    quarter_round(s, 2, 7, 8, 13);
    quarter_round(s, 3, 4, 9, 14);
  }
  for (i = 0; i < 16; i++) out[i] = s[i] + init[i];
}

/* chacha_prg.rs:153-178: key = seed || seed, nonce 0, blocks with counter 0
 * and 1; L = b0[0..4], R = b0[4..8], tL = b1[0] & 1, tR = b1[1] & 1. */
void mgo_prg_expand(const uint32_t seed[4], uint32_t left[4], uint32_t right[4],
                    uint8_t* left_t, uint8_t* right_t) {
  uint32_t key[8], b0[16], b1[16];
  const uint32_t nonce[3] = {0, 0, 0};
  int i;
  for (i = 0; i < 4; i++) { key[i] = seed[i]; key[4 + i] = seed[i]; }
  mgo_chacha_block(key, 0, nonce, 4, b0);
  mgo_chacha_block(key, 1, nonce, 4, b1);
  for (i = 0; i < 4; i++) { left[i] = b0[i]; right[i] = b0[4 + i]; }
  *left_t = (uint8_t)(b1[0] & 1u);
  *right_t = (uint8_t)(b1[1] & 1u);
}

static inline uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static inline void put_le32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}

/* dpf.rs:277-316.  -1: "Byte array too short"; -2: "Invalid byte array
 * length"; -3: more levels than this oracle holds (MGO_MAX_LEVELS). */
int mgo_key_from_bytes(const uint8_t* b, size_t len, mgo_key* k) {
  size_t expected, off;
  uint32_t d, l;
  int i;
  if (len < 19 + 16) return -1;
  d = b[18];
  expected = 19 + (size_t)d * 18 + 16;
  if (len != expected) return -2;
  if (d > MGO_MAX_LEVELS) return -3;
  memset(k, 0, sizeof *k);
  for (i = 0; i < 4; i++) k->root_seed[i] = le32(b + 4 * i);
  k->root_t = b[16];
  k->party = b[17];
  k->domain_bits = d;
  off = 19;
  for (l = 0; l < d; l++) {
    for (i = 0; i < 4; i++) k->cw_seed[l][i] = le32(b + off + 4 * i);
    k->cw_tl[l] = b[off + 16];
    k->cw_tr[l] = b[off + 17];
    off += 18;
  }
  for (i = 0; i < 4; i++) k->final_cw[i] = le32(b + off + 4 * i);
  return 0;
}

/* dpf.rs:259-274 */
size_t mgo_key_to_bytes(const mgo_key* k, uint8_t* out) {
  size_t off = 0;
  uint32_t l;
  int i;
  for (i = 0; i < 4; i++) put_le32(out + 4 * i, k->root_seed[i]);
  out[16] = k->root_t;
  out[17] = k->party;
  out[18] = (uint8_t)k->domain_bits;
  off = 19;
  for (l = 0; l < k->domain_bits; l++) {
    for (i = 0; i < 4; i++) put_le32(out + off + 4 * i, k->cw_seed[l][i]);
    out[off + 16] = k->cw_tl[l];
    out[off + 17] = k->cw_tr[l];
    off += 18;
  }
  for (i = 0; i < 4; i++) put_le32(out + off + 4 * i, k->final_cw[i]);
  return off + 16;
}

/* One tree step shared by eval and the subtree prefix walk (dpf.rs:107-133):
 * expand, pick the child selected by bit, correct it when t == 1. */
static inline void step(const mgo_key* k, uint32_t level, int bit, uint32_t seed[4], uint8_t* t) {
  uint32_t L[4], R[4], *c;
  uint8_t lt, rt, ct;
  int i;
  mgo_prg_expand(seed, L, R, &lt, &rt);
  c = bit ? R : L;
  ct = bit ? rt : lt;
  if (*t == 1) {
    for (i = 0; i < 4; i++) c[i] ^= k->cw_seed[level][i];
    ct ^= bit ? k->cw_tr[level] : k->cw_tl[level];
  }
  for (i = 0; i < 4; i++) seed[i] = c[i];
  *t = ct;
}

/* dpf.rs:103-142 (MSB-first bit order). */
void mgo_eval(const mgo_key* k, uint64_t index, uint32_t out[4]) {
  uint32_t seed[4];
  uint8_t t = k->root_t;
  uint32_t level;
  int i;
  for (i = 0; i < 4; i++) seed[i] = k->root_seed[i];
  for (level = 0; level < k->domain_bits; level++) {
    int bit = (int)((index >> (k->domain_bits - 1 - level)) & 1u);
    step(k, level, bit, seed, &t);
  }
  for (i = 0; i < 4; i++) out[i] = seed[i] ^ (t == 1 ? k->final_cw[i] : 0u);
}

/* dpf.rs:210-246 (depth-first GGM expansion). */
static void expand_recursive(const mgo_key* k, uint32_t level, const uint32_t seed[4], uint8_t t,
                             uint32_t* out, uint64_t n) {
  uint32_t L[4], R[4];
  uint8_t lt, rt;
  int i;
  if (level == k->domain_bits) {
    for (i = 0; i < 4; i++) out[i] = seed[i] ^ (t == 1 ? k->final_cw[i] : 0u);
    return;
  }
  mgo_prg_expand(seed, L, R, &lt, &rt);
  if (t == 1) {
    for (i = 0; i < 4; i++) { L[i] ^= k->cw_seed[level][i]; R[i] ^= k->cw_seed[level][i]; }
    lt ^= k->cw_tl[level];
    rt ^= k->cw_tr[level];
  }
  expand_recursive(k, level + 1, L, lt, out, n / 2);
  expand_recursive(k, level + 1, R, rt, out + 4 * (n / 2), n / 2);
}

/* dpf.rs:164-208 */
int mgo_eval_subtree(const mgo_key* k, uint64_t start, uint64_t n, uint32_t* out) {
  uint32_t seed[4], depth = 0, root_level, level;
  uint8_t t = k->root_t;
  int i;
  if (n == 0 || (n & (n - 1)) != 0) return -1;
  if (start % n != 0) return -1;
  while ((1ull << depth) < n) depth++;
  root_level = k->domain_bits > depth ? k->domain_bits - depth : 0;
  for (i = 0; i < 4; i++) seed[i] = k->root_seed[i];
  for (level = 0; level < root_level; level++) {
    int bit = (int)((start >> (k->domain_bits - 1 - level)) & 1u);
    step(k, level, bit, seed, &t);
  }
  expand_recursive(k, root_level, seed, t, out, n);
  return 0;
}

/* dpf.rs:322-432 */
int mgo_keygen(uint32_t d, uint64_t target, const uint32_t seed0[4], const uint32_t seed1[4],
               mgo_key* k0, mgo_key* k1) {
  uint32_t s0[4], s1[4], level;
  uint8_t t0 = 0, t1 = 1;
  int i;
  if (d == 0 || d > 32) return -1;             /* ChaChaParams::new, dpf.rs:65-79 */
  if (target >= (1ull << d)) return -2;        /* PageIndexTooLarge, dpf.rs:326-329 */
  memset(k0, 0, sizeof *k0);
  memset(k1, 0, sizeof *k1);
  for (i = 0; i < 4; i++) { s0[i] = seed0[i]; s1[i] = seed1[i]; }
  for (level = 0; level < d; level++) {
    uint32_t L0[4], R0[4], L1[4], R1[4];
    uint8_t lt0, rt0, lt1, rt1;
    int bit = (int)((target >> (d - 1 - level)) & 1u);
    uint32_t *keep0, *keep1, *lose0, *lose1;
    uint8_t keep_t0, keep_t1, lose_t0, lose_t1, tcw_keep, tcw_lose;
    mgo_prg_expand(s0, L0, R0, &lt0, &rt0);
    mgo_prg_expand(s1, L1, R1, &lt1, &rt1);
    keep0 = bit ? R0 : L0; lose0 = bit ? L0 : R0;
    keep1 = bit ? R1 : L1; lose1 = bit ? L1 : R1;
    keep_t0 = bit ? rt0 : lt0; lose_t0 = bit ? lt0 : rt0;
    keep_t1 = bit ? rt1 : lt1; lose_t1 = bit ? lt1 : rt1;
    for (i = 0; i < 4; i++) k0->cw_seed[level][i] = lose0[i] ^ lose1[i];
    tcw_lose = (uint8_t)(lose_t0 ^ lose_t1 ^ t0 ^ t1 ^ 1);
    tcw_keep = (uint8_t)(keep_t0 ^ keep_t1 ^ t0 ^ t1);
    k0->cw_tl[level] = bit ? tcw_lose : tcw_keep;
    k0->cw_tr[level] = bit ? tcw_keep : tcw_lose;
    for (i = 0; i < 4; i++) {
      s0[i] = keep0[i] ^ (t0 == 1 ? k0->cw_seed[level][i] : 0u);
      s1[i] = keep1[i] ^ (t1 == 1 ? k0->cw_seed[level][i] : 0u);
    }
    {
      uint8_t nt0 = (uint8_t)(keep_t0 ^ (t0 == 1 ? tcw_keep : 0));
      uint8_t nt1 = (uint8_t)(keep_t1 ^ (t1 == 1 ? tcw_keep : 0));
      t0 = nt0; t1 = nt1;
    }
  }
  for (i = 0; i < 4; i++) k0->final_cw[i] = s0[i] ^ s1[i] ^ 0xFFFFFFFFu;
  for (i = 0; i < 4; i++) { k0->root_seed[i] = seed0[i]; k1->root_seed[i] = seed1[i]; }
  k0->root_t = 0; k1->root_t = 1;
  k0->party = 0; k1->party = 1;
  k0->domain_bits = d; k1->domain_bits = d;
  memcpy(k1->cw_seed, k0->cw_seed, sizeof k0->cw_seed);
  memcpy(k1->cw_tl, k0->cw_tl, sizeof k0->cw_tl);
  memcpy(k1->cw_tr, k0->cw_tr, sizeof k0->cw_tr);
  memcpy(k1->final_cw, k0->final_cw, sizeof k0->final_cw);
  return 0;
}

/* kernel.rs:1243-1256 generalised to R-byte rows: acc ^= row & mask, the
 * 16-byte mask repeated over each 16-byte lane. */
static inline void xor_row_masked(uint32_t* acc, const uint32_t* row, const uint32_t m[4],
                                  uint32_t words) {
  uint32_t w;
  for (w = 0; w < words; w += 4) {
    acc[w + 0] ^= row[w + 0] & m[0];
    acc[w + 1] ^= row[w + 1] & m[1];
    acc[w + 2] ^= row[w + 2] & m[2];
    acc[w + 3] ^= row[w + 3] & m[3];
  }
}

static uint64_t domain_size(uint32_t d) { return d >= 64 ? ~0ull : (1ull << d); }

#if defined(__x86_64__)
#include <immintrin.h>
#define MGO_AVX512 __attribute__((target("avx512f")))

/* The AND/XOR accumulate of rows [0, n) of one tile in 512-bit registers,
 * eight rows per step, in the shape of the reference server's AVX-512 row
 * scan (crates/morphogen-server/src/scan.rs:719-895, scan_chunk_avx512_inner:
 * eight rows loaded, ANDed with their broadcast masks, XOR-folded into the
 * accumulator).  There the mask is one DPF bit broadcast to 64 bytes; here it
 * is the row's 16-byte DPF output repeated over its 16-byte lanes, so the
 * result is xor_row_masked's exactly. */
MGO_AVX512 static void xor_rows_masked_avx512(uint32_t* acc, const uint8_t* rows, const uint32_t* masks,
                                              uint64_t n, uint32_t row_bytes) {
  uint64_t i = 0;
  if (row_bytes % 64 == 0) {
    const uint32_t vecs = row_bytes / 64;
    for (uint32_t v = 0; v < vecs; v++) {
      __m512i a = _mm512_loadu_si512(acc + 16 * v);
      const uint8_t* base = rows + 64 * (size_t)v;
#define MGO_ROWV(j)                                                                          \
  _mm512_and_si512(_mm512_loadu_si512(base + (i + (j)) * (uint64_t)row_bytes),              \
                   _mm512_broadcast_i32x4(_mm_loadu_si128((const __m128i*)(masks + 4 * (i + (j))))))
      for (i = 0; i + 8 <= n; i += 8) {
        const __m512i x01 = _mm512_xor_si512(MGO_ROWV(0), MGO_ROWV(1));
        const __m512i x23 = _mm512_xor_si512(MGO_ROWV(2), MGO_ROWV(3));
        const __m512i x45 = _mm512_xor_si512(MGO_ROWV(4), MGO_ROWV(5));
        const __m512i x67 = _mm512_xor_si512(MGO_ROWV(6), MGO_ROWV(7));
        a = _mm512_xor_si512(a, _mm512_xor_si512(_mm512_xor_si512(x01, x23), _mm512_xor_si512(x45, x67)));
      }
      for (; i < n; i++) a = _mm512_xor_si512(a, MGO_ROWV(0));
#undef MGO_ROWV
      _mm512_storeu_si512(acc + 16 * v, a);
    }
    return;
  }
  if (row_bytes == 32 || row_bytes == 16) {
    /* Several rows per vector: 32-B rows two at a time (lanes mask_i, mask_i,
     * mask_i+1, mask_i+1), 16-B rows four at a time (the masks of rows
     * i..i+3 are consecutive). */
    const uint64_t per = 64 / row_bytes;
    __m512i a = _mm512_setzero_si512();
#define MGO_MASKV(r)                                                                          \
  (row_bytes == 16 ? _mm512_loadu_si512(masks + 4 * (r))                                      \
                   : _mm512_shuffle_i64x2(_mm512_castsi256_si512(_mm256_loadu_si256((const __m256i*)(masks + 4 * (r)))), \
                                          _mm512_castsi256_si512(_mm256_loadu_si256((const __m256i*)(masks + 4 * (r)))), 0x50))
#define MGO_VEC(r) _mm512_and_si512(_mm512_loadu_si512(rows + (r) * (uint64_t)row_bytes), MGO_MASKV(r))
    for (i = 0; i + 8 <= n; i += 8) {
      __m512i x = _mm512_xor_si512(MGO_VEC(i), MGO_VEC(i + per));
      if (per == 2) x = _mm512_xor_si512(x, _mm512_xor_si512(MGO_VEC(i + 4), MGO_VEC(i + 6)));
      a = _mm512_xor_si512(a, x);
    }
#undef MGO_VEC
#undef MGO_MASKV
    {
      uint32_t lanes[16];
      _mm512_storeu_si512(lanes, a);
      for (uint32_t w = 0; w < 16; w++) acc[w % (row_bytes / 4)] ^= lanes[w];
    }
    for (; i < n; i++) xor_row_masked(acc, (const uint32_t*)(rows + i * (uint64_t)row_bytes), masks + 4 * i,
                                      row_bytes / 4);
    return;
  }
  for (i = 0; i < n; i++)
    xor_row_masked(acc, (const uint32_t*)(rows + i * (uint64_t)row_bytes), masks + 4 * i, row_bytes / 4);
}
#endif

/* kernel.rs:1276-1371.  avx512: accumulate with xor_rows_masked_avx512
 * instead of xor_row_masked (same result). */
static int scan_fused_impl(const mgo_key* keys, int nkeys, const uint8_t* rows, uint64_t nrows,
                           uint32_t row_bytes, uint64_t row_base, uint8_t* out, int nthreads, int avx512) {
  uint32_t min_d = 64, words = row_bytes / 4;
  uint64_t tile, first_tile, last_tile;
  int k;
  if (nkeys <= 0 || row_bytes == 0 || row_bytes % 16 != 0) return -1;
  for (k = 0; k < nkeys; k++) {
    if (keys[k].domain_bits < min_d) min_d = keys[k].domain_bits;
    if (row_base + nrows > domain_size(keys[k].domain_bits)) return -1; /* kernel.rs:1283-1285 */
  }
  memset(out, 0, (size_t)nkeys * row_bytes);
  if (nrows == 0) return 0;
  tile = 2048;
  if (domain_size(min_d) < tile) tile = domain_size(min_d);
  first_tile = row_base / tile;
  last_tile = (row_base + nrows - 1) / tile;
  if (nthreads <= 0) {
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
  }
#pragma omp parallel num_threads(nthreads)
  {
    uint32_t* acc = (uint32_t*)calloc((size_t)nkeys * words, 4);
    uint32_t* masks = (uint32_t*)malloc((size_t)tile * 16);
    int64_t ti;
#pragma omp for schedule(dynamic, 1)
    for (ti = (int64_t)first_tile; ti <= (int64_t)last_tile; ti++) {
      uint64_t start = (uint64_t)ti * tile, lo = start, hi = start + tile, i;
      if (lo < row_base) lo = row_base;
      if (hi > row_base + nrows) hi = row_base + nrows;
      for (int kk = 0; kk < nkeys; kk++) {
        mgo_eval_subtree(&keys[kk], start, tile, masks);
#if defined(__x86_64__)
        if (avx512) {
          xor_rows_masked_avx512(acc + (size_t)kk * words, rows + (lo - row_base) * (uint64_t)row_bytes,
                                 masks + 4 * (lo - start), hi - lo, row_bytes);
          continue;
        }
#endif
        for (i = lo; i < hi; i++)
          xor_row_masked(acc + (size_t)kk * words,
                         (const uint32_t*)(rows + (i - row_base) * (uint64_t)row_bytes),
                         masks + 4 * (i - start), words);
      }
    }
#pragma omp critical
    {
      uint32_t* o = (uint32_t*)out;
      size_t w;
      for (w = 0; w < (size_t)nkeys * words; w++) o[w] ^= acc[w];
    }
    free(acc);
    free(masks);
  }
  return 0;
}

int mgo_scan_fused(const mgo_key* keys, int nkeys, const uint8_t* rows, uint64_t nrows,
                   uint32_t row_bytes, uint64_t row_base, uint8_t* out, int nthreads) {
  return scan_fused_impl(keys, nkeys, rows, nrows, row_bytes, row_base, out, nthreads, 0);
}

int mgo_avx512_available(void) {
#if defined(__x86_64__)
  return __builtin_cpu_supports("avx512f") ? 1 : 0;
#else
  return 0;
#endif
}

int mgo_scan_fused_avx512(const mgo_key* keys, int nkeys, const uint8_t* rows, uint64_t nrows,
                          uint32_t row_bytes, uint64_t row_base, uint8_t* out, int nthreads) {
  if (!mgo_avx512_available()) return -2;
  return scan_fused_impl(keys, nkeys, rows, nrows, row_bytes, row_base, out, nthreads, 1);
}

/* kernel.rs:1374-1383 */
int mgo_scan_pointwise(const mgo_key* key, const uint8_t* rows, uint64_t nrows,
                       uint32_t row_bytes, uint8_t* out) {
  uint64_t i;
  uint32_t m[4];
  if (row_bytes == 0 || row_bytes % 16 != 0) return -1;
  memset(out, 0, row_bytes);
  for (i = 0; i < nrows; i++) {
    mgo_eval(key, i, m);
    xor_row_masked((uint32_t*)out, (const uint32_t*)(rows + i * (uint64_t)row_bytes), m,
                   row_bytes / 4);
  }
  return 0;
}

/* crates/morphogen-server/src/scan.rs:434-485, row mode (one row per leaf). */
int mgo_delta_apply(const mgo_key* keys, int nkeys, const uint64_t* row_idx, const uint8_t* diffs,
                    uint64_t nentries, uint32_t row_bytes, uint8_t* out) {
  uint64_t e;
  int k;
  if (row_bytes == 0 || row_bytes % 16 != 0) return -1;
  for (e = 0; e < nentries; e++) {
    for (k = 0; k < nkeys; k++) {
      uint32_t m[4];
      mgo_eval(&keys[k], row_idx[e], m);
      xor_row_masked((uint32_t*)(out + (size_t)k * row_bytes),
                     (const uint32_t*)(diffs + e * (uint64_t)row_bytes), m, row_bytes / 4);
    }
  }
  return 0;
}

/* SplitMix64 (Steele, Lea, Flood 2014): output i of the stream seeded with
 * seed, i.e. the finaliser applied to seed + (i + 1) * golden-gamma. */
uint64_t mgo_splitmix_word(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void mgo_fill_splitmix(uint8_t* buf, uint64_t off, uint64_t n, uint64_t seed) {
  int64_t o;
#pragma omp parallel for schedule(static)
  for (o = 0; o < (int64_t)n; o++) {
    uint64_t g = off + (uint64_t)o;
    buf[o] = (uint8_t)(mgo_splitmix_word(seed, g >> 3) >> (8 * (g & 7)));
  }
}

/* chunked_matrix.rs:83-93 */
void mgo_fill_lcg(uint8_t* buf, uint64_t n, uint64_t seed) {
  uint64_t state = seed, i;
  for (i = 0; i < n; i++) {
    state = state * 6364136223846793005ull + 1ull;
    buf[i] = (uint8_t)(state >> 56);
  }
}

/* kernel.rs:1390-1403 */
void mgo_fill_test_rows(uint8_t* buf, uint64_t nrows, uint32_t row_bytes) {
  uint64_t i;
  uint32_t j;
  for (i = 0; i < nrows; i++) {
    uint8_t* p = buf + i * (uint64_t)row_bytes;
    p[0] = (uint8_t)(i & 0xFF);
    if (row_bytes > 1) p[1] = (uint8_t)((i >> 8) & 0xFF);
    for (j = 2; j < row_bytes; j++) p[j] = (uint8_t)((i + j) & 0xFF);
  }
}
