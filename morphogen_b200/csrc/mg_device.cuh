// mg_device.cuh -- device-side ChaCha8 GGM PRG and DPF key layout (sm_100a).
//
// The PRG is the reference's ChaCha8Prg::expand
// (crates/morphogen-gpu-dpf/src/chacha_prg.rs:153-178): ChaCha key = seed||seed,
// nonce 0, two blocks with counters 0 and 1 (RFC 8439 state layout, 4 double
// rounds, feed-forward add, chacha_prg.rs:112-144).  Children: L = block0[0..4],
// R = block0[4..8], tL = block1[0] & 1, tR = block1[1] & 1.
//
// B200 notes: the path is integer-ALU bound.  Adds and 3-input logic run at
// the full 128 lanes/clk/SM, funnel shifts and byte permutes at half rate, so
// the code is issue-bound at ~12 instructions per quarter round.  Both blocks
// are written out in one straight-line function so the compiler shares the
// three counter-independent column quarter rounds of round 1 and drops the
// parts of block 1 that do not reach bit 0 of words 0 and 1.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mg {

constexpr int kThreads = 256;    // CTA size of the scan kernel
constexpr int kMaxLevels = 32;   // MG_MAX_DOMAIN_BITS
constexpr int kMaxSegs = 8;      // (table, domain) segments per launch
constexpr uint32_t kSigma0 = 0x61707865u;  // "expand 32-byte k"
constexpr uint32_t kSigma1 = 0x3320646eu;
constexpr uint32_t kSigma2 = 0x79622d32u;
constexpr uint32_t kSigma3 = 0x6b206574u;

// Device key: the wire key (dpf.rs:259-274) re-laid out for 16-byte loads.
// t bytes keep the reference's byte semantics (a node applies its correction
// word iff t == 1, dpf.rs:122,192,228).
struct alignas(16) KeyDev {
  uint4 root_seed;
  uint4 final_cw;
  uint4 cw_seed[kMaxLevels];
  uint8_t cw_tl[kMaxLevels];
  uint8_t cw_tr[kMaxLevels];
  uint32_t root_t;
  uint32_t domain_bits;
  uint32_t pad[2];
};
static_assert(sizeof(KeyDev) == 624, "KeyDev layout");

// Per-key constants of the warp-independent kernel, derived on the host from
// the key.  That kernel carries a node's t as a mask (all ones iff t == 1);
// for a parent mask m and the PRG's child bit b, the child's mask is
//   (-b ^ (one & m)) & ~(big & m)
// where, per level and side, one = all ones iff the t correction byte is 1
// and big = all ones iff it is 2..255 (the child's t byte is then >= 2 and
// never corrects).  This equals the byte rule of dpf.rs:122,192,228 exactly.
// A last-level child's mask is only needed to pick its leaf's XOR term, so
// that step is a table lookup by the parent's bit p and the child's PRG bit b:
// leaf[4 * side + 2 * p + b] = (p ? cw_seed[d - 1] : 0) ^ (c ? final_cw : 0)
// with c the child's corrected bit (side 0 left, 1 right); the leaf mask is
// the PRG seed XOR that entry.
struct alignas(16) KeyAux {
  uint4 cw_tm[kMaxLevels];  // x: tl one, y: tl big, z: tr one, w: tr big (0 or ~0)
  uint4 leaf[8];
};
static_assert(sizeof(KeyAux) == 640, "KeyAux layout");

__device__ __forceinline__ uint32_t rotl16(uint32_t x) { return __byte_perm(x, 0, 0x1032); }
__device__ __forceinline__ uint32_t rotl8(uint32_t x) { return __byte_perm(x, 0, 0x2103); }
__device__ __forceinline__ uint32_t rotl12(uint32_t x) { return __funnelshift_l(x, x, 12); }
__device__ __forceinline__ uint32_t rotl7(uint32_t x) { return __funnelshift_l(x, x, 7); }

#define MG_QR(a, b, c, d)              \
  a += b; d ^= a; d = mg::rotl16(d);   \
  c += d; b ^= c; b = mg::rotl12(b);   \
  a += b; d ^= a; d = mg::rotl8(d);    \
  c += d; b ^= c; b = mg::rotl7(b);

#define MG_DOUBLE_ROUND(x)                                        \
  MG_QR(x##0, x##4, x##8, x##12) MG_QR(x##1, x##5, x##9, x##13)   \
  MG_QR(x##2, x##6, x##10, x##14) MG_QR(x##3, x##7, x##11, x##15) \
  MG_QR(x##0, x##5, x##10, x##15) MG_QR(x##1, x##6, x##11, x##12) \
  MG_QR(x##2, x##7, x##8, x##13) MG_QR(x##3, x##4, x##9, x##14)

// ChaCha8Prg::expand.  tl/tr are 0 or 1.
__device__ __forceinline__ void prg_expand(const uint4 s, uint4& L, uint4& R, uint32_t& tl,
                                           uint32_t& tr) {
  uint32_t x0 = kSigma0, x1 = kSigma1, x2 = kSigma2, x3 = kSigma3;
  uint32_t x4 = s.x, x5 = s.y, x6 = s.z, x7 = s.w;
  uint32_t x8 = s.x, x9 = s.y, x10 = s.z, x11 = s.w;
  uint32_t x12 = 0u, x13 = 0u, x14 = 0u, x15 = 0u;
  uint32_t y0 = kSigma0, y1 = kSigma1, y2 = kSigma2, y3 = kSigma3;
  uint32_t y4 = s.x, y5 = s.y, y6 = s.z, y7 = s.w;
  uint32_t y8 = s.x, y9 = s.y, y10 = s.z, y11 = s.w;
  uint32_t y12 = 1u, y13 = 0u, y14 = 0u, y15 = 0u;
  MG_DOUBLE_ROUND(x) MG_DOUBLE_ROUND(y)
  MG_DOUBLE_ROUND(x) MG_DOUBLE_ROUND(y)
  MG_DOUBLE_ROUND(x) MG_DOUBLE_ROUND(y)
  MG_DOUBLE_ROUND(x) MG_DOUBLE_ROUND(y)
  L = make_uint4(x0 + kSigma0, x1 + kSigma1, x2 + kSigma2, x3 + kSigma3);
  R = make_uint4(x4 + s.x, x5 + s.y, x6 + s.z, x7 + s.w);
  tl = (y0 + kSigma0) & 1u;
  tr = (y1 + kSigma1) & 1u;
  (void)x8; (void)x9; (void)x10; (void)x11; (void)x12; (void)x13; (void)x14; (void)x15;
  (void)y2; (void)y3; (void)y4; (void)y5; (void)y6; (void)y7; (void)y8; (void)y9;
  (void)y10; (void)y11; (void)y12; (void)y13; (void)y14; (void)y15;
}

// One GGM node expansion with the level's correction word applied to both
// children when t == 1 (dpf.rs:221-239).
__device__ __forceinline__ void expand_cw(const uint4 s, const uint32_t t, const KeyDev& k,
                                          const uint32_t level, uint4& L, uint32_t& tl, uint4& R,
                                          uint32_t& tr) {
  const uint4 cw = k.cw_seed[level];
  const uint32_t cwl = k.cw_tl[level];
  const uint32_t cwr = k.cw_tr[level];
  prg_expand(s, L, R, tl, tr);
  const uint32_t m = (t == 1u) ? 0xFFFFFFFFu : 0u;
  L.x ^= cw.x & m; L.y ^= cw.y & m; L.z ^= cw.z & m; L.w ^= cw.w & m;
  R.x ^= cw.x & m; R.y ^= cw.y & m; R.z ^= cw.z & m; R.w ^= cw.w & m;
  tl ^= cwl & m;
  tr ^= cwr & m;
}

// Leaf output: seed, XOR final_cw when t == 1 (dpf.rs:136-139, 211-218).
__device__ __forceinline__ uint4 leaf_mask(const uint4 s, const uint32_t t, const KeyDev& k) {
  const uint32_t m = (t == 1u) ? 0xFFFFFFFFu : 0u;
  const uint4 f = k.final_cw;
  return make_uint4(s.x ^ (f.x & m), s.y ^ (f.y & m), s.z ^ (f.z & m), s.w ^ (f.w & m));
}

// Same as expand_cw with the key read through the read-only data path (the
// key is uniform across a warp, so every load is a broadcast L1 hit).
__device__ __forceinline__ void expand_cw_g(const uint4 s, const uint32_t t, const KeyDev* __restrict__ k,
                                            const uint32_t level, uint4& L, uint32_t& tl, uint4& R,
                                            uint32_t& tr) {
  const uint4 cw = __ldg(&k->cw_seed[level]);
  const uint32_t cwl = __ldg(&k->cw_tl[level]);
  const uint32_t cwr = __ldg(&k->cw_tr[level]);
  prg_expand(s, L, R, tl, tr);
  const uint32_t m = (t == 1u) ? 0xFFFFFFFFu : 0u;
  L.x ^= cw.x & m; L.y ^= cw.y & m; L.z ^= cw.z & m; L.w ^= cw.w & m;
  R.x ^= cw.x & m; R.y ^= cw.y & m; R.z ^= cw.z & m; R.w ^= cw.w & m;
  tl ^= cwl & m;
  tr ^= cwr & m;
}

__device__ __forceinline__ uint4 leaf_mask_g(const uint4 s, const uint32_t t, const KeyDev* __restrict__ k) {
  const uint32_t m = (t == 1u) ? 0xFFFFFFFFu : 0u;
  const uint4 f = __ldg(&k->final_cw);
  return make_uint4(s.x ^ (f.x & m), s.y ^ (f.y & m), s.z ^ (f.z & m), s.w ^ (f.w & m));
}

// expand_cw_g with t carried as a mask (KeyAux): m is all ones iff the
// parent's t == 1; ml / mr are the children's masks.
__device__ __forceinline__ void expand_cw_m(const uint4 s, const uint32_t m, const KeyDev* __restrict__ k,
                                            const KeyAux* __restrict__ a, const uint32_t level, uint4& L,
                                            uint32_t& ml, uint4& R, uint32_t& mr) {
  const uint4 cw = __ldg(&k->cw_seed[level]);
  const uint4 tm = __ldg(&a->cw_tm[level]);
  uint32_t tl, tr;
  prg_expand(s, L, R, tl, tr);
  L.x ^= cw.x & m; L.y ^= cw.y & m; L.z ^= cw.z & m; L.w ^= cw.w & m;
  R.x ^= cw.x & m; R.y ^= cw.y & m; R.z ^= cw.z & m; R.w ^= cw.w & m;
  ml = ((0u - tl) ^ (tm.x & m)) & ~(tm.y & m);
  mr = ((0u - tr) ^ (tm.z & m)) & ~(tm.w & m);
}

// Last level (level d - 1): both children's leaf masks straight from the PRG
// seeds, with the level's correction word and the final correction word
// folded into one table entry per child.
__device__ __forceinline__ void leaf_pair_m(const uint4 s, const uint32_t m, const KeyAux* __restrict__ a,
                                            uint4& mask_l, uint4& mask_r) {
  uint32_t bl, br;
  prg_expand(s, mask_l, mask_r, bl, br);
  const uint32_t p2 = m & 2u;  // 2 * parent bit
  const uint4 cl = __ldg(&a->leaf[p2 | bl]);
  const uint4 cr = __ldg(&a->leaf[4u + (p2 | br)]);
  mask_l.x ^= cl.x; mask_l.y ^= cl.y; mask_l.z ^= cl.z; mask_l.w ^= cl.w;
  mask_r.x ^= cr.x; mask_r.y ^= cr.y; mask_r.z ^= cr.z; mask_r.w ^= cr.w;
}

__device__ __forceinline__ uint4 xor_and(uint4 acc, const uint4 d, const uint4 m) {
  acc.x ^= d.x & m.x; acc.y ^= d.y & m.y; acc.z ^= d.z & m.z; acc.w ^= d.w & m.w;
  return acc;
}
__device__ __forceinline__ uint4 xor4(uint4 a, const uint4 b) {
  a.x ^= b.x; a.y ^= b.y; a.z ^= b.z; a.w ^= b.w;
  return a;
}

// One (table, domain) segment of a pass.  Work items of the segment are
// (tile, group) pairs, tile-major so that CTAs running at the same time
// share row tiles through L2.
struct Segment {
  const uint4* table;   // rows * V uint4, row-major
  uint64_t first;       // logical index of table row 0 (row-range tables)
  uint64_t rows;        // rows scanned (first + rows <= 2^d)
  uint64_t item_begin;  // first global item index of the segment
  uint32_t tiles;       // 2^S-leaf tiles intersecting [first, first + rows)
  uint32_t groups;      // key groups
  uint32_t V;           // uint4 per row (row_bytes / 16), 1..256
  uint32_t d;           // domain bits of every key in the segment
  uint32_t S;           // tile depth: 2^S leaves per item (S <= d)
  uint32_t U;           // breadth-first levels below the tile root (2^U DFS roots)
  uint32_t M;           // depth-first levels per thread (S - U)
  uint32_t g;           // keys per group (<= kernel G)
  uint32_t key_base;    // KeyDev index of group 0, key 0
  uint32_t col_base;    // partial column of group 0, key 0, lane 0
};

struct ScanParams {
  Segment seg[kMaxSegs];
  const KeyDev* keys;
  uint4* partial;       // [gridDim.x][cols]
  uint64_t items;
  uint32_t nsegs;
  uint32_t cols;        // total share uint4s of the pass
  uint32_t slots;       // stack slots per key per thread allocated in smem
};

// ---- warp-independent scan ------------------------------------------------
//
// A frontier holds, for every key, the tree nodes at level F = d - M whose
// subtrees intersect the table's rows [first, first + rows).  A warp work
// item is 32 consecutive frontier nodes of one key group ("warp tile", 32 x
// 2^M rows); each lane walks its node's 2^M leaves depth-first.

// Widest CTA of the warp-independent kernel (16 warps, one CTA per SM: the
// 128 registers per thread of 512 threads fill the register file); CTAs of
// 8 or 4 warps are used when 16 warps' stacks do not fit.
constexpr int kWarpThreads = 512;
constexpr int kWarps = kWarpThreads / 32;

struct WarpSeg {
  const uint4* table;   // rows * V uint4
  uint64_t first;       // logical index of table row 0
  uint64_t rows;
  uint64_t item_begin;  // first global item of the segment
  uint64_t fr_base;     // frontier index of the segment's key 0 (key j at fr_base + j * nF)
  uint64_t nF;          // frontier nodes per key (level d - M nodes meeting the rows)
  uint32_t tiles;       // warp tiles per key group = ceil(nF / 32)
  uint32_t groups;      // key groups (items are group-major)
  uint32_t d;           // domain bits
  uint32_t M;           // depth-first levels per lane (>= 1)
  uint32_t g;           // keys per group
  uint32_t key_base;    // KeyDev index of the segment's key 0
  uint32_t col_base;    // first share column of the segment
  uint32_t pad;
};

struct WarpScanParams {
  WarpSeg seg[kMaxSegs];
  const KeyDev* keys;
  const KeyAux* aux;    // one per key, same index as keys
  const uint4* fr_seed;
  const uint8_t* fr_t;
  uint4* partial;       // [gridDim.x * warps per CTA][cols]
  uint4* out;           // the launch's cols shares (wide rows: zeroed before the launch, CTAs XOR into them)
  uint64_t items;
  uint32_t nsegs;
  uint32_t cols;
  uint32_t slots;       // depth-first stack slots per key per lane (>= max M)
};

// Levels one frontier-chain step expands (its last level's 2^10 nodes fit the
// CTA's shared memory).
constexpr uint32_t kFrontierLevels = 10;

// One breadth-first step of the frontier chain: every CTA expands `per`
// nodes of level L_in of key blockIdx.y by c <= kFrontierLevels levels and
// stores the nodes of level L_in + c that meet the table.  With `walk` set
// (per == 1) the CTA's root is not read from in_seed: the CTA derives it from
// the key's root by the L_in-level path walk of ChaCha::eval, so the first
// step of a chain needs no narrow one-CTA-per-key launch above it.
struct FrontierStep {
  const KeyDev* keys;     // the segment's keys
  const uint4* in_seed;   // level L_in (unused when L_in == 0): key j at j * n_in
  const uint8_t* in_t;
  uint4* out_seed;        // key j at out_base + j * out_stride
  uint8_t* out_t;
  uint64_t in_first;      // level index of input slot 0
  uint64_t out_first;     // level index of output slot 0
  uint64_t n_in;
  uint64_t n_out;
  uint64_t out_base;
  uint64_t out_stride;
  uint32_t L_in;
  uint32_t c;
  uint32_t per;           // input nodes per CTA (per << c <= 2^kFrontierLevels)
  uint32_t walk;          // 1: each CTA walks from the key's root to its level-L_in node
  uint4* zero_out;        // CTA (0, 0) zeroes these zero_n shares first (or null)
  uint64_t zero_n;
};

}  // namespace mg
