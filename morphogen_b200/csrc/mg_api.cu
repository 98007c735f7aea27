// mg_api.cu -- C ABI (include/morphogen_gpu.h) over the sm_100a kernels.
//
// Host-side counterpart of the reference's GpuScanner / GpuPageMatrix /
// BatchWorkspace (crates/morphogen-gpu-dpf/src/{kernel,storage}.rs): key
// parsing from the unchanged wire format, pass planning (segments of
// (table, domain), key groups, tile depth), persistent device workspaces,
// CUDA-graph replay, and host deadlines instead of unbounded waits.
#include <algorithm>
#include <cmath>
#include <array>
#include <map>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mg_internal.h"
#include "morphogen_gpu.h"

using mg::KeyDev;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define MG_CUDA(expr)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess) return fail(MG_ECUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

// ---- host ChaCha8 PRG (keygen only; chacha_prg.rs:93-178) -------------------
inline uint32_t hrotl(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

void host_block(const uint32_t key[8], uint32_t ctr, uint32_t out[16]) {
  uint32_t s[16] = {mg::kSigma0, mg::kSigma1, mg::kSigma2, mg::kSigma3, key[0], key[1], key[2],
                    key[3],      key[4],      key[5],      key[6],      key[7], ctr,    0,
                    0,           0};
  uint32_t x[16];
  std::memcpy(x, s, sizeof s);
  auto qr = [&](int a, int b, int c, int d) {
    x[a] += x[b]; x[d] ^= x[a]; x[d] = hrotl(x[d], 16);
    x[c] += x[d]; x[b] ^= x[c]; x[b] = hrotl(x[b], 12);
    x[a] += x[b]; x[d] ^= x[a]; x[d] = hrotl(x[d], 8);
    x[c] += x[d]; x[b] ^= x[c]; x[b] = hrotl(x[b], 7);
  };
  for (int r = 0; r < 4; ++r) {
    qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
    qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
  }
  for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

void host_expand(const uint32_t seed[4], uint32_t L[4], uint32_t R[4], uint8_t& lt, uint8_t& rt) {
  const uint32_t key[8] = {seed[0], seed[1], seed[2], seed[3], seed[0], seed[1], seed[2], seed[3]};
  uint32_t b0[16], b1[16];
  host_block(key, 0, b0);
  host_block(key, 1, b1);
  for (int i = 0; i < 4; ++i) { L[i] = b0[i]; R[i] = b0[4 + i]; }
  lt = (uint8_t)(b1[0] & 1u);
  rt = (uint8_t)(b1[1] & 1u);
}

inline uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
inline void put_le32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}

// ChaChaKey::from_bytes (dpf.rs:277-316) into the device layout.
int parse_key(const uint8_t* b, size_t len, KeyDev* k) {
  if (!b) return fail(MG_EINVAL, "null key pointer");
  if (len < 19 + 16) return fail(MG_EKEY, "invalid key format: byte array too short (%zu)", len);
  const uint32_t d = b[18];
  const size_t expected = 19 + (size_t)d * 18 + 16;
  if (len != expected)
    return fail(MG_EKEY, "invalid key format: invalid byte array length %zu (expected %zu)", len,
                expected);
  if (d > MG_MAX_DOMAIN_BITS)
    return fail(MG_ERANGE, "key domain_bits %u exceeds the supported maximum %d", d,
                MG_MAX_DOMAIN_BITS);
  std::memset(k, 0, sizeof *k);
  k->root_seed = make_uint4(le32(b), le32(b + 4), le32(b + 8), le32(b + 12));
  k->root_t = b[16];
  k->domain_bits = d;
  size_t off = 19;
  for (uint32_t l = 0; l < d; ++l) {
    k->cw_seed[l] = make_uint4(le32(b + off), le32(b + off + 4), le32(b + off + 8), le32(b + off + 12));
    k->cw_tl[l] = b[off + 16];
    k->cw_tr[l] = b[off + 17];
    off += 18;
  }
  k->final_cw = make_uint4(le32(b + off), le32(b + off + 4), le32(b + off + 8), le32(b + off + 12));
  return MG_OK;
}

// The warp kernel's per-key constants (KeyAux): t correction bytes as
// masks, and the eight last-level XOR terms of a leaf mask.
void make_aux(const KeyDev& k, mg::KeyAux* a) {
  std::memset(a, 0, sizeof *a);
  const auto one = [](uint8_t t) { return t == 1 ? 0xFFFFFFFFu : 0u; };
  const auto big = [](uint8_t t) { return t >= 2 ? 0xFFFFFFFFu : 0u; };
  for (uint32_t l = 0; l < k.domain_bits; ++l)
    a->cw_tm[l] = make_uint4(one(k.cw_tl[l]), big(k.cw_tl[l]), one(k.cw_tr[l]), big(k.cw_tr[l]));
  const uint4 f = k.final_cw;
  const uint32_t last = k.domain_bits ? k.domain_bits - 1 : 0;
  const uint4 c = k.domain_bits ? k.cw_seed[last] : make_uint4(0u, 0u, 0u, 0u);
  for (uint32_t side = 0; side < 2; ++side) {
    const uint8_t t = k.domain_bits ? (side ? k.cw_tr[last] : k.cw_tl[last]) : 0;
    for (uint32_t p = 0; p < 2; ++p)
      for (uint32_t b = 0; b < 2; ++b) {
        const uint32_t child = p ? (t == 1 ? b ^ 1u : (t >= 2 ? 0u : b)) : b;
        const uint4 cp = p ? c : make_uint4(0u, 0u, 0u, 0u);
        const uint4 fc = child ? f : make_uint4(0u, 0u, 0u, 0u);
        a->leaf[4 * side + 2 * p + b] = make_uint4(cp.x ^ fc.x, cp.y ^ fc.y, cp.z ^ fc.z, cp.w ^ fc.w);
      }
  }
}

int wait_event(cudaEvent_t ev, uint32_t timeout_ms) {
  if (timeout_ms == 0) {
    MG_CUDA(cudaEventSynchronize(ev));
    return MG_OK;
  }
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
  for (;;) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return MG_OK;
    if (e != cudaErrorNotReady) return fail(MG_ECUDA, "cudaEventQuery: %s", cudaGetErrorString(e));
    if (std::chrono::steady_clock::now() >= deadline)
      return fail(MG_ETIMEDOUT, "pass not complete after %u ms", timeout_ms);
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

uint64_t domain_size(uint32_t d) { return 1ull << d; }

}  // namespace

namespace mg {
void set_last_error(const char* msg) { g_err = msg ? msg : ""; }
}  // namespace mg

struct mg_context {
  int device = 0;
  int sms = 0;
  size_t smem_optin = 0;
  bool mapped_host = false;   // pinned host buffers are addressable from kernels (unified addressing)
  std::mutex mu;              // serialises the one-call path (mg_scan)
  mg_batch* internal = nullptr;
  std::mutex tune_mu;  // tuned launch shapes per workload signature
  std::map<std::string, std::array<uint32_t, 3>> tuned;  // {kind, subtree_bits, keys_per_item}
};

struct mg_table {
  mg_context* ctx = nullptr;
  int device = 0;
  int sms = 0;
  void* d = nullptr;
  uint64_t first = 0;  // logical index of row 0 (row-range tables)
  uint64_t rows = 0;
  uint32_t row_bytes = 0;
  // Pending epoch delta (DeltaBuffer, crates/morphogen-core/src/delta.rs):
  // entries are folded into every pass over the table until merged.
  uint64_t* d_delta_idx = nullptr;
  void* d_delta_diff = nullptr;
  uint32_t* d_delta_count = nullptr;  // entry count read by the delta kernel
  uint32_t delta_cap = 0;
  uint32_t delta_count = 0;
  uint64_t epoch = 0;
};

struct mg_batch {
  struct Launch {
    int kind = MG_KERNEL_CTA;
    mg::ScanParams p;      // CTA kernel parameters
    mg::WarpScanParams w;  // warp kernel parameters
    std::vector<mg::FrontierStep> steps;  // warp kernel: frontier chain, in order
    std::vector<uint32_t> step_keys;      // keys (grid.y) of each chain step
    uint32_t grid = 0;     // CTAs
    uint32_t nparts = 0;   // partial rows (CTAs or warps)
    uint32_t cols = 0;
    size_t smem = 0;
    int G = 1;
    uint32_t VT = 0;
    uint32_t NW = 0;       // warp kernel: warps per CTA
    uint32_t col0 = 0;     // first share column of this launch
  };
  mg_context* ctx = nullptr;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_k0 = nullptr, ev_km = nullptr, ev_k1 = nullptr, ev_done = nullptr, ev_h0 = nullptr, ev_h1 = nullptr;
  KeyDev* d_keys = nullptr;
  KeyDev* h_keys = nullptr;
  size_t cap_keys = 0;
  uint4* d_partial = nullptr;
  size_t cap_partial = 0;
  uint4* d_out = nullptr;
  uint8_t* h_out = nullptr;
  size_t cap_out = 0;
  uint4* d_fr_seed = nullptr;  // frontier nodes of every warp-kernel key
  uint8_t* d_fr_t = nullptr;
  size_t cap_fr = 0;
  uint4* d_tmp_seed[2] = {nullptr, nullptr};  // frontier chain intermediates
  uint8_t* d_tmp_t[2] = {nullptr, nullptr};
  size_t cap_tmp = 0;
  std::vector<Launch> launches;
  struct DeltaLaunch {
    const mg_table* table;
    uint32_t job0, njobs;  // range in d_jobs
  };
  std::vector<DeltaLaunch> deltas;
  uint2* d_jobs = nullptr;
  uint2* h_jobs = nullptr;
  size_t cap_jobs = 0;
  uint32_t total_cols = 0;
  std::vector<uint32_t> key_col;    // first share column of input key i
  std::vector<uint32_t> key_bytes;  // share bytes of input key i
  size_t total_share_bytes = 0;
  uint32_t shape_S = 0, shape_G = 0;  // pinned by mg_batch_set_shape (0 = planner)
  int kind_pref = MG_KERNEL_AUTO;     // pinned by mg_batch_set_kernel
  uint32_t eff_S = 0, eff_G = 0;      // shape used by the current plan
  int eff_kind = MG_KERNEL_AUTO;
  std::vector<KeyDev> in_keys;        // parsed keys of the current pass, input order
  std::vector<const mg_table*> in_tables;
  std::string signature;              // workload signature for the tuned-shape cache
  mg_plan_info info{};
  bool planned = false;
  bool launched = false;
  cudaGraphExec_t gexec = nullptr;
  std::vector<uint8_t> graph_sig;
  // The one-call path (mg_scan): key upload, pass and share download in one
  // graph, replayed while the plan is reused.
  cudaGraphExec_t gexec_io = nullptr;
  std::vector<uint8_t> graph_io_sig;
  bool defer_key_copy = false;  // set_keys leaves a reused plan's key upload to the caller
  size_t key_copy_bytes = 0;
  // What the current plan was made for: a later set_keys with the same
  // tables, key depths, shape and delta buffers only restages the keys.
  std::vector<uint32_t> plan_slot;     // input key i -> key slot
  std::vector<uint32_t> plan_depth;    // input key i -> domain bits
  std::vector<const mg_table*> plan_tables;
  std::vector<std::pair<const void*, uint32_t>> plan_deltas;  // per input key: delta buffer, capacity
  std::vector<std::array<uint64_t, 4>> plan_shapes;  // per input key: table memory, rows, row bytes, first row
  int plan_kind = -1;
  uint32_t plan_S = 0, plan_G = 0;
  bool plan_reused = false;           // the last set_keys kept the plan
};

namespace {

// What a plan depends on in a table besides its identity (a destroyed table's
// address can come back for a different table).
std::array<uint64_t, 4> table_shape(const mg_table* t) {
  return {(uint64_t)(uintptr_t)t->d, t->rows, t->row_bytes, t->first};
}


template <class T>
int set_device(const T* obj) {
  MG_CUDA(cudaSetDevice(obj->device));
  return MG_OK;
}

// The kernels' shared-memory limits are process-wide per device; the
// launchers keep one high-water mark for every caller (scan_prepare /
// warp_prepare only raise it), so nothing is cached per context.
int prepare_g(mg_context* ctx, int G, size_t smem) {
  (void)ctx;
  MG_CUDA(mg::scan_prepare(G, smem));
  return MG_OK;
}

int prepare_warp(mg_context* ctx, int G, uint32_t VT, size_t smem) {
  (void)ctx;
  MG_CUDA(mg::warp_prepare(G, VT, smem));
  return MG_OK;
}

template <class T>
int grow_dev(T*& p, size_t& cap, size_t need, const char* what) {
  if (need <= cap) return MG_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  if (cudaMalloc(&p, need * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return fail(MG_ENOMEM, "cannot allocate %zu bytes of %s", need * sizeof(T), what);
  }
  cap = need;
  return MG_OK;
}

int grow(mg_batch* b, size_t nkeys, size_t partial_u4, size_t out_u4, size_t fr_nodes, size_t tmp_nodes) {
  if (nkeys > b->cap_keys) {
    if (b->d_keys) cudaFree(b->d_keys);
    if (b->h_keys) cudaFreeHost(b->h_keys);
    b->d_keys = nullptr;
    b->h_keys = nullptr;
    b->cap_keys = 0;
    // Keys, then their warp-kernel constants (KeyAux) right after the pass's keys.
    const size_t bytes = nkeys * (sizeof(KeyDev) + sizeof(mg::KeyAux));
    if (cudaMalloc(&b->d_keys, bytes) != cudaSuccess || cudaMallocHost(&b->h_keys, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(MG_ENOMEM, "cannot allocate key buffers for %zu keys", nkeys);
    }
    b->cap_keys = nkeys;
  }
  if (int rc = grow_dev(b->d_partial, b->cap_partial, partial_u4, "partial rows")) return rc;
  if (out_u4 > b->cap_out) {
    if (b->d_out) cudaFree(b->d_out);
    if (b->h_out) cudaFreeHost(b->h_out);
    b->d_out = nullptr;
    b->h_out = nullptr;
    b->cap_out = 0;
    if (cudaMalloc(&b->d_out, out_u4 * 16) != cudaSuccess ||
        cudaMallocHost(&b->h_out, out_u4 * 16) != cudaSuccess) {
      cudaGetLastError();
      return fail(MG_ENOMEM, "cannot allocate share buffers (%zu bytes)", out_u4 * 16);
    }
    b->cap_out = out_u4;
  }
  if (fr_nodes > b->cap_fr) {
    size_t c1 = b->cap_fr, c2 = b->cap_fr;
    if (int rc = grow_dev(b->d_fr_seed, c1, fr_nodes, "frontier seeds")) return rc;
    if (int rc = grow_dev(b->d_fr_t, c2, fr_nodes, "frontier control bits")) return rc;
    b->cap_fr = fr_nodes;
  }
  if (tmp_nodes > b->cap_tmp) {
    for (int i = 0; i < 2; ++i) {
      size_t c1 = b->cap_tmp, c2 = b->cap_tmp;
      if (int rc = grow_dev(b->d_tmp_seed[i], c1, tmp_nodes, "frontier chain")) return rc;
      if (int rc = grow_dev(b->d_tmp_t[i], c2, tmp_nodes, "frontier chain")) return rc;
    }
    b->cap_tmp = tmp_nodes;
  }
  return MG_OK;
}

struct SegPlan {
  const mg_table* table;
  uint32_t d;
  std::vector<uint32_t> keys;  // input key indices, group-major
  uint32_t g;
  bool warp;
};

// Keys evaluated together on one work item.  Rows of up to 128 B leave the
// pass bound by ChaCha8 issue slots, so one key per item maximises the
// number of independent items (re-reads of a row by sibling items hit L2);
// wider rows share each row load across up to 4 keys.
int choose_g(uint32_t V, size_t nkeys, uint32_t pinned, bool warp) {
  int g = pinned ? (int)pinned : (V <= 8 ? 1 : 4);
  if (warp && g > 4) g = 4;
  if ((size_t)g > nkeys) g = (int)nkeys;
  if (g < 1) g = 1;
  if (warp) {
    while (!mg::warp_g_supported(g)) --g;
  } else {
    while (!mg::scan_g_supported(g)) --g;
  }
  return g;
}

void shape_for(uint32_t d, uint32_t S_target, uint32_t& S, uint32_t& U, uint32_t& M) {
  S = std::min(S_target, d);
  U = S >= 1 ? std::min<uint32_t>(8u, S - 1) : 0u;
  M = S - U;
}


// Tree nodes 2^s leaves wide that meet the table's rows [first, first + rows):
// their first level index and their count.
uint64_t level_first(const mg_table* t, uint32_t s) { return s >= 64 ? 0 : t->first >> s; }
uint64_t level_count(const mg_table* t, uint32_t s) {
  if (t->rows == 0) return 0;
  if (s >= 64) return 1;
  return ((t->first + t->rows - 1) >> s) - (t->first >> s) + 1;
}

}  // namespace

extern "C" {

const char* mg_last_error(void) { return g_err.c_str(); }

int mg_context_create(int device, mg_context** out) {
  if (!out) return fail(MG_EINVAL, "null output pointer");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(MG_ENODEV, "no CUDA device available");
  }
  if (device < 0 || device >= n) return fail(MG_EINVAL, "device %d out of range (%d devices)", device, n);
  MG_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  MG_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(MG_ENODEV, "device %d is sm_%d%d; this library is built for sm_100a only", device,
                prop.major, prop.minor);
  MG_CUDA(cudaFree(nullptr));
  mg_context* c = new mg_context();
  c->device = device;
  c->sms = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  c->mapped_host = prop.unifiedAddressing != 0 && prop.canMapHostMemory != 0;
  *out = c;
  return MG_OK;
}

int mg_context_destroy(mg_context* ctx) {
  if (!ctx) return MG_OK;
  if (ctx->internal) mg_batch_destroy(ctx->internal);
  delete ctx;
  return MG_OK;
}

int mg_device_info(mg_context* ctx, int* sm_count, uint64_t* free_bytes, uint64_t* total_bytes) {
  if (!ctx) return fail(MG_EINVAL, "null context");
  if (int rc = set_device(ctx)) return rc;
  size_t f = 0, t = 0;
  MG_CUDA(cudaMemGetInfo(&f, &t));
  if (sm_count) *sm_count = ctx->sms;
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return MG_OK;
}

// ---- tables -----------------------------------------------------------------

int mg_table_create(mg_context* ctx, uint64_t rows, uint32_t row_bytes, mg_table** out) {
  return mg_table_create_range(ctx, 0, rows, row_bytes, out);
}

int mg_table_create_range(mg_context* ctx, uint64_t first_row, uint64_t rows, uint32_t row_bytes, mg_table** out) {
  if (!ctx || !out) return fail(MG_EINVAL, "null argument");
  *out = nullptr;
  if (row_bytes == 0 || row_bytes % 16 != 0 || row_bytes > MG_MAX_ROW_BYTES)
    return fail(MG_EINVAL, "row_bytes %u must be a multiple of 16 in [16, %d]", row_bytes,
                MG_MAX_ROW_BYTES);
  if (first_row > (1ull << MG_MAX_DOMAIN_BITS) || rows > (1ull << MG_MAX_DOMAIN_BITS) - first_row)
    return fail(MG_ERANGE, "rows [%llu, %llu) exceed the 2^%d-row domain limit", (unsigned long long)first_row,
                (unsigned long long)(first_row + rows), MG_MAX_DOMAIN_BITS);
  if (int rc = set_device(ctx)) return rc;
  mg_table* t = new mg_table();
  t->ctx = ctx;
  t->device = ctx->device;
  t->sms = ctx->sms;
  t->first = first_row;
  t->rows = rows;
  t->row_bytes = row_bytes;
  const size_t bytes = (size_t)rows * row_bytes;
  if (bytes) {
    if (cudaMalloc(&t->d, bytes) != cudaSuccess) {
      cudaGetLastError();
      delete t;
      return fail(MG_ENOMEM, "cannot allocate a %zu-byte table", bytes);
    }
    if (cudaMemset(t->d, 0, bytes) != cudaSuccess) {
      cudaFree(t->d);
      delete t;
      return fail(MG_ECUDA, "cudaMemset of the table failed");
    }
  }
  *out = t;
  return MG_OK;
}

int mg_table_destroy(mg_table* t) {
  if (!t) return MG_OK;
  set_device(t);
  if (t->d_delta_idx) cudaFree(t->d_delta_idx);
  if (t->d_delta_diff) cudaFree(t->d_delta_diff);
  if (t->d_delta_count) cudaFree(t->d_delta_count);
  if (t->d) cudaFree(t->d);
  delete t;
  return MG_OK;
}

int mg_table_write_rows(mg_table* t, uint64_t first, const void* host, uint64_t n) {
  if (!t || (!host && n)) return fail(MG_EINVAL, "null argument");
  if (first > t->rows || n > t->rows - first)
    return fail(MG_ERANGE, "rows [%llu, %llu) outside the %llu-row table", (unsigned long long)first,
                (unsigned long long)(first + n), (unsigned long long)t->rows);
  if (int rc = set_device(t)) return rc;
  if (n) MG_CUDA(cudaMemcpy((uint8_t*)t->d + first * t->row_bytes, host, n * t->row_bytes,
                            cudaMemcpyHostToDevice));
  return MG_OK;
}

int mg_table_read_rows(const mg_table* t, uint64_t first, void* host, uint64_t n) {
  if (!t || (!host && n)) return fail(MG_EINVAL, "null argument");
  if (first > t->rows || n > t->rows - first)
    return fail(MG_ERANGE, "rows [%llu, %llu) outside the %llu-row table", (unsigned long long)first,
                (unsigned long long)(first + n), (unsigned long long)t->rows);
  if (int rc = set_device(t)) return rc;
  if (n) MG_CUDA(cudaMemcpy(host, (const uint8_t*)t->d + first * t->row_bytes, n * t->row_bytes,
                            cudaMemcpyDeviceToHost));
  return MG_OK;
}

int mg_table_fill_splitmix(mg_table* t, uint64_t seed) {
  if (!t) return fail(MG_EINVAL, "null table");
  if (int rc = set_device(t)) return rc;
  // Logical byte offset: a row-range table holds the logical table's rows.
  MG_CUDA(mg::launch_fill_splitmix(t->d, t->rows * t->row_bytes / 8, seed, t->first * t->row_bytes / 8, t->sms,
                                   nullptr));
  MG_CUDA(cudaDeviceSynchronize());
  return MG_OK;
}

int mg_table_xor_rows(mg_table* t, const uint64_t* idx, const void* diffs, uint64_t n) {
  if (!t || (n && (!idx || !diffs))) return fail(MG_EINVAL, "null argument");
  if (n == 0) return MG_OK;
  for (uint64_t i = 0; i < n; ++i)
    if (idx[i] >= t->rows)
      return fail(MG_ERANGE, "row %llu outside the %llu-row table", (unsigned long long)idx[i],
                  (unsigned long long)t->rows);
  if (int rc = set_device(t)) return rc;
  void* d_idx = nullptr;
  void* d_diff = nullptr;
  if (cudaMalloc(&d_idx, n * 8) != cudaSuccess || cudaMalloc(&d_diff, n * t->row_bytes) != cudaSuccess) {
    cudaGetLastError();
    if (d_idx) cudaFree(d_idx);
    return fail(MG_ENOMEM, "cannot stage %llu delta rows", (unsigned long long)n);
  }
  int rc = MG_OK;
  cudaError_t e = cudaMemcpy(d_idx, idx, n * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_diff, diffs, n * t->row_bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = mg::launch_xor_rows(t->d, t->row_bytes / 16, (const uint64_t*)d_idx, d_diff, n,
                                                t->sms, nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) rc = fail(MG_ECUDA, "xor_rows: %s", cudaGetErrorString(e));
  cudaFree(d_idx);
  cudaFree(d_diff);
  return rc;
}

uint64_t mg_table_rows(const mg_table* t) { return t ? t->rows : 0; }
uint64_t mg_table_first_row(const mg_table* t) { return t ? t->first : 0; }
uint32_t mg_table_row_bytes(const mg_table* t) { return t ? t->row_bytes : 0; }
const void* mg_table_device_ptr(const mg_table* t) { return t ? t->d : nullptr; }

int mg_table_delta_reserve(mg_table* t, uint32_t capacity) {
  if (!t) return fail(MG_EINVAL, "null table");
  if (capacity < t->delta_count)
    return fail(MG_EINVAL, "capacity %u below the %u pending entries", capacity, t->delta_count);
  if (capacity == t->delta_cap) return MG_OK;
  if (int rc = set_device(t)) return rc;
  uint64_t* idx = nullptr;
  void* diff = nullptr;
  uint32_t* cnt = t->d_delta_count;
  if (capacity) {
    if (cudaMalloc(&idx, (size_t)capacity * 8) != cudaSuccess ||
        cudaMalloc(&diff, (size_t)capacity * t->row_bytes) != cudaSuccess ||
        (!cnt && cudaMalloc(&cnt, 4) != cudaSuccess)) {
      cudaGetLastError();
      if (idx) cudaFree(idx);
      if (diff) cudaFree(diff);
      return fail(MG_ENOMEM, "cannot allocate a %u-entry delta buffer", capacity);
    }
    cudaError_t e = cudaSuccess;
    if (t->delta_count) {
      e = cudaMemcpy(idx, t->d_delta_idx, (size_t)t->delta_count * 8, cudaMemcpyDeviceToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(diff, t->d_delta_diff, (size_t)t->delta_count * t->row_bytes, cudaMemcpyDeviceToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(cnt, &t->delta_count, 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(idx);
      cudaFree(diff);
      return fail(MG_ECUDA, "delta reserve: %s", cudaGetErrorString(e));
    }
  }
  if (t->d_delta_idx) cudaFree(t->d_delta_idx);
  if (t->d_delta_diff) cudaFree(t->d_delta_diff);
  t->d_delta_idx = idx;
  t->d_delta_diff = diff;
  t->d_delta_count = cnt;
  t->delta_cap = capacity;
  return MG_OK;
}

int mg_table_delta_push(mg_table* t, const uint64_t* row_idx, const void* diffs, uint32_t n) {
  if (!t || (n && (!row_idx || !diffs))) return fail(MG_EINVAL, "null argument");
  if (n == 0) return MG_OK;
  if ((uint64_t)t->delta_count + n > t->delta_cap)
    return fail(MG_ERANGE, "delta buffer full: %u entries (max %u)", t->delta_count + n, t->delta_cap);
  for (uint32_t i = 0; i < n; ++i)
    if (row_idx[i] >= t->rows)
      return fail(MG_ERANGE, "delta row %llu outside the %llu-row table", (unsigned long long)row_idx[i],
                  (unsigned long long)t->rows);
  if (int rc = set_device(t)) return rc;
  // Entries first, then the device-side count that makes them visible.
  MG_CUDA(cudaMemcpy(t->d_delta_idx + t->delta_count, row_idx, (size_t)n * 8, cudaMemcpyHostToDevice));
  MG_CUDA(cudaMemcpy((uint8_t*)t->d_delta_diff + (size_t)t->delta_count * t->row_bytes, diffs,
                     (size_t)n * t->row_bytes, cudaMemcpyHostToDevice));
  const uint32_t c = t->delta_count + n;
  MG_CUDA(cudaMemcpy(t->d_delta_count, &c, 4, cudaMemcpyHostToDevice));
  t->delta_count = c;
  return MG_OK;
}

uint32_t mg_table_delta_count(const mg_table* t) { return t ? t->delta_count : 0; }

int mg_table_delta_clear(mg_table* t) {
  if (!t) return fail(MG_EINVAL, "null table");
  if (!t->delta_cap) return MG_OK;
  if (int rc = set_device(t)) return rc;
  const uint32_t z = 0;
  MG_CUDA(cudaDeviceSynchronize());
  MG_CUDA(cudaMemcpy(t->d_delta_count, &z, 4, cudaMemcpyHostToDevice));
  t->delta_count = 0;
  return MG_OK;
}

int mg_table_delta_merge(mg_table* t) {
  if (!t) return fail(MG_EINVAL, "null table");
  if (int rc = set_device(t)) return rc;
  // Passes already enqueued must finish against the old epoch first.
  MG_CUDA(cudaDeviceSynchronize());
  if (t->delta_count) {
    MG_CUDA(mg::launch_xor_rows(t->d, t->row_bytes / 16, t->d_delta_idx, t->d_delta_diff, t->delta_count, t->sms,
                                nullptr));
    const uint32_t z = 0;
    MG_CUDA(cudaMemcpy(t->d_delta_count, &z, 4, cudaMemcpyHostToDevice));
    MG_CUDA(cudaDeviceSynchronize());
    t->delta_count = 0;
  }
  ++t->epoch;
  return MG_OK;
}

uint64_t mg_table_epoch(const mg_table* t) { return t ? t->epoch : 0; }

// ---- keys -------------------------------------------------------------------

size_t mg_key_size(uint32_t d) { return 19 + (size_t)d * 18 + 16; }

int mg_key_check(const uint8_t* key, size_t len, uint32_t* domain_bits, uint8_t* party) {
  KeyDev k;
  if (int rc = parse_key(key, len, &k)) return rc;
  if (domain_bits) *domain_bits = k.domain_bits;
  if (party) *party = key[17];
  return MG_OK;
}

int mg_keygen(uint32_t d, uint64_t target, const uint8_t root0[16], const uint8_t root1[16],
              uint8_t* key0, uint8_t* key1) {
  if (!root0 || !root1 || !key0 || !key1) return fail(MG_EINVAL, "null argument");
  if (d == 0 || d > 32) return fail(MG_EINVAL, "invalid domain bits %u: must be in [1, 32]", d);
  if (target >= domain_size(d))
    return fail(MG_ERANGE, "page index %llu exceeds max %llu", (unsigned long long)target,
                (unsigned long long)domain_size(d));
  uint32_t s0[4], s1[4];
  for (int i = 0; i < 4; ++i) { s0[i] = le32(root0 + 4 * i); s1[i] = le32(root1 + 4 * i); }
  uint8_t t0 = 0, t1 = 1;
  const size_t len = mg_key_size(d);
  for (int i = 0; i < 16; ++i) { key0[i] = root0[i]; key1[i] = root1[i]; }
  key0[16] = 0; key1[16] = 1;
  key0[17] = 0; key1[17] = 1;
  key0[18] = (uint8_t)d; key1[18] = (uint8_t)d;
  size_t off = 19;
  for (uint32_t lvl = 0; lvl < d; ++lvl) {
    uint32_t L0[4], R0[4], L1[4], R1[4];
    uint8_t lt0, rt0, lt1, rt1;
    host_expand(s0, L0, R0, lt0, rt0);
    host_expand(s1, L1, R1, lt1, rt1);
    const int bit = (int)((target >> (d - 1 - lvl)) & 1u);
    const uint32_t* keep0 = bit ? R0 : L0;
    const uint32_t* lose0 = bit ? L0 : R0;
    const uint32_t* keep1 = bit ? R1 : L1;
    const uint32_t* lose1 = bit ? L1 : R1;
    const uint8_t keep_t0 = bit ? rt0 : lt0, lose_t0 = bit ? lt0 : rt0;
    const uint8_t keep_t1 = bit ? rt1 : lt1, lose_t1 = bit ? lt1 : rt1;
    uint32_t cw[4];
    for (int i = 0; i < 4; ++i) cw[i] = lose0[i] ^ lose1[i];
    const uint8_t tcw_lose = (uint8_t)(lose_t0 ^ lose_t1 ^ t0 ^ t1 ^ 1);
    const uint8_t tcw_keep = (uint8_t)(keep_t0 ^ keep_t1 ^ t0 ^ t1);
    for (int i = 0; i < 4; ++i) { put_le32(key0 + off + 4 * i, cw[i]); put_le32(key1 + off + 4 * i, cw[i]); }
    key0[off + 16] = key1[off + 16] = bit ? tcw_lose : tcw_keep;
    key0[off + 17] = key1[off + 17] = bit ? tcw_keep : tcw_lose;
    off += 18;
    for (int i = 0; i < 4; ++i) {
      s0[i] = keep0[i] ^ (t0 == 1 ? cw[i] : 0u);
      s1[i] = keep1[i] ^ (t1 == 1 ? cw[i] : 0u);
    }
    const uint8_t n0 = (uint8_t)(keep_t0 ^ (t0 == 1 ? tcw_keep : 0));
    const uint8_t n1 = (uint8_t)(keep_t1 ^ (t1 == 1 ? tcw_keep : 0));
    t0 = n0;
    t1 = n1;
  }
  for (int i = 0; i < 4; ++i) {
    const uint32_t f = s0[i] ^ s1[i] ^ 0xFFFFFFFFu;
    put_le32(key0 + off + 4 * i, f);
    put_le32(key1 + off + 4 * i, f);
  }
  (void)len;
  return MG_OK;
}

// ---- workspaces -------------------------------------------------------------

int mg_batch_create(mg_context* ctx, mg_batch** out) {
  if (!ctx || !out) return fail(MG_EINVAL, "null argument");
  *out = nullptr;
  if (int rc = set_device(ctx)) return rc;
  mg_batch* b = new mg_batch();
  b->ctx = ctx;
  b->device = ctx->device;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev_k0) != cudaSuccess || cudaEventCreate(&b->ev_km) != cudaSuccess ||
      cudaEventCreate(&b->ev_k1) != cudaSuccess ||
      cudaEventCreate(&b->ev_h0) != cudaSuccess || cudaEventCreate(&b->ev_h1) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    mg_batch_destroy(b);
    return fail(MG_ECUDA, "cannot create workspace stream/events");
  }
  *out = b;
  return MG_OK;
}

int mg_batch_destroy(mg_batch* b) {
  if (!b) return MG_OK;
  set_device(b);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->gexec_io) cudaGraphExecDestroy(b->gexec_io);
  if (b->d_keys) cudaFree(b->d_keys);
  if (b->h_keys) cudaFreeHost(b->h_keys);
  if (b->d_partial) cudaFree(b->d_partial);
  if (b->d_out) cudaFree(b->d_out);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->d_jobs) cudaFree(b->d_jobs);
  if (b->h_jobs) cudaFreeHost(b->h_jobs);
  if (b->d_fr_seed) cudaFree(b->d_fr_seed);
  if (b->d_fr_t) cudaFree(b->d_fr_t);
  for (int i = 0; i < 2; ++i) {
    if (b->d_tmp_seed[i]) cudaFree(b->d_tmp_seed[i]);
    if (b->d_tmp_t[i]) cudaFree(b->d_tmp_t[i]);
  }
  for (cudaEvent_t e : {b->ev_k0, b->ev_km, b->ev_k1, b->ev_done, b->ev_h0, b->ev_h1})
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return MG_OK;
}

int mg_batch_set_shape(mg_batch* b, uint32_t subtree_bits, uint32_t keys_per_cta) {
  if (!b) return fail(MG_EINVAL, "null workspace");
  if (subtree_bits > 32) return fail(MG_EINVAL, "subtree_bits %u > 32", subtree_bits);
  if (keys_per_cta && !mg::scan_g_supported((int)keys_per_cta))
    return fail(MG_EINVAL, "keys_per_cta %u not in {1,2,3,4,8}", keys_per_cta);
  b->shape_S = subtree_bits;
  b->shape_G = keys_per_cta;
  return MG_OK;
}

int mg_batch_set_kernel(mg_batch* b, int kind) {
  if (!b) return fail(MG_EINVAL, "null workspace");
  if (kind != MG_KERNEL_AUTO && kind != MG_KERNEL_CTA && kind != MG_KERNEL_WARP)
    return fail(MG_EINVAL, "unknown kernel kind %d", kind);
  b->kind_pref = kind;
  return MG_OK;
}

namespace {

// Plan one CTA-kernel launch over segs (at most kMaxSegs): tile depth S, the
// deepest in [8, 14] that still gives >= 4 waves of items (or the pinned one).
int plan_cta(mg_batch* b, const std::vector<SegPlan>& segs, int G, uint32_t col0, size_t& key_cursor,
             std::vector<uint32_t>& key_col, std::vector<uint32_t>& key_bytes, std::vector<uint32_t>& key_slot,
             mg_batch::Launch& out) {
  mg_context* ctx = b->ctx;
  for (uint32_t S_target = b->eff_S ? b->eff_S : 14;; --S_target) {
    mg_batch::Launch L;
    std::memset(&L.p, 0, sizeof L.p);
    L.kind = MG_KERNEL_CTA;
    L.G = G;
    L.col0 = col0;
    uint32_t slots = 2, cols = 0;
    uint64_t items = 0;
    size_t cursor = key_cursor;
    std::vector<std::pair<uint32_t, uint32_t>> assign;  // (key, column)
    for (size_t si = 0; si < segs.size(); ++si) {
      const SegPlan& sp = segs[si];
      mg::Segment& sg = L.p.seg[si];
      uint32_t S, U, M;
      shape_for(sp.d, S_target, S, U, M);
      sg.table = reinterpret_cast<const uint4*>(sp.table->d);
      sg.first = sp.table->first;
      sg.rows = sp.table->rows;
      sg.V = sp.table->row_bytes / 16;
      sg.d = sp.d;
      sg.S = S;
      sg.U = U;
      sg.M = M;
      sg.g = sp.g;
      sg.groups = (uint32_t)(sp.keys.size() / sp.g);
      sg.tiles = (uint32_t)level_count(sp.table, S);
      sg.item_begin = items;
      sg.key_base = (uint32_t)cursor;
      sg.col_base = cols;
      for (size_t j = 0; j < sp.keys.size(); ++j) {
        key_col[sp.keys[j]] = col0 + cols + (uint32_t)j * sg.V;
        key_bytes[sp.keys[j]] = sp.table->row_bytes;
        key_slot[sp.keys[j]] = (uint32_t)(cursor + j);
      }
      cursor += sp.keys.size();
      items += (uint64_t)sg.tiles * sg.groups;
      cols += (uint32_t)sp.keys.size() * sg.V;
      slots = std::max(slots, M);
    }
    L.p.nsegs = (uint32_t)segs.size();
    L.p.items = items;
    L.p.cols = cols;
    L.p.slots = slots;
    L.cols = cols;
    L.smem = mg::scan_smem_bytes(G, slots);
    int occ = 0;
    if (L.smem <= ctx->smem_optin) {
      if (int rc = prepare_g(ctx, G, L.smem)) return rc;
      occ = mg::scan_occupancy(G, L.smem);
    }
    const uint64_t slots_total = (uint64_t)std::max(occ, 1) * ctx->sms;
    const bool enough = occ > 0 && items >= 4 * slots_total;
    if (b->eff_S || enough || S_target <= 8) {
      if (occ <= 0) return fail(MG_EINVAL, "launch shape S=%u G=%d does not fit the device", S_target, G);
      L.grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(items, slots_total));
      L.nparts = L.grid;
      key_cursor = cursor;
      out = std::move(L);
      return MG_OK;
    }
  }
}

// Plan one warp-kernel launch over segs (same V, at most kMaxSegs): depth-first
// levels per lane M and the CTA width (16 warps, one CTA per SM, when their
// stacks fit the shared memory, else 8 or 4 warps).  The CTAs take their items
// dynamically, so an SM's four schedulers finish within about one item of one
// another; M is the deepest whose items per scheduler round up by at most 3%
// (fewer, deeper items need fewer frontier nodes), or pinned as
// subtree_bits = M + 5.
int plan_warp(mg_batch* b, const std::vector<SegPlan>& segs, int G, uint32_t VT, uint32_t col0,
              size_t& key_cursor, std::vector<uint32_t>& key_col, std::vector<uint32_t>& key_bytes,
              std::vector<uint32_t>& key_slot, uint64_t& fr_cursor, size_t& tmp_need, mg_batch::Launch& out) {
  mg_context* ctx = b->ctx;
  struct Cand { uint32_t M; double bal; uint64_t items; int occ; size_t smem; uint32_t nw; };
  std::vector<Cand> cands;
  const uint32_t pinned = b->eff_S;
  for (uint32_t Mt = 10; Mt >= 1; --Mt) {
    if (pinned && !(pinned >= 6 ? Mt == pinned - 5 : Mt == 1)) continue;
    uint64_t items = 0;
    uint32_t slots = 1;
    for (const SegPlan& sp : segs) {
      const uint32_t M = std::min(Mt, sp.d);
      const uint64_t nF = level_count(sp.table, M);
      items += (sp.keys.size() / sp.g) * ((nF + 31) / 32);
      slots = std::max(slots, M);
    }
    uint32_t nw = (uint32_t)mg::kWarps;
    size_t smem = mg::warp_smem_bytes(G, VT, slots, nw);
    while (smem > ctx->smem_optin && nw > 4) {
      nw /= 2;
      smem = mg::warp_smem_bytes(G, VT, slots, nw);
    }
    if (smem > ctx->smem_optin) continue;
    if (int rc = prepare_warp(ctx, G, VT, smem)) return rc;
    const int occ = mg::warp_occupancy(G, VT, smem, nw);
    if (occ <= 0) continue;
    // Items per warp scheduler (4 per SM), rounded up: the last item of
    // the busiest scheduler bounds the pass.
    const uint64_t sched = (uint64_t)ctx->sms * 4;
    const uint64_t worst = (items + sched - 1) / sched;
    const double bal = worst ? (double)items / ((double)worst * (double)sched) : 1.0;
    cands.push_back({Mt, bal, items, occ, smem, nw});
  }
  if (cands.empty()) return fail(MG_EINVAL, "no warp-kernel shape fits the device (G=%d)", G);
  const Cand* best = nullptr;
  for (const Cand& c : cands)
    if (c.bal >= 0.97) { best = &c; break; }  // deepest balanced
  if (!best) {
    best = &cands[0];
    for (const Cand& c : cands)
      if (c.bal > best->bal + 0.01) best = &c;
  }

  mg_batch::Launch L;
  std::memset(&L.w, 0, sizeof L.w);
  L.kind = MG_KERNEL_WARP;
  L.G = G;
  L.VT = VT;
  L.col0 = col0;
  uint64_t items = 0;
  uint32_t cols = 0, slots = 1;
  size_t cursor = key_cursor;
  for (size_t si = 0; si < segs.size(); ++si) {
    const SegPlan& sp = segs[si];
    mg::WarpSeg& sg = L.w.seg[si];
    const uint32_t M = std::min(best->M, sp.d);
    const uint64_t nF = level_count(sp.table, M);
    const uint32_t nk = (uint32_t)sp.keys.size();
    sg.table = reinterpret_cast<const uint4*>(sp.table->d);
    sg.first = sp.table->first;
    sg.rows = sp.table->rows;
    sg.item_begin = items;
    sg.fr_base = fr_cursor;
    sg.nF = nF;
    sg.tiles = (uint32_t)((nF + 31) / 32);
    sg.groups = nk / sp.g;
    sg.d = sp.d;
    sg.M = M;
    sg.g = sp.g;
    sg.key_base = (uint32_t)cursor;
    sg.col_base = cols;
    for (uint32_t j = 0; j < nk; ++j) {
      key_col[sp.keys[j]] = col0 + cols + j * VT;
      key_bytes[sp.keys[j]] = sp.table->row_bytes;
      key_slot[sp.keys[j]] = (uint32_t)(cursor + j);
    }
    // Frontier chain: levels 0 -> F = d - M.  Up to kFrontierLevels levels
    // it is one step from each key's root.  Deeper, every step expands
    // kFrontierLevels levels below one root per CTA, and the first step's
    // CTAs reach their roots (level A = F - kFrontierLevels * nsteps, 1..10)
    // by walking the path from the key's root themselves, so no narrow
    // one-CTA-per-key step sits above them.
    const uint32_t F = sp.d - M;
    const uint32_t FL = mg::kFrontierLevels;
    const uint32_t nsteps = F <= FL ? 1u : (F - 1) / FL;
    const uint32_t A = F <= FL ? 0u : F - FL * nsteps;
    uint32_t Lv = A;
    for (uint32_t st = 0; st < nsteps; ++st) {
      mg::FrontierStep f;
      std::memset(&f, 0, sizeof f);
      const uint32_t c = F <= FL ? F : FL;
      f.L_in = Lv;
      f.c = c;
      f.per = 1u;
      f.walk = (st == 0 && A > 0) ? 1u : 0u;
      f.n_in = Lv ? level_count(sp.table, sp.d - Lv) : 1;
      f.in_first = Lv ? level_first(sp.table, sp.d - Lv) : 0;
      f.n_out = level_count(sp.table, sp.d - (Lv + c));
      f.out_first = level_first(sp.table, sp.d - (Lv + c));
      const bool last = st + 1 == nsteps;
      f.out_base = last ? fr_cursor : 0;
      f.out_stride = last ? nF : f.n_out;
      if (!last) tmp_need = std::max<size_t>(tmp_need, (size_t)nk * f.n_out);
      f.keys = nullptr;  // set after allocation (key_base offset kept in in_t slot below)
      L.steps.push_back(f);
      L.step_keys.push_back(nk);
      Lv += c;
    }
    fr_cursor += (uint64_t)nk * nF;
    cursor += nk;
    items += (uint64_t)sg.groups * sg.tiles;
    cols += nk * VT;
    slots = std::max(slots, M);
  }
  L.w.nsegs = (uint32_t)segs.size();
  L.w.items = items;
  L.w.cols = cols;
  L.w.slots = slots;
  L.cols = cols;
  L.NW = best->nw;
  // A CTA's warps take its items in rounds.  When a CTA holds only a few
  // rounds and 16 warps leave much of the last one idle (4096 items on 148
  // CTAs: 27.7 per CTA, 1.73 per warp), 14 warps fill it (1.98 per warp):
  // measured 1% faster on the 2^20 x 256 B pass.  With many rounds the
  // 16 warps' latency hiding counts for more.
  if (L.NW == (uint32_t)mg::kWarps) {
    const double ipc = (double)items / (double)ctx->sms;
    auto fill = [&](uint32_t w) { return ipc / ((double)w * std::ceil(ipc / (double)w)); };
    if (std::ceil(ipc / mg::kWarps) <= 4.0 && fill(14) > fill(mg::kWarps) + 0.05 &&
        mg::warp_smem_bytes(G, VT, slots, 14) <= ctx->smem_optin)
      L.NW = 14;
  }
  L.smem = mg::warp_smem_bytes(G, VT, slots, L.NW);
  if (int rc = prepare_warp(ctx, G, VT, L.smem)) return rc;
  const int occ = mg::warp_occupancy(G, VT, L.smem, L.NW);
  if (occ <= 0) return fail(MG_EINVAL, "warp kernel does not fit the device");
  const uint64_t nctas = (uint64_t)occ * ctx->sms;
  const uint64_t need_ctas = (items + L.NW - 1) / L.NW;
  L.grid = (uint32_t)std::max<uint64_t>(1, std::min(nctas, need_ctas));
  L.nparts = L.grid * L.NW;
  key_cursor = cursor;
  out = std::move(L);
  return MG_OK;
}

}  // namespace

// mark: event recorded after the last scan launch (before its reduction),
// so that the scan kernels can be timed apart from the reductions.
static int enqueue_pass(mg_batch* b, cudaStream_t st, cudaEvent_t mark, bool out_zeroed = false) {
  for (size_t i = 0; i < b->launches.size(); ++i) {
    const mg_batch::Launch& L = b->launches[i];
    if (L.kind == MG_KERNEL_CTA) {
      MG_CUDA(mg::launch_scan(L.G, L.p, L.grid, L.smem, st));
    } else if (!mg::warp_reduces_in_kernel(L.G, L.VT)) {
      for (size_t k = 0; k < L.steps.size(); ++k) MG_CUDA(mg::launch_frontier(L.steps[k], L.step_keys[k], st));
      MG_CUDA(mg::launch_scan_warp(L.G, L.VT, L.w, L.grid, L.NW, L.smem, st));
    } else {
      // The scan CTAs reduce into the shares themselves; the first frontier
      // step zeroes them (a memset when no frontier step runs).
      bool zeroed = out_zeroed || L.cols == 0;
      for (size_t k = 0; k < L.steps.size(); ++k) {
        mg::FrontierStep f = L.steps[k];
        if (!zeroed && f.n_in > 0 && L.step_keys[k] > 0) {
          f.zero_out = b->d_out + L.col0;
          f.zero_n = L.cols;
          zeroed = true;
        }
        MG_CUDA(mg::launch_frontier(f, L.step_keys[k], st));
      }
      if (!zeroed) MG_CUDA(cudaMemsetAsync(b->d_out + L.col0, 0, (size_t)L.cols * 16, st));
      MG_CUDA(mg::launch_scan_warp(L.G, L.VT, L.w, L.grid, L.NW, L.smem, st));
    }
    if (mark && i + 1 == b->launches.size()) MG_CUDA(cudaEventRecord(mark, st));
    if (L.kind == MG_KERNEL_CTA || !mg::warp_reduces_in_kernel(L.G, L.VT))
      MG_CUDA(mg::launch_reduce(b->d_partial, L.nparts, L.cols, b->d_out + L.col0, st, out_zeroed));
  }
  for (const mg_batch::DeltaLaunch& dl : b->deltas)
    MG_CUDA(mg::launch_delta(b->d_keys, b->d_jobs + dl.job0, dl.njobs, dl.table->d_delta_idx, dl.table->d_delta_diff,
                             dl.table->d_delta_count, dl.table->delta_cap, dl.table->row_bytes / 16, dl.table->first,
                             b->d_out, st));
  return MG_OK;
}

namespace {

// Plan the pass for b->in_keys / b->in_tables with the effective shape
// (b->eff_kind, b->eff_S, b->eff_G), allocate, stage the keys and copy them
// to the device on the workspace stream.
int plan_pass(mg_batch* b) {
  const uint32_t nkeys = (uint32_t)b->in_keys.size();
  std::vector<KeyDev>& parsed = b->in_keys;
  std::vector<SegPlan> segs;
  for (uint32_t i = 0; i < nkeys; ++i) {
    const mg_table* t = b->in_tables[i];
    const uint32_t d = parsed[i].domain_bits;
    auto it = std::find_if(segs.begin(), segs.end(),
                           [&](const SegPlan& s) { return s.table == t && s.d == d; });
    if (it == segs.end()) {
      segs.push_back(SegPlan{t, d, {}, 1, false});
      it = segs.end() - 1;
    }
    it->keys.push_back(i);
  }

  // Kernel per segment: the warp kernel for rows of 16..512 B (V dividing
  // 32) and d >= 1, the CTA kernel otherwise.
  for (SegPlan& sp : segs) {
    const uint32_t V = sp.table->row_bytes / 16;
    const bool ok = mg::warp_vt_supported(V) && sp.d >= 1;
    if (b->eff_kind == MG_KERNEL_WARP && !ok)
      return fail(MG_EINVAL, "the warp kernel needs row_bytes in {16..512, powers of two} and d >= 1");
    sp.warp = ok && b->eff_kind != MG_KERNEL_CTA;
  }
  uint32_t Vc = 1, Vw = 1;
  size_t nc = 1, nwk = 1;
  for (const SegPlan& sp : segs) {
    const uint32_t V = sp.table->row_bytes / 16;
    if (sp.warp) { Vw = std::max(Vw, V); nwk = std::max(nwk, sp.keys.size()); }
    else { Vc = std::max(Vc, V); nc = std::max(nc, sp.keys.size()); }
  }
  const int Gc = choose_g(Vc, nc, b->eff_G, false);
  const int Gw = choose_g(Vw, nwk, b->eff_G, true);
  std::vector<SegPlan> split;
  for (SegPlan& sp : segs) {
    const int G = sp.warp ? Gw : Gc;
    const uint32_t g = (uint32_t)std::min<size_t>((size_t)G, sp.keys.size());
    const size_t full = sp.keys.size() / g * g;
    split.push_back(SegPlan{sp.table, sp.d, std::vector<uint32_t>(sp.keys.begin(), sp.keys.begin() + full), g, sp.warp});
    if (full < sp.keys.size())
      split.push_back(SegPlan{sp.table, sp.d, std::vector<uint32_t>(sp.keys.begin() + full, sp.keys.end()),
                              (uint32_t)(sp.keys.size() - full), sp.warp});
  }

  // Launches: CTA-kernel segments in chunks of kMaxSegs; warp-kernel segments
  // grouped by V, then chunks of kMaxSegs.
  std::vector<mg_batch::Launch> launches;
  std::vector<uint32_t> key_col(nkeys), key_bytes(nkeys), key_slot(nkeys);
  size_t key_cursor = 0, tmp_need = 0;
  uint64_t fr_cursor = 0;
  uint32_t total_cols = 0;
  std::vector<SegPlan> cta_segs;
  for (const SegPlan& sp : split)
    if (!sp.warp) cta_segs.push_back(sp);
  for (size_t s0 = 0; s0 < cta_segs.size(); s0 += mg::kMaxSegs) {
    std::vector<SegPlan> chunk(cta_segs.begin() + s0,
                               cta_segs.begin() + std::min(cta_segs.size(), s0 + mg::kMaxSegs));
    mg_batch::Launch L;
    if (int rc = plan_cta(b, chunk, Gc, total_cols, key_cursor, key_col, key_bytes, key_slot, L)) return rc;
    total_cols += L.cols;
    launches.push_back(std::move(L));
  }
  for (uint32_t VT = 1; VT <= 32; VT *= 2) {
    std::vector<SegPlan> ws;
    for (const SegPlan& sp : split)
      if (sp.warp && sp.table->row_bytes / 16 == VT) ws.push_back(sp);
    for (size_t s0 = 0; s0 < ws.size(); s0 += mg::kMaxSegs) {
      std::vector<SegPlan> chunk(ws.begin() + s0, ws.begin() + std::min(ws.size(), s0 + mg::kMaxSegs));
      mg_batch::Launch L;
      if (int rc = plan_warp(b, chunk, Gw, VT, total_cols, key_cursor, key_col, key_bytes, key_slot, fr_cursor,
                             tmp_need, L))
        return rc;
      total_cols += L.cols;
      launches.push_back(std::move(L));
    }
  }

  // Delta folding: one launch per table that holds a delta buffer.
  std::vector<mg_batch::DeltaLaunch> deltas;
  std::vector<uint2> jobs;
  for (uint32_t i = 0; i < nkeys; ++i) {
    const mg_table* t = b->in_tables[i];
    if (!t->delta_cap) continue;
    auto it = std::find_if(deltas.begin(), deltas.end(), [&](const mg_batch::DeltaLaunch& x) { return x.table == t; });
    if (it == deltas.end()) {
      deltas.push_back({t, 0, 0});
      it = deltas.end() - 1;
    }
  }
  for (mg_batch::DeltaLaunch& dl : deltas) {
    dl.job0 = (uint32_t)jobs.size();
    for (uint32_t i = 0; i < nkeys; ++i)
      if (b->in_tables[i] == dl.table) jobs.push_back(make_uint2(key_slot[i], key_col[i]));
    dl.njobs = (uint32_t)jobs.size() - dl.job0;
  }
  if (jobs.size() > b->cap_jobs) {
    if (b->d_jobs) cudaFree(b->d_jobs);
    if (b->h_jobs) cudaFreeHost(b->h_jobs);
    b->d_jobs = nullptr;
    b->h_jobs = nullptr;
    b->cap_jobs = 0;
    if (cudaMalloc(&b->d_jobs, jobs.size() * sizeof(uint2)) != cudaSuccess ||
        cudaMallocHost(&b->h_jobs, jobs.size() * sizeof(uint2)) != cudaSuccess) {
      cudaGetLastError();
      return fail(MG_ENOMEM, "cannot allocate delta job lists");
    }
    b->cap_jobs = jobs.size();
  }
  if (!jobs.empty()) {
    std::memcpy(b->h_jobs, jobs.data(), jobs.size() * sizeof(uint2));
    MG_CUDA(cudaMemcpyAsync(b->d_jobs, b->h_jobs, jobs.size() * sizeof(uint2), cudaMemcpyHostToDevice, b->stream));
  }
  b->deltas = std::move(deltas);

  size_t max_partial = 0;
  for (const mg_batch::Launch& L : launches) max_partial = std::max(max_partial, (size_t)L.nparts * L.cols);
  if (int rc = grow(b, nkeys, max_partial, total_cols, (size_t)fr_cursor, tmp_need)) return rc;
  mg::KeyAux* const h_aux = reinterpret_cast<mg::KeyAux*>(b->h_keys + nkeys);
  const mg::KeyAux* const d_aux = reinterpret_cast<const mg::KeyAux*>(b->d_keys + nkeys);
  for (uint32_t i = 0; i < nkeys; ++i) {
    b->h_keys[key_slot[i]] = parsed[i];
    make_aux(parsed[i], &h_aux[key_slot[i]]);
  }
  for (mg_batch::Launch& L : launches) {
    if (L.kind == MG_KERNEL_CTA) {
      L.p.keys = b->d_keys;
      L.p.partial = b->d_partial;
      continue;
    }
    L.w.keys = b->d_keys;
    L.w.aux = d_aux;
    L.w.fr_seed = b->d_fr_seed;
    L.w.fr_t = b->d_fr_t;
    L.w.partial = b->d_partial;
    L.w.out = b->d_out + L.col0;
    // Wire the frontier chains: each segment's steps are consecutive.
    size_t st = 0;
    for (uint32_t si = 0; si < L.w.nsegs; ++si) {
      const mg::WarpSeg& sg = L.w.seg[si];
      const uint32_t F = sg.d - sg.M;
      const uint32_t nsteps = F <= mg::kFrontierLevels ? 1u : (F - 1) / mg::kFrontierLevels;
      for (uint32_t k = 0; k < nsteps; ++k, ++st) {
        mg::FrontierStep& f = L.steps[st];
        f.keys = b->d_keys + sg.key_base;
        f.in_seed = k ? b->d_tmp_seed[(k - 1) & 1] : nullptr;
        f.in_t = k ? b->d_tmp_t[(k - 1) & 1] : nullptr;
        const bool last = k + 1 == nsteps;
        f.out_seed = last ? b->d_fr_seed : b->d_tmp_seed[k & 1];
        f.out_t = last ? b->d_fr_t : b->d_tmp_t[k & 1];
      }
    }
  }
  MG_CUDA(cudaMemcpyAsync(b->d_keys, b->h_keys, (size_t)nkeys * (sizeof(KeyDev) + sizeof(mg::KeyAux)),
                          cudaMemcpyHostToDevice, b->stream));
  b->launches = std::move(launches);
  b->total_cols = total_cols;
  b->plan_slot = key_slot;
  b->plan_depth.resize(nkeys);
  b->plan_deltas.resize(nkeys);
  for (uint32_t i = 0; i < nkeys; ++i) {
    b->plan_depth[i] = parsed[i].domain_bits;
    b->plan_deltas[i] = {b->in_tables[i]->d_delta_idx, b->in_tables[i]->delta_cap};
  }
  b->plan_tables = b->in_tables;
  b->plan_shapes.resize(nkeys);
  for (uint32_t i = 0; i < nkeys; ++i) b->plan_shapes[i] = table_shape(b->in_tables[i]);
  b->plan_kind = b->eff_kind;
  b->plan_S = b->eff_S;
  b->plan_G = b->eff_G;
  b->key_col = std::move(key_col);
  b->key_bytes = std::move(key_bytes);
  b->total_share_bytes = 0;
  for (uint32_t i = 0; i < nkeys; ++i) b->total_share_bytes += b->key_bytes[i];
  const mg_batch::Launch& L0 = b->launches[0];
  b->info.kernel = (uint32_t)L0.kind;
  b->info.keys_per_cta = (uint32_t)L0.G;
  b->info.grid = L0.grid;
  b->info.items = (uint32_t)(L0.kind == MG_KERNEL_CTA ? L0.p.items : L0.w.items);
  b->info.segments = (uint32_t)split.size();
  b->info.smem_bytes = (uint32_t)L0.smem;
  b->info.subtree_bits = 0;
  for (const mg_batch::Launch& L : b->launches) {
    if (L.kind == MG_KERNEL_CTA)
      for (uint32_t s = 0; s < L.p.nsegs; ++s) b->info.subtree_bits = std::max(b->info.subtree_bits, L.p.seg[s].S);
    else
      for (uint32_t s = 0; s < L.w.nsegs; ++s) b->info.subtree_bits = std::max(b->info.subtree_bits, L.w.seg[s].M + 5);
  }
  b->info.frontier_nodes = (uint32_t)std::min<uint64_t>(fr_cursor, 0xFFFFFFFFu);
  b->info.kernels = 0;
  for (const mg_batch::Launch& L : b->launches)
    b->info.kernels += (L.kind == MG_KERNEL_CTA || !mg::warp_reduces_in_kernel(L.G, L.VT) ? 2u : 1u) +
                       (uint32_t)L.steps.size();
  b->info.kernels += (uint32_t)b->deltas.size();
  b->planned = true;
  return MG_OK;
}

// Workload signature: the (rows, row bytes, depth, keys) of every segment.
std::string signature_of(const mg_batch* b) {
  std::vector<std::array<uint64_t, 4>> segs;
  for (size_t i = 0; i < b->in_keys.size(); ++i) {
    const mg_table* t = b->in_tables[i];
    const uint64_t d = b->in_keys[i].domain_bits;
    bool found = false;
    for (auto& s : segs)
      if (s[0] == (uint64_t)t->rows && s[1] == t->row_bytes && s[2] == d && !found) {
        ++s[3];
        found = true;
      }
    if (!found) segs.push_back({(uint64_t)t->rows, t->row_bytes, d, 1});
  }
  std::string sig = std::to_string(b->ctx->sms);
  for (auto& s : segs)
    for (uint64_t v : s) sig += ":" + std::to_string(v);
  return sig;
}

}  // namespace

int mg_batch_set_keys(mg_batch* b, const mg_table* const* tables, const uint8_t* const* keys,
                      const size_t* key_lens, uint32_t nkeys) {
  if (!b || !tables || !keys || !key_lens) return fail(MG_EINVAL, "null argument");
  if (nkeys == 0) return fail(MG_EINVAL, "no keys");
  if (int rc = set_device(b)) return rc;
  if (b->launched && cudaEventQuery(b->ev_done) == cudaErrorNotReady)
    return fail(MG_EBUSY, "workspace still owns a pass in flight");
  cudaGetLastError();
  mg_context* ctx = b->ctx;
  std::vector<KeyDev> parsed(nkeys);
  std::vector<const mg_table*> tabs(nkeys);
  for (uint32_t i = 0; i < nkeys; ++i) {
    const mg_table* t = tables[i];
    if (!t) return fail(MG_EINVAL, "null table for key %u", i);
    if (t->ctx != ctx) return fail(MG_EINVAL, "table of key %u belongs to another context", i);
    if (int rc = parse_key(keys[i], key_lens[i], &parsed[i])) return rc;
    const uint32_t d = parsed[i].domain_bits;
    if (t->first + t->rows > domain_size(d))
      return fail(MG_ERANGE, "more rows than domain size: rows [%llu, %llu), key %u has %u domain bits",
                  (unsigned long long)t->first, (unsigned long long)(t->first + t->rows), i, d);
    tabs[i] = t;
  }
  // Same tables, key depths and delta buffers as the planned pass, and the
  // same effective shape: keep the plan and its buffers, restage the keys.
  if (b->planned && tabs == b->plan_tables) {
    bool same = true;
    for (uint32_t i = 0; i < nkeys && same; ++i)
      same = parsed[i].domain_bits == b->plan_depth[i] && b->plan_shapes[i] == table_shape(tabs[i]) &&
             b->plan_deltas[i] == std::make_pair((const void*)tabs[i]->d_delta_idx, tabs[i]->delta_cap);
    int kind = b->kind_pref;
    uint32_t S = b->shape_S, G = b->shape_G;
    if (same && kind == MG_KERNEL_AUTO && S == 0 && G == 0) {
      // b->signature is this workload's signature (same tables and depths).
      std::lock_guard<std::mutex> lk(ctx->tune_mu);
      auto it = ctx->tuned.find(b->signature);
      if (it != ctx->tuned.end()) {
        kind = (int)it->second[0];
        S = it->second[1];
        G = it->second[2];
      }
    }
    if (same && kind == b->plan_kind && S == b->plan_S && G == b->plan_G) {
      mg::KeyAux* const h_aux = reinterpret_cast<mg::KeyAux*>(b->h_keys + nkeys);
      for (uint32_t i = 0; i < nkeys; ++i) {
        b->h_keys[b->plan_slot[i]] = parsed[i];
        make_aux(parsed[i], &h_aux[b->plan_slot[i]]);
      }
      b->key_copy_bytes = (size_t)nkeys * (sizeof(KeyDev) + sizeof(mg::KeyAux));
      if (!b->defer_key_copy)
        MG_CUDA(cudaMemcpyAsync(b->d_keys, b->h_keys, b->key_copy_bytes, cudaMemcpyHostToDevice, b->stream));
      b->in_keys = std::move(parsed);
      b->plan_reused = true;
      return MG_OK;
    }
  }
  b->plan_reused = false;
  b->in_keys = std::move(parsed);
  b->in_tables = std::move(tabs);
  b->signature = signature_of(b);
  // Effective shape: what the caller pinned, else a tuned shape for this
  // workload, else the planner's heuristics.
  b->eff_kind = b->kind_pref;
  b->eff_S = b->shape_S;
  b->eff_G = b->shape_G;
  if (b->kind_pref == MG_KERNEL_AUTO && b->shape_S == 0 && b->shape_G == 0) {
    std::lock_guard<std::mutex> lk(ctx->tune_mu);
    auto it = ctx->tuned.find(b->signature);
    if (it != ctx->tuned.end()) {
      b->eff_kind = (int)it->second[0];
      b->eff_S = it->second[1];
      b->eff_G = it->second[2];
    }
  }
  return plan_pass(b);
}

int mg_batch_autotune(mg_batch* b, uint32_t budget_ms, mg_plan_info* best_info, double* best_ms) {
  if (!b) return fail(MG_EINVAL, "null workspace");
  if (!b->planned) return fail(MG_EINVAL, "mg_batch_set_keys has not been called");
  if (int rc = set_device(b)) return rc;
  if (b->launched && cudaEventQuery(b->ev_done) == cudaErrorNotReady)
    return fail(MG_EBUSY, "workspace still owns a pass in flight");
  cudaGetLastError();
  struct Cand { int kind; uint32_t S, G; };
  std::vector<Cand> cands;
  cands.push_back({MG_KERNEL_AUTO, 0, 0});
  size_t nk = b->in_keys.size();
  bool warp_ok = true;
  for (size_t i = 0; i < nk; ++i)
    warp_ok = warp_ok && mg::warp_vt_supported(b->in_tables[i]->row_bytes / 16) && b->in_keys[i].domain_bits >= 1;
  const uint32_t Gs[4] = {1, 2, 3, 4};
  for (uint32_t G : Gs) {
    if (G > nk && G != 1) continue;
    if (warp_ok)
      for (uint32_t sb = 15; sb >= 6; --sb) cands.push_back({MG_KERNEL_WARP, sb, G});
    for (uint32_t S = 14; S >= 8; --S) cands.push_back({MG_KERNEL_CTA, S, G});
  }
  const int save_kind = b->eff_kind;
  const uint32_t save_S = b->eff_S, save_G = b->eff_G;
  std::vector<uint8_t> ref, got;
  double best = 1e300;
  Cand best_c = cands[0];
  std::vector<std::pair<double, size_t>> timed;  // (best ms, candidate index)
  const auto t0 = std::chrono::steady_clock::now();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  MG_CUDA(cudaEventCreate(&e0));
  MG_CUDA(cudaEventCreate(&e1));
  int rc = MG_OK;
  for (size_t ci = 0; ci < cands.size(); ++ci) {
    const Cand& c = cands[ci];
    if (ci > 0 && budget_ms &&
        std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(budget_ms))
      break;
    b->eff_kind = c.kind;
    b->eff_S = c.S;
    b->eff_G = c.G;
    if (plan_pass(b) != MG_OK) continue;  // shape does not fit: skip
    // Warm-up launch, then the best of three timed launches.
    if ((rc = enqueue_pass(b, b->stream, nullptr))) break;
    float ms_best = 1e30f;
    for (int r = 0; r < 3 && rc == MG_OK; ++r) {
      cudaEventRecord(e0, b->stream);
      rc = enqueue_pass(b, b->stream, nullptr);
      cudaEventRecord(e1, b->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(MG_ECUDA, "autotune launch failed"); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms_best = std::min(ms_best, ms);
      if (ci > 0 && ms > 4 * best) break;  // clearly worse: stop timing it
    }
    if (rc) break;
    got.resize((size_t)b->total_cols * 16);
    if (cudaMemcpy(got.data(), b->d_out, got.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = fail(MG_ECUDA, "autotune read-back failed");
      break;
    }
    // Same shares from every shape, compared in input-key order.
    std::vector<uint8_t> ordered;
    for (size_t i = 0; i < b->key_col.size(); ++i)
      ordered.insert(ordered.end(), got.begin() + (size_t)b->key_col[i] * 16,
                     got.begin() + (size_t)b->key_col[i] * 16 + b->key_bytes[i]);
    if (ref.empty()) ref = ordered;
    else if (ordered != ref) { rc = fail(MG_ECUDA, "autotune: shape %d/%u/%u changed the shares", c.kind, c.S, c.G); break; }
    if (ms_best < best) { best = ms_best; best_c = c; }
    timed.push_back({ms_best, ci});
  }
  // Confirmation: the three fastest shapes are timed again, alternating, so
  // that a drift of the clocks during the sweep (power or thermal limits on
  // HBM-bound passes) does not decide the choice.
  if (rc == MG_OK && timed.size() > 1) {
    std::sort(timed.begin(), timed.end());
    const size_t top = std::min<size_t>(3, timed.size());
    std::vector<double> again(top, 1e300);
    for (int round = 0; round < 2 && rc == MG_OK; ++round)
      for (size_t j = 0; j < top && rc == MG_OK; ++j) {
        const Cand& c = cands[timed[j].second];
        b->eff_kind = c.kind;
        b->eff_S = c.S;
        b->eff_G = c.G;
        if (plan_pass(b) != MG_OK) continue;
        if ((rc = enqueue_pass(b, b->stream, nullptr))) break;
        for (int r = 0; r < 2 && rc == MG_OK; ++r) {
          cudaEventRecord(e0, b->stream);
          rc = enqueue_pass(b, b->stream, nullptr);
          cudaEventRecord(e1, b->stream);
          if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(MG_ECUDA, "autotune launch failed"); break; }
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          again[j] = std::min(again[j], (double)ms);
        }
      }
    if (rc == MG_OK) {
      size_t bj = 0;
      for (size_t j = 1; j < top; ++j)
        if (again[j] < again[bj]) bj = j;
      best = again[bj];
      best_c = cands[timed[bj].second];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    b->eff_kind = save_kind; b->eff_S = save_S; b->eff_G = save_G;
    plan_pass(b);
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(b->ctx->tune_mu);
    b->ctx->tuned[b->signature] = {(uint32_t)best_c.kind, best_c.S, best_c.G};
  }
  b->eff_kind = best_c.kind;
  b->eff_S = best_c.S;
  b->eff_G = best_c.G;
  if ((rc = plan_pass(b))) return rc;
  if (best_info) *best_info = b->info;
  if (best_ms) *best_ms = best;
  return MG_OK;
}

int mg_batch_launch(mg_batch* b, void* stream) {
  if (!b) return fail(MG_EINVAL, "null workspace");
  if (!b->planned) return fail(MG_EINVAL, "mg_batch_set_keys has not been called");
  if (int rc = set_device(b)) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  if (st != b->stream) {
    // keys were staged on the workspace stream
    MG_CUDA(cudaEventRecord(b->ev_done, b->stream));
    MG_CUDA(cudaStreamWaitEvent(st, b->ev_done, 0));
  }
  MG_CUDA(cudaEventRecord(b->ev_k0, st));
  if (int rc = enqueue_pass(b, st, b->ev_km)) return rc;
  MG_CUDA(cudaEventRecord(b->ev_k1, st));
  MG_CUDA(cudaEventRecord(b->ev_done, st));
  b->launched = true;
  return MG_OK;
}

namespace {

// Everything baked into a captured pass: launch shapes and parameters (with
// every device pointer), delta buffers and the share buffer.
std::vector<uint8_t> pass_signature(const mg_batch* b) {
  std::vector<uint8_t> sig;
  auto add = [&](const void* p, size_t n) {
    const uint8_t* q = static_cast<const uint8_t*>(p);
    sig.insert(sig.end(), q, q + n);
  };
  for (const mg_batch::Launch& L : b->launches) {
    add(&L.kind, sizeof L.kind);
    add(&L.grid, sizeof L.grid);
    add(&L.smem, sizeof L.smem);
    add(&L.G, sizeof L.G);
    add(&L.VT, sizeof L.VT);
    add(&L.NW, sizeof L.NW);
    add(&L.col0, sizeof L.col0);
    if (L.kind == MG_KERNEL_CTA) add(&L.p, sizeof L.p);
    else add(&L.w, sizeof L.w);
    for (const mg::FrontierStep& f : L.steps) add(&f, sizeof f);
  }
  for (const mg_batch::DeltaLaunch& dl : b->deltas) {
    add(&dl, sizeof dl);
    add(&dl.table->d_delta_idx, sizeof dl.table->d_delta_idx);
    add(&dl.table->delta_cap, sizeof dl.table->delta_cap);
  }
  add(&b->d_out, sizeof b->d_out);
  return sig;
}

// mg_scan's replay of a reused plan: one graph holds the key upload (pinned
// staging buffer -> d_keys, clearing the shares), the pass and the share
// download (d_out -> pinned h_out), so a call costs one graph launch and one
// wait.  The graph is timed as a whole by events recorded around it.
int launch_io_graph(mg_batch* b) {
  std::vector<uint8_t> sig = pass_signature(b);
  auto add = [&](const void* p, size_t n) {
    const uint8_t* q = static_cast<const uint8_t*>(p);
    sig.insert(sig.end(), q, q + n);
  };
  add(&b->d_keys, sizeof b->d_keys);
  add(&b->h_keys, sizeof b->h_keys);
  add(&b->key_copy_bytes, sizeof b->key_copy_bytes);
  add(&b->h_out, sizeof b->h_out);
  add(&b->total_cols, sizeof b->total_cols);
  if (!b->gexec_io || sig != b->graph_io_sig) {
    if (b->gexec_io) {
      cudaGraphExecDestroy(b->gexec_io);
      b->gexec_io = nullptr;
    }
    cudaStream_t cap;
    MG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int rc = MG_OK;
    // Pinned host buffers are mapped at the same address on the device
    // (unified addressing), so kernels read the keys and write the shares
    // across the host link directly.
    const bool mapped = b->ctx->mapped_host;
    if (e == cudaSuccess) {
      if (mapped) {
        e = mg::launch_copy_u4(b->h_keys, b->d_keys, (uint32_t)(b->key_copy_bytes / 16), cap, b->d_out,
                               b->total_cols);
      } else {
        e = cudaMemcpyAsync(b->d_keys, b->h_keys, b->key_copy_bytes, cudaMemcpyHostToDevice, cap);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->d_out, 0, (size_t)b->total_cols * 16, cap);
      }
    }
    if (e == cudaSuccess) rc = enqueue_pass(b, cap, nullptr, true);
    if (e == cudaSuccess && rc == MG_OK)
      e = mapped ? mg::launch_copy_u4(b->d_out, b->h_out, b->total_cols, cap)
                 : cudaMemcpyAsync(b->h_out, b->d_out, (size_t)b->total_cols * 16, cudaMemcpyDeviceToHost, cap);
    // End the capture whatever happened above, so the stream can be destroyed.
    const cudaError_t e_end = cudaStreamEndCapture(cap, &graph);
    if (e == cudaSuccess) e = e_end;
    if (e == cudaSuccess && rc == MG_OK) e = cudaGraphInstantiate(&b->gexec_io, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (rc != MG_OK) return rc;
    if (e != cudaSuccess) {
      b->gexec_io = nullptr;
      return fail(MG_ECUDA, "graph capture: %s", cudaGetErrorString(e));
    }
    b->graph_io_sig = std::move(sig);
  }
  MG_CUDA(cudaEventRecord(b->ev_k0, b->stream));
  MG_CUDA(cudaGraphLaunch(b->gexec_io, b->stream));
  MG_CUDA(cudaEventRecord(b->ev_k1, b->stream));
  b->launched = true;
  return MG_OK;
}

}  // namespace

int mg_batch_launch_graph(mg_batch* b, void* stream) {
  if (!b) return fail(MG_EINVAL, "null workspace");
  if (!b->planned) return fail(MG_EINVAL, "mg_batch_set_keys has not been called");
  if (int rc = set_device(b)) return rc;
  const std::vector<uint8_t> sig = pass_signature(b);
  if (!b->gexec || sig != b->graph_sig) {
    if (b->gexec) {
      cudaGraphExecDestroy(b->gexec);
      b->gexec = nullptr;
    }
    cudaStream_t cap;
    MG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int rc = MG_OK;
    if (e == cudaSuccess) {
      rc = enqueue_pass(b, cap, nullptr);
      e = cudaStreamEndCapture(cap, &graph);
    }
    if (e == cudaSuccess && rc == MG_OK) e = cudaGraphInstantiate(&b->gexec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (rc != MG_OK) return rc;
    if (e != cudaSuccess) return fail(MG_ECUDA, "graph capture: %s", cudaGetErrorString(e));
    b->graph_sig = sig;
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  if (st != b->stream) {
    MG_CUDA(cudaEventRecord(b->ev_done, b->stream));
    MG_CUDA(cudaStreamWaitEvent(st, b->ev_done, 0));
  }
  MG_CUDA(cudaEventRecord(b->ev_k0, st));
  MG_CUDA(cudaGraphLaunch(b->gexec, st));
  MG_CUDA(cudaEventRecord(b->ev_km, st));  // a replayed pass is timed as a whole
  MG_CUDA(cudaEventRecord(b->ev_k1, st));
  MG_CUDA(cudaEventRecord(b->ev_done, st));
  b->launched = true;
  return MG_OK;
}

int mg_batch_read(mg_batch* b, uint8_t* out, void* stream) {
  if (!b || !out) return fail(MG_EINVAL, "null argument");
  if (!b->launched) return fail(MG_EINVAL, "no pass launched");
  if (int rc = set_device(b)) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  if (st != b->stream) {
    MG_CUDA(cudaStreamWaitEvent(b->stream, b->ev_done, 0));
  }
  MG_CUDA(cudaEventRecord(b->ev_h0, b->stream));
  MG_CUDA(cudaMemcpyAsync(b->h_out, b->d_out, (size_t)b->total_cols * 16, cudaMemcpyDeviceToHost,
                          b->stream));
  MG_CUDA(cudaEventRecord(b->ev_h1, b->stream));
  MG_CUDA(cudaEventRecord(b->ev_done, b->stream));
  MG_CUDA(cudaEventSynchronize(b->ev_done));
  size_t off = 0;
  for (size_t i = 0; i < b->key_col.size(); ++i) {
    std::memcpy(out + off, b->h_out + (size_t)b->key_col[i] * 16, b->key_bytes[i]);
    off += b->key_bytes[i];
  }
  return MG_OK;
}

int mg_batch_sync(mg_batch* b, uint32_t timeout_ms) {
  if (!b) return fail(MG_EINVAL, "null workspace");
  if (!b->launched) return MG_OK;
  if (int rc = set_device(b)) return rc;
  return wait_event(b->ev_done, timeout_ms);
}

int mg_batch_shares_device(mg_batch* b, const void** dptr, size_t* bytes) {
  if (!b || !dptr) return fail(MG_EINVAL, "null argument");
  *dptr = b->d_out;
  if (bytes) *bytes = (size_t)b->total_cols * 16;
  return MG_OK;
}

int mg_batch_plan(mg_batch* b, mg_plan_info* info) {
  if (!b || !info) return fail(MG_EINVAL, "null argument");
  if (!b->planned) return fail(MG_EINVAL, "mg_batch_set_keys has not been called");
  *info = b->info;
  return MG_OK;
}

int mg_batch_last_kernel_ns(mg_batch* b, uint64_t* ns) {
  if (!b || !ns) return fail(MG_EINVAL, "null argument");
  if (!b->launched) return fail(MG_EINVAL, "no pass launched");
  if (int rc = set_device(b)) return rc;
  float ms = 0.f;
  MG_CUDA(cudaEventSynchronize(b->ev_k1));
  MG_CUDA(cudaEventElapsedTime(&ms, b->ev_k0, b->ev_k1));
  *ns = (uint64_t)((double)ms * 1e6);
  return MG_OK;
}

int mg_batch_last_scan_ns(mg_batch* b, uint64_t* ns) {
  if (!b || !ns) return fail(MG_EINVAL, "null argument");
  if (!b->launched) return fail(MG_EINVAL, "no pass launched");
  if (int rc = set_device(b)) return rc;
  float ms = 0.f;
  MG_CUDA(cudaEventSynchronize(b->ev_km));
  MG_CUDA(cudaEventElapsedTime(&ms, b->ev_k0, b->ev_km));
  *ns = (uint64_t)((double)ms * 1e6);
  return MG_OK;
}

int mg_prg_peak(mg_context* ctx, uint32_t iters, double* expands_per_s) {
  if (!ctx || !expands_per_s) return fail(MG_EINVAL, "null argument");
  if (int rc = set_device(ctx)) return rc;
  uint32_t blocks = 0, threads = 0;
  uint32_t* d_out = nullptr;
  MG_CUDA(mg::prg_peak_shape(ctx->sms, &blocks, &threads));
  if (cudaMalloc(&d_out, (size_t)blocks * threads * 4) != cudaSuccess) {
    cudaGetLastError();
    return fail(MG_ENOMEM, "cannot allocate the microbenchmark output");
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t e = mg::launch_prg_peak(d_out, iters, blocks, threads, nullptr);  // warm-up
  float best = 0.f;
  for (int r = 0; r < 3 && e == cudaSuccess; ++r) {
    cudaEventRecord(e0);
    e = mg::launch_prg_peak(d_out, iters, blocks, threads, nullptr);
    cudaEventRecord(e1);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess && (best == 0.f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_out);
  if (e != cudaSuccess) return fail(MG_ECUDA, "prg peak: %s", cudaGetErrorString(e));
  *expands_per_s = (double)blocks * threads * iters / ((double)best * 1e-3);
  return MG_OK;
}

// ---- one-call scan ----------------------------------------------------------

int mg_scan(mg_context* ctx, const mg_table* const* tables, const uint8_t* const* keys,
            const size_t* key_lens, uint32_t nkeys, uint8_t* out, uint32_t timeout_ms,
            mg_timing* timing) {
  if (!ctx || !out) return fail(MG_EINVAL, "null argument");
  const auto t0 = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (int rc = set_device(ctx)) return rc;
  if (!ctx->internal) {
    mg_batch* b = nullptr;
    if (int rc = mg_batch_create(ctx, &b)) return rc;
    ctx->internal = b;
  }
  mg_batch* b = ctx->internal;
  if (b->launched && cudaEventQuery(b->ev_done) == cudaErrorNotReady)
    return fail(MG_EBUSY, "the previous pass on this context has not completed");
  cudaGetLastError();
  // A repeated workload (same plan as the previous call) leaves the key
  // upload to one CUDA graph with the pass and the share download; a new
  // one is planned (set_keys uploads its keys) and launched directly.
  b->defer_key_copy = true;
  int rc = mg_batch_set_keys(b, tables, keys, key_lens, nkeys);
  b->defer_key_copy = false;
  if (rc) return rc;
  const bool replay = b->plan_reused;
  if (replay) {
    if ((rc = launch_io_graph(b))) {
      // Nothing of the graph ran: upload the keys here so the workspace's
      // device keys match the call's whatever the caller does next.
      cudaGetLastError();
      cudaMemcpyAsync(b->d_keys, b->h_keys, b->key_copy_bytes, cudaMemcpyHostToDevice, b->stream);
      return rc;
    }
  } else {
    MG_CUDA(cudaEventRecord(b->ev_h0, b->stream));  // key H2D was enqueued before this point
    if ((rc = mg_batch_launch(b, nullptr))) return rc;
    MG_CUDA(cudaMemcpyAsync(b->h_out, b->d_out, (size_t)b->total_cols * 16, cudaMemcpyDeviceToHost,
                            b->stream));
    MG_CUDA(cudaEventRecord(b->ev_h1, b->stream));
  }
  MG_CUDA(cudaEventRecord(b->ev_done, b->stream));
  if ((rc = wait_event(b->ev_done, timeout_ms))) return rc;
  size_t off = 0;
  for (size_t i = 0; i < b->key_col.size(); ++i) {
    std::memcpy(out + off, b->h_out + (size_t)b->key_col[i] * 16, b->key_bytes[i]);
    off += b->key_bytes[i];
  }
  if (timing) {
    // A replayed call's graph holds the copies too: its device time is
    // reported as kernel time.
    float k_ms = 0.f, d_ms = 0.f;
    cudaEventElapsedTime(&k_ms, b->ev_k0, b->ev_k1);
    if (!replay) cudaEventElapsedTime(&d_ms, b->ev_k1, b->ev_h1);
    timing->kernel_ns = (uint64_t)((double)k_ms * 1e6);
    timing->d2h_ns = (uint64_t)((double)d_ms * 1e6);
    timing->total_ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                           std::chrono::steady_clock::now() - t0).count();
    const uint64_t rest = timing->kernel_ns + timing->d2h_ns;
    timing->h2d_ns = timing->total_ns > rest ? timing->total_ns - rest : 0;
  }
  return MG_OK;
}

// ---- point evaluation -------------------------------------------------------

int mg_eval_points(mg_context* ctx, const uint8_t* key, size_t key_len, const uint64_t* idx, uint64_t n,
                   uint8_t* out) {
  if (!ctx || (n && (!idx || !out))) return fail(MG_EINVAL, "null argument");
  KeyDev k;
  if (int rc = parse_key(key, key_len, &k)) return rc;
  if (n == 0) return MG_OK;
  if (int rc = set_device(ctx)) return rc;
  void *d_key = nullptr, *d_idx = nullptr, *d_out = nullptr;
  if (cudaMalloc(&d_key, sizeof k) != cudaSuccess || cudaMalloc(&d_idx, n * 8) != cudaSuccess ||
      cudaMalloc(&d_out, n * 16) != cudaSuccess) {
    cudaGetLastError();
    if (d_key) cudaFree(d_key);
    if (d_idx) cudaFree(d_idx);
    return fail(MG_ENOMEM, "cannot stage %llu evaluation points", (unsigned long long)n);
  }
  cudaError_t e = cudaMemcpy(d_key, &k, sizeof k, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_idx, idx, n * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = mg::launch_eval_points((const KeyDev*)d_key, (const uint64_t*)d_idx, n, d_out, ctx->sms, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(out, d_out, n * 16, cudaMemcpyDeviceToHost);
  cudaFree(d_key);
  cudaFree(d_idx);
  cudaFree(d_out);
  if (e != cudaSuccess) return fail(MG_ECUDA, "eval_points: %s", cudaGetErrorString(e));
  return MG_OK;
}

}  // extern "C"

namespace mg {
bool batch_done(mg_batch* b) {
  if (!b->launched) return true;
  cudaSetDevice(b->device);
  const cudaError_t e = cudaEventQuery(b->ev_done);
  if (e == cudaErrorNotReady) return false;
  cudaGetLastError();
  return true;
}
int context_device(const mg_context* ctx) { return ctx->device; }
}  // namespace mg
