// mg_kernels.cu -- sm_100a kernels of the per-server PIR answer path.
//
// scan_kernel<G>: persistent CTAs walk a list of (tile, key group) work items.
// For one item (an aligned subtree of 2^S rows and g <= G keys):
//   1. threads 0..g-1 walk each key from its root to the tile root (d - S
//      levels; the prefix walk of dpf.rs:183-203);
//   2. the CTA expands U levels breadth-first in shared memory, giving every
//      thread one node 2^M leaves above the rows (the GGM tree of
//      dpf.rs:210-246 in breadth-first order);
//   3. each thread walks its node depth-first with a per-thread stack in
//      shared memory, one leaf pair per step; the 16-byte leaf outputs
//      (masks) of all g keys go to shared memory;
//   4. the CTA scans the step's rows with coalesced 128-bit loads and
//      XOR-accumulates row & mask per key in registers (kernel.rs:1243-1256);
//   5. after the last step the per-thread accumulators are XOR-reduced with
//      warp shuffles and shared memory and folded into this CTA's own row of
//      the partial buffer (no atomics).
// reduce_kernel XORs the partial rows (per CTA, or per warp for the warp
// kernel) into the shares: slices of the rows in parallel, combined with
// 64-bit XOR atomics into the zeroed shares.  XOR is
// associative and commutative, so the shares are bit-exact whatever the
// schedule.  The kernels contain no waits on other CTAs or on the host.
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include "mg_device.cuh"
#include "mg_internal.h"
#include "morphogen_gpu.h"

namespace mg {

// Up to 4 keys per CTA the kernel is held to 80 registers so that three
// CTAs share an SM (page mode: more bytes in flight per SM).
template <int G>
__global__ void __launch_bounds__(kThreads, (G <= 4 ? 3 : 2)) scan_kernel(const __grid_constant__ ScanParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  KeyDev* s_keys = reinterpret_cast<KeyDev*>(smem_raw);
  uint4* s_mask = reinterpret_cast<uint4*>(smem_raw + G * sizeof(KeyDev));  // [G][2*T]
  uint4* s_seed = s_mask + G * 2 * kThreads;                                 // [G][slots][T]
  uint8_t* s_t = reinterpret_cast<uint8_t*>(s_seed + (size_t)G * p.slots * kThreads);
  const uint32_t tid = threadIdx.x;
  const uint32_t slots = p.slots;

  uint4* my_partial = p.partial + (size_t)blockIdx.x * p.cols;
  for (uint32_t c = tid; c < p.cols; c += kThreads) my_partial[c] = make_uint4(0u, 0u, 0u, 0u);

  for (uint64_t item = blockIdx.x; item < p.items; item += gridDim.x) {
    uint32_t si = 0;
    while (si + 1 < p.nsegs && item >= p.seg[si + 1].item_begin) ++si;
    const Segment& sg = p.seg[si];
    const uint64_t local = item - sg.item_begin;
    const uint32_t group = (uint32_t)(local % sg.groups);
    const uint32_t g = sg.g, V = sg.V, d = sg.d, S = sg.S, U = sg.U, M = sg.M;
    const uint32_t L0 = d - S;
    // Global index of the tile at level L0 (row-range tables start mid-domain).
    const uint32_t tile = (uint32_t)(local / sg.groups + (sg.first >> S));

    __syncthreads();  // the previous item is done with shared memory
    {
      const uint4* src = reinterpret_cast<const uint4*>(p.keys + sg.key_base + (size_t)group * g);
      uint4* dst = reinterpret_cast<uint4*>(s_keys);
      const uint32_t n = g * (uint32_t)(sizeof(KeyDev) / 16);
      for (uint32_t i = tid; i < n; i += kThreads) dst[i] = src[i];
    }
    __syncthreads();

    // 1. prefix walk to the tile root; the breadth-first ping-pong below
    //    starts in slot (U & 1) so that it ends in slot 0.
    const uint32_t start_slot = U & 1u;
    if (tid < g) {
      const KeyDev& K = s_keys[tid];
      uint4 s = K.root_seed;
      uint32_t t = K.root_t;
      for (uint32_t lvl = 0; lvl < L0; ++lvl) {
        uint4 Lc, Rc;
        uint32_t tl, tr;
        expand_cw(s, t, K, lvl, Lc, tl, Rc, tr);
        const uint32_t bit = (tile >> (L0 - 1 - lvl)) & 1u;
        s = bit ? Rc : Lc;
        t = bit ? tr : tl;
      }
      s_seed[(tid * slots + start_slot) * kThreads] = s;
      s_t[(tid * slots + start_slot) * kThreads] = (uint8_t)t;
    }
    __syncthreads();

    // 2. breadth-first expansion of U levels below the tile root.
    uint32_t cur = start_slot;
    for (uint32_t j = 0; j < U; ++j) {
      const uint32_t nxt = cur ^ 1u;
      const uint32_t work = g << j;
      for (uint32_t it = tid; it < work; it += kThreads) {
        const uint32_t k = it >> j, i = it & ((1u << j) - 1u);
        const size_t src = (k * slots + cur) * kThreads + i;
        const size_t dst = (k * slots + nxt) * kThreads + 2 * i;
        uint4 Lc, Rc;
        uint32_t tl, tr;
        expand_cw(s_seed[src], s_t[src], s_keys[k], L0 + j, Lc, tl, Rc, tr);
        s_seed[dst] = Lc;
        s_seed[dst + 1] = Rc;
        s_t[dst] = (uint8_t)tl;
        s_t[dst + 1] = (uint8_t)tr;
      }
      __syncthreads();
      cur = nxt;
    }

    // 3-4. depth-first leaf pairs + scan of the step's rows.
    uint4 acc[G];
#pragma unroll
    for (int k = 0; k < G; ++k) acc[k] = make_uint4(0u, 0u, 0u, 0u);
    const uint32_t NR = 1u << U;
    const uint32_t pairs = M ? (1u << (M - 1)) : 1u;
    const uint64_t tile_row0 = ((uint64_t)tile << S) - sg.first;  // table row of the tile's first leaf (may wrap)
    const uint32_t rpi = kThreads / V;  // rows per scan sweep
    const uint32_t lane = tid % V, rslot = tid / V;
    const bool scan_thread = tid < rpi * V;
    const uint4* __restrict__ tbl = sg.table;
    const uint64_t nrows = sg.rows;
    const uint32_t abs0 = d - M;  // tree level of the depth-first roots
    // Every row of the tile inside the table and every sweep of 8 rows full:
    // loads need no bounds checks.
    const bool full_tile = tile_row0 < nrows && nrows - tile_row0 >= (1ull << S) &&
                           (2 * NR) % (8 * rpi) == 0 && M > 0;

    for (uint32_t pi = 0; pi < pairs; ++pi) {
      if (tid < NR) {
#pragma unroll 1
        for (uint32_t k = 0; k < g; ++k) {
          const KeyDev& K = s_keys[k];
          uint4* col_seed = s_seed + (size_t)k * slots * kThreads + tid;
          uint8_t* col_t = s_t + (size_t)k * slots * kThreads + tid;
          uint4* mk = s_mask + (size_t)k * 2 * kThreads + 2 * tid;
          if (M == 0) {
            mk[0] = leaf_mask(col_seed[0], col_t[0], K);
            mk[1] = make_uint4(0u, 0u, 0u, 0u);
            continue;
          }
          // Pair pi's parent path re-joins the stack at relative level
          // M - 1 - ctz(pi) (root for pi == 0).
          uint32_t lvl = pi ? (M - (uint32_t)__ffs((int)pi)) : 0u;
          uint4 s = col_seed[lvl * kThreads];
          uint32_t t = col_t[lvl * kThreads];
          for (;; ++lvl) {
            uint4 Lc, Rc;
            uint32_t tl, tr;
            expand_cw(s, t, K, abs0 + lvl, Lc, tl, Rc, tr);
            if (lvl == M - 1) {
              mk[0] = leaf_mask(Lc, tl, K);
              mk[1] = leaf_mask(Rc, tr, K);
              break;
            }
            col_seed[(lvl + 1) * kThreads] = Rc;
            col_t[(lvl + 1) * kThreads] = (uint8_t)tr;
            s = Lc;
            t = tl;
          }
        }
      }
      __syncthreads();
      if (scan_thread && full_tile) {
        const uint4* __restrict__ bp = tbl + (tile_row0 + 2u * pi) * V + lane;
        for (uint32_t rb = rslot; rb < 2 * NR; rb += 8 * rpi) {
          uint4 dat[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const uint32_t r = rb + (uint32_t)u * rpi;
            dat[u] = __ldg(bp + (size_t)(((r >> 1) << M) + (r & 1u)) * V);
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const uint32_t r = rb + (uint32_t)u * rpi;
#pragma unroll
            for (int k = 0; k < G; ++k)
              if ((uint32_t)k < g) acc[k] = xor_and(acc[k], dat[u], s_mask[(size_t)k * 2 * kThreads + r]);
          }
        }
      } else if (scan_thread) {
        // Eight independent 128-bit loads in flight per thread before any
        // is consumed (wide rows leave one lane position per thread, so
        // this is what keeps enough bytes in flight for HBM).
        for (uint32_t rb = rslot; rb < 2 * NR; rb += 8 * rpi) {
          uint4 dat[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const uint32_t r = rb + (uint32_t)u * rpi;
            // Leaves before the table's first row wrap to huge values and fail the check.
            const uint64_t row = tile_row0 + ((uint64_t)(r >> 1) << M) + 2u * pi + (r & 1u);
            dat[u] = (r < 2 * NR && row < nrows) ? __ldg(tbl + row * V + lane) : make_uint4(0u, 0u, 0u, 0u);
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const uint32_t r = rb + (uint32_t)u * rpi;
            if (r < 2 * NR) {
#pragma unroll
              for (int k = 0; k < G; ++k)
                if ((uint32_t)k < g) acc[k] = xor_and(acc[k], dat[u], s_mask[(size_t)k * 2 * kThreads + r]);
            }
          }
        }
      }
      __syncthreads();
    }

    // 5. reduce the accumulators of threads holding the same lane.
    uint4* s_red = s_mask;  // G * T uint4 fit in the mask buffer
    const bool pow2 = (V & (V - 1)) == 0;
    if (pow2 && V < 32) {
#pragma unroll
      for (int k = 0; k < G; ++k) {
        uint4 v = acc[k];
        for (uint32_t off = 16; off >= V; off >>= 1) {
          v.x ^= __shfl_xor_sync(0xFFFFFFFFu, v.x, off);
          v.y ^= __shfl_xor_sync(0xFFFFFFFFu, v.y, off);
          v.z ^= __shfl_xor_sync(0xFFFFFFFFu, v.z, off);
          v.w ^= __shfl_xor_sync(0xFFFFFFFFu, v.w, off);
        }
        if ((tid & 31u) < V) s_red[(size_t)k * kThreads + (tid >> 5) * V + (tid & 31u)] = v;
      }
      __syncthreads();
      for (uint32_t o = tid; o < g * V; o += kThreads) {
        const uint32_t k = o / V, ln = o % V;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        for (uint32_t w = 0; w < kThreads / 32; ++w) v = xor4(v, s_red[(size_t)k * kThreads + w * V + ln]);
        const size_t col = sg.col_base + ((size_t)group * g + k) * V + ln;
        my_partial[col] = xor4(my_partial[col], v);
      }
    } else {
#pragma unroll
      for (int k = 0; k < G; ++k)
        s_red[(size_t)k * kThreads + tid] = scan_thread ? acc[k] : make_uint4(0u, 0u, 0u, 0u);
      __syncthreads();
      for (uint32_t o = tid; o < g * V; o += kThreads) {
        const uint32_t k = o / V, ln = o % V;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        for (uint32_t j = 0; j < rpi; ++j) v = xor4(v, s_red[(size_t)k * kThreads + ln + j * V]);
        const size_t col = sg.col_base + ((size_t)group * g + k) * V + ln;
        my_partial[col] = xor4(my_partial[col], v);
      }
    }
  }
}

// ---- warp-independent path -------------------------------------------------

// Frontier chain step: CTA (x, key) expands the `per` consecutive input slots
// x * per .. (level indices in_first + slot) of level L_in of key `blockIdx.y`
// by c <= kFrontierLevels levels breadth-first in shared memory (per * 2^c <=
// 2^kFrontierLevels nodes) and stores the nodes of level L_in + c that
// intersect the table, at slot (level index - out_first).  Several roots per
// CTA keep the top levels of a wide step busy; the first step (one root per
// key) is a latency chain either way.  The c levels' correction words are
// loaded into shared memory once, up front, so the level-by-level expansion
// waits on no memory access.
__global__ void __launch_bounds__(kThreads) frontier_kernel(const __grid_constant__ FrontierStep f) {
  constexpr uint32_t kNodes = 1u << kFrontierLevels;
  __shared__ uint4 sa[kNodes], sb[kNodes];
  __shared__ uint8_t ta[kNodes], tb[kNodes];
  __shared__ uint4 s_cw[kFrontierLevels];
  __shared__ uint32_t s_cwl[kFrontierLevels], s_cwr[kFrontierLevels];
  const uint32_t tid = threadIdx.x;
  const uint64_t node0 = (uint64_t)blockIdx.x * f.per, j = blockIdx.y;
  // The pass's shares start at zero: the scan CTAs XOR into them.
  if (f.zero_out && blockIdx.x == 0 && blockIdx.y == 0)
    for (uint64_t i = tid; i < f.zero_n; i += kThreads) f.zero_out[i] = make_uint4(0u, 0u, 0u, 0u);
  const uint32_t nroots = (uint32_t)(f.n_in - node0 < f.per ? f.n_in - node0 : f.per);
  const uint64_t g_out0 = (f.in_first + node0) << f.c;  // level index of the first child
  const uint64_t n = (uint64_t)nroots << f.c;
  if (g_out0 + n <= f.out_first || g_out0 >= f.out_first + f.n_out) return;  // uniform per CTA
  const KeyDev* __restrict__ K = f.keys + j;
  if (tid < f.c) {
    s_cw[tid] = __ldg(&K->cw_seed[f.L_in + tid]);
    s_cwl[tid] = __ldg(&K->cw_tl[f.L_in + tid]);
    s_cwr[tid] = __ldg(&K->cw_tr[f.L_in + tid]);
  }
  if (f.L_in == 0 || f.walk) {
    // The CTA's root (per == 1 when walking): node in_first + node0 of level
    // L_in, reached from the key's root as ChaCha::eval does (dpf.rs:103-142).
    // Warp 1 walks while warp 0 loads the step's correction words.
    if ((tid >> 5) == 1) {
      uint4 s = __ldg(&K->root_seed);
      uint32_t t = __ldg(&K->root_t);
      const uint64_t a = f.in_first + node0;
      for (uint32_t lvl = 0; lvl < f.L_in; ++lvl) {
        uint4 Lc, Rc;
        uint32_t tl, tr;
        expand_cw_g(s, t, K, lvl, Lc, tl, Rc, tr);
        const uint32_t bit = (uint32_t)(a >> (f.L_in - 1 - lvl)) & 1u;
        s = bit ? Rc : Lc;
        t = bit ? tr : tl;
      }
      if (tid == 32) {
        sa[0] = s;
        ta[0] = (uint8_t)t;
      }
    }
  } else {
    for (uint32_t r = tid; r < nroots; r += kThreads) {
      sa[r] = f.in_seed[j * f.n_in + node0 + r];
      ta[r] = f.in_t[j * f.n_in + node0 + r];
    }
  }
  __syncthreads();
  uint4* cs = sa; uint8_t* ct = ta;
  uint4* ns = sb; uint8_t* nt = tb;
  for (uint32_t lv = 0; lv < f.c; ++lv) {
    // Level lv holds nroots * 2^lv nodes, root-major; node i's children are
    // 2i and 2i + 1 of the next level.
    for (uint32_t i = tid; i < (nroots << lv); i += kThreads) {
      uint4 Lc, Rc;
      uint32_t tl, tr;
      prg_expand(cs[i], Lc, Rc, tl, tr);
      // dpf.rs:221-239: correction word on both children when t == 1.
      const uint32_t m = (ct[i] == 1) ? 0xFFFFFFFFu : 0u;
      const uint4 cw = s_cw[lv];
      Lc.x ^= cw.x & m; Lc.y ^= cw.y & m; Lc.z ^= cw.z & m; Lc.w ^= cw.w & m;
      Rc.x ^= cw.x & m; Rc.y ^= cw.y & m; Rc.z ^= cw.z & m; Rc.w ^= cw.w & m;
      ns[2 * i] = Lc;
      ns[2 * i + 1] = Rc;
      nt[2 * i] = (uint8_t)(tl ^ (s_cwl[lv] & m));
      nt[2 * i + 1] = (uint8_t)(tr ^ (s_cwr[lv] & m));
    }
    __syncthreads();
    uint4* x = cs; cs = ns; ns = x;
    uint8_t* y = ct; ct = nt; nt = y;
  }
  for (uint32_t i = tid; i < n; i += kThreads) {
    const uint64_t o = g_out0 + i - f.out_first;  // wraps for children before the range
    if (o < f.n_out) {
      f.out_seed[f.out_base + j * f.out_stride + o] = cs[i];
      f.out_t[f.out_base + j * f.out_stride + o] = ct[i];
    }
  }
}

// out ^= v with two 64-bit XOR atomics.
__device__ __forceinline__ void xor_out(uint4* out, const uint4 v) {
  unsigned long long* o = reinterpret_cast<unsigned long long*>(out);
  atomicXor(o, ((unsigned long long)v.y << 32) | v.x);
  atomicXor(o + 1, ((unsigned long long)v.w << 32) | v.z);
}

// Warp-independent fused expansion + scan.  A CTA of W warps (16 when its
// shared memory fits, else 8 or 4) owns a contiguous range
// of the pass's work items, in (tile, key group) order with the groups of a
// tile next to each other; its warps take the items one at a time from a
// shared-memory counter, so warps that share an SMSP with fewer busy warps
// simply take more items and every SM finishes within about one item of the
// others.  Per item each lane loads its frontier node and walks its 2^M
// leaves depth-first (stack in the warp's shared-memory slice); a step yields
// one leaf pair per lane for every key.  Accumulators stay in registers and
// are flushed (warp shuffle XOR) into the warp's own partial row when the
// group or segment changes.
// For rows of VT * G <= 2 uint4 each lane ANDs its own two rows with its own
// masks.  Otherwise the masks are exchanged through shared memory with
// __syncwarp only, and the warp scans the step's 64 rows (32 runs of 2) with
// coalesced 128-bit loads; VT divides 32, so a lane always holds the same
// 16-byte position of a row.  The first 8 of a lane's loads of a step are
// issued before the step's ChaCha work; wider rows load the rest after it,
// for 128-B rows in two halves each issued before the previous batch is
// consumed.
#ifndef MG_WARP_PREFETCH
#define MG_WARP_PREFETCH 8
#endif

// One depth-first step of a lane's walk: leaf pair `pi` of the lane's
// subtree (root at tree level F, M levels deep).  The path re-joins the
// stack (col_seed / col_t, stride 32) at relative level M - ffs(pi) (the
// root for pi == 0), pushes the right children it passes and returns the
// two leaf masks.
__device__ __forceinline__ void leaf_walk(const KeyDev* __restrict__ K, const KeyAux* __restrict__ A,
                                          uint4* col_seed, int8_t* col_t, uint32_t pi, uint32_t M, uint32_t F,
                                          uint4& ml, uint4& mr) {
  uint32_t lvl = pi ? (M - (uint32_t)__ffs((int)pi)) : 0u;
  uint4 s = col_seed[lvl * 32];
  uint32_t m = (uint32_t)(int32_t)col_t[lvl * 32];
  for (; lvl < M - 1; ++lvl) {
    uint4 Lc, Rc;
    uint32_t mlc, mrc;
    expand_cw_m(s, m, K, A, F + lvl, Lc, mlc, Rc, mrc);
    col_seed[(lvl + 1) * 32] = Rc;
    col_t[(lvl + 1) * 32] = (int8_t)mrc;
    s = Lc;
    m = mlc;
  }
  leaf_pair_m(s, m, A, ml, mr);
}

// Two depth-first steps at once (M >= 2): node q of relative level M - 2,
// whose children are the nodes of leaf pairs 2q and 2q + 1.  The path
// re-joins the stack at relative level M - 1 - ffs(q) (the root for q == 0),
// pushes the right children it passes and expands node q itself, so the
// second child stays in registers instead of taking a stack round trip.
__device__ __forceinline__ void pair_walk(const KeyDev* __restrict__ K, const KeyAux* __restrict__ A,
                                          uint4* col_seed, int8_t* col_t, uint32_t q, uint32_t M, uint32_t F,
                                          uint4& s0, uint32_t& m0, uint4& s1, uint32_t& m1) {
  uint32_t lvl = q ? (M - 1 - (uint32_t)__ffs((int)q)) : 0u;
  uint4 s = col_seed[lvl * 32];
  uint32_t m = (uint32_t)(int32_t)col_t[lvl * 32];
  for (; lvl < M - 2; ++lvl) {
    uint4 Lc, Rc;
    uint32_t mlc, mrc;
    expand_cw_m(s, m, K, A, F + lvl, Lc, mlc, Rc, mrc);
    col_seed[(lvl + 1) * 32] = Rc;
    col_t[(lvl + 1) * 32] = (int8_t)mrc;
    s = Lc;
    m = mlc;
  }
  expand_cw_m(s, m, K, A, F + M - 2, s0, m0, s1, m1);
}

template <int G, int VT>
__global__ void __launch_bounds__(kWarpThreads, 1) scan_warp_kernel(const __grid_constant__ WarpScanParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t s_next;  // next item of this CTA's range
  constexpr int NL = 2 * VT;            // uint4 loads per lane per step
  constexpr int PF = NL < MG_WARP_PREFETCH ? NL : MG_WARP_PREFETCH;  // loads issued before the ChaCha work
  constexpr uint32_t RPL = 32 / VT;     // rows covered by one warp-wide load
  // Rows of at most 32 B (one key per warp) or 16 B (two): every lane scans
  // its own subtree's two rows of the step (64 contiguous bytes, whole
  // sectors) against its own leaf masks, with no shared-memory exchange and
  // VT accumulators per key.  Wider rows use the exchange, which keeps the
  // loads coalesced and the register count flat.
  constexpr bool OWN = VT * G <= 2;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t nw = blockDim.x >> 5;
  const uint32_t slots = p.slots;
  uint4* const base4 = reinterpret_cast<uint4*>(smem_raw);
  uint4* const w_mask = base4 + (size_t)warp * G * 64;                                      // [G][64]
  uint4* const w_seed = base4 + (size_t)nw * G * 64 + (size_t)warp * G * slots * 32;           // [G][slots][32]
  // Stack t masks, one byte each (0 or 0xFF; sign-extended on load).
  int8_t* const w_t = reinterpret_cast<int8_t*>(base4 + (size_t)nw * G * 64 + (size_t)nw * G * slots * 32) +
                      (size_t)warp * G * slots * 32;

  const uint64_t gw = (uint64_t)blockIdx.x * nw + warp;
  uint4* const my_partial = p.partial + gw * p.cols;
  for (uint32_t c = lane; c < p.cols; c += 32) my_partial[c] = make_uint4(0u, 0u, 0u, 0u);
  const uint64_t c_begin = (uint64_t)blockIdx.x * p.items / gridDim.x;
  const uint64_t c_end = (uint64_t)(blockIdx.x + 1) * p.items / gridDim.x;
  if (threadIdx.x == 0) s_next = 0;
  __syncthreads();

  const uint32_t pos = lane % VT, r0 = lane / VT;
  constexpr int AV = OWN ? VT : 1;
  uint4 acc[G];
  uint4 own[G][AV];
#pragma unroll
  for (int k = 0; k < G; ++k) {
    acc[k] = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int v = 0; v < AV; ++v) own[k][v] = make_uint4(0u, 0u, 0u, 0u);
  }
  int cur_seg = -1;
  uint32_t cur_group = 0;

  auto flush_own = [&](const WarpSeg& sg, uint32_t group) {
#pragma unroll
    for (int k = 0; k < G; ++k) {
#pragma unroll
      for (int v = 0; v < AV; ++v) {
        uint4 x = own[k][v];
#pragma unroll
        for (uint32_t off = 16; off >= 1; off >>= 1) {
          x.x ^= __shfl_xor_sync(0xFFFFFFFFu, x.x, off);
          x.y ^= __shfl_xor_sync(0xFFFFFFFFu, x.y, off);
          x.z ^= __shfl_xor_sync(0xFFFFFFFFu, x.z, off);
          x.w ^= __shfl_xor_sync(0xFFFFFFFFu, x.w, off);
        }
        if ((uint32_t)k < sg.g && lane == (uint32_t)v) {
          const size_t col = sg.col_base + ((size_t)group * sg.g + k) * VT + v;
          my_partial[col] = xor4(my_partial[col], x);
        }
        own[k][v] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
  };

  auto flush = [&](const WarpSeg& sg, uint32_t group) {
    if constexpr (OWN) {
      flush_own(sg, group);
      return;
    }
#pragma unroll
    for (int k = 0; k < G; ++k) {
      uint4 v = acc[k];
#pragma unroll
      for (uint32_t off = 16; off >= (uint32_t)VT; off >>= 1) {
        v.x ^= __shfl_xor_sync(0xFFFFFFFFu, v.x, off);
        v.y ^= __shfl_xor_sync(0xFFFFFFFFu, v.y, off);
        v.z ^= __shfl_xor_sync(0xFFFFFFFFu, v.z, off);
        v.w ^= __shfl_xor_sync(0xFFFFFFFFu, v.w, off);
      }
      if ((uint32_t)k < sg.g && lane < (uint32_t)VT) {
        const size_t col = sg.col_base + ((size_t)group * sg.g + k) * VT + lane;
        my_partial[col] = xor4(my_partial[col], v);
      }
      acc[k] = make_uint4(0u, 0u, 0u, 0u);
    }
  };


  for (;;) {
    uint32_t rel = 0;
    if (lane == 0) rel = atomicAdd(&s_next, 1u);
    rel = __shfl_sync(0xFFFFFFFFu, rel, 0);
    const uint64_t item = c_begin + rel;
    if (item >= c_end) break;
    uint32_t si = 0;
    while (si + 1 < p.nsegs && item >= p.seg[si + 1].item_begin) ++si;
    const WarpSeg& sg = p.seg[si];
    const uint64_t local = item - sg.item_begin;
    const uint32_t tile = (uint32_t)(local / sg.groups);
    const uint32_t group = (uint32_t)(local % sg.groups);
    if ((int)si != cur_seg || group != cur_group) {
      if (cur_seg >= 0) flush(p.seg[cur_seg], cur_group);
      cur_seg = (int)si;
      cur_group = group;
    }
    const uint32_t g = sg.g, M = sg.M;
    const uint32_t F = sg.d - M;
    const uint64_t node = (uint64_t)tile * 32 + lane;
    const bool valid = node < sg.nF;
    const KeyDev* __restrict__ kp = p.keys + sg.key_base + (size_t)group * g;
    const KeyAux* __restrict__ ap = p.aux + sg.key_base + (size_t)group * g;
    for (uint32_t k = 0; k < g; ++k) {
      const uint64_t idx = sg.fr_base + ((uint64_t)group * g + k) * sg.nF + node;
      w_seed[(k * slots) * 32 + lane] = valid ? p.fr_seed[idx] : make_uint4(0u, 0u, 0u, 0u);
      w_t[(k * slots) * 32 + lane] = (valid && p.fr_t[idx] == 1) ? (int8_t)-1 : (int8_t)0;
    }
    const uint4* __restrict__ tbl = sg.table;
    const uint64_t nrows = sg.rows;
    // Table row of the warp tile's first leaf (wraps below the first row).
    const uint64_t row0 = (((sg.first >> M) + (uint64_t)tile * 32) << M) - sg.first;
    const uint32_t pairs = 1u << (M - 1);
    // A warp tile whose 32 x 2^M rows all lie in the table takes the
    // unchecked path: per-lane row pointers advance by one leaf pair per step
    // (load jj of a step is RPL / 2 producing lanes further on; RPL is even
    // for rows up to 256 B).
    const bool full = row0 < nrows && nrows - row0 >= ((uint64_t)32 << M);
    const uint4* const lp = full ? tbl + (row0 + ((uint64_t)(r0 >> 1) << M) + (r0 & 1u)) * VT + pos : tbl;
    const size_t jstride = ((size_t)(RPL >> 1) << M) * VT;
    // Own-rows path: the lane's first row of the tile (its subtree's leaves).
    const uint4* const own_lp = full ? tbl + (row0 + ((uint64_t)lane << M)) * VT : tbl;
    auto run_own = [&](auto full_tag) {
    constexpr bool FULL = decltype(full_tag)::value;
    if constexpr (FULL && G == 1) {
      // Odd leaf pairs are the right children of the even steps' last
      // expansion: they stay in registers (carry) instead of taking a
      // stack round trip.
      if (M >= 2) {
        const KeyDev* __restrict__ K0 = kp;
        const KeyAux* __restrict__ A0 = ap;
        uint4 carry_s = make_uint4(0u, 0u, 0u, 0u);
        uint32_t carry_m = 0u;
        for (uint32_t pi = 0; pi < pairs; ++pi) {
          uint4 dat[2 * AV];
#pragma unroll
          for (int j = 0; j < 2 * AV; ++j) dat[j] = __ldg(own_lp + (size_t)pi * (2 * VT) + j);
          uint4 sl;
          uint32_t msl;
          if (pi & 1u) {
            sl = carry_s;
            msl = carry_m;
          } else {
            pair_walk(K0, A0, w_seed + lane, w_t + lane, pi >> 1, M, F, sl, msl, carry_s, carry_m);
          }
          uint4 ml, mr;
          leaf_pair_m(sl, msl, A0, ml, mr);
#pragma unroll
          for (int v = 0; v < AV; ++v) {
            own[0][v] = xor_and(own[0][v], dat[v], ml);
            own[0][v] = xor_and(own[0][v], dat[AV + v], mr);
          }
        }
        return;
      }
    }
    for (uint32_t pi = 0; pi < pairs; ++pi) {
      uint4 dat[2 * AV];
#pragma unroll
      for (int j = 0; j < 2 * AV; ++j) {
        if constexpr (FULL) {
          dat[j] = __ldg(own_lp + (size_t)pi * (2 * VT) + j);
        } else {
          const uint64_t row = row0 + ((uint64_t)lane << M) + 2u * pi + (uint32_t)(j / AV);
          dat[j] = row < nrows ? __ldg(tbl + row * VT + (j % AV)) : make_uint4(0u, 0u, 0u, 0u);
        }
      }
#pragma unroll
      for (int k = 0; k < G; ++k) {
        if ((uint32_t)k >= g) break;
        uint4 ml, mr;
        leaf_walk(kp + k, ap + k, w_seed + (size_t)k * slots * 32 + lane, w_t + (size_t)k * slots * 32 + lane,
                  pi, M, F, ml, mr);
#pragma unroll
        for (int v = 0; v < AV; ++v) {
          own[k][v] = xor_and(own[k][v], dat[v], ml);
          own[k][v] = xor_and(own[k][v], dat[AV + v], mr);
        }
      }
    }
    };
    auto run_steps = [&](auto full_tag) {
    constexpr bool FULL = decltype(full_tag)::value && (RPL % 2 == 0);
    for (uint32_t pi = 0; pi < pairs; ++pi) {
      // Rows of this step: r = 2 * (producing lane) + leaf.
      uint4 dat[PF > 0 ? PF : 1];
#pragma unroll
      for (int jj = 0; jj < PF; ++jj) {
        const uint32_t r = r0 + (uint32_t)jj * RPL;
        const uint64_t row = row0 + ((uint64_t)(r >> 1) << M) + 2u * pi + (r & 1u);
        if constexpr (FULL) {
          (void)row;
          dat[jj] = __ldg(lp + (size_t)pi * (2 * VT) + (size_t)jj * jstride);
        } else {
          dat[jj] = row < nrows ? __ldg(tbl + row * VT + pos) : make_uint4(0u, 0u, 0u, 0u);
        }
      }
#pragma unroll 1
      for (uint32_t k = 0; k < g; ++k) {
        uint4 ml, mr;
        leaf_walk(kp + k, ap + k, w_seed + (size_t)k * slots * 32 + lane, w_t + (size_t)k * slots * 32 + lane,
                  pi, M, F, ml, mr);
        w_mask[k * 64 + 2 * lane] = ml;
        w_mask[k * 64 + 2 * lane + 1] = mr;
      }
      __syncwarp();
      auto load_rows = [&](uint4* buf, int j0, auto n_tag) {
        constexpr int N = decltype(n_tag)::value;
#pragma unroll
        for (int jj = 0; jj < N; ++jj) {
          const uint32_t r = r0 + (uint32_t)(j0 + jj) * RPL;
          const uint64_t row = row0 + ((uint64_t)(r >> 1) << M) + 2u * pi + (r & 1u);
          if constexpr (FULL) {
            (void)row;
            buf[jj] = __ldg(lp + (size_t)pi * (2 * VT) + (size_t)(j0 + jj) * jstride);
          } else {
            buf[jj] = row < nrows ? __ldg(tbl + row * VT + pos) : make_uint4(0u, 0u, 0u, 0u);
          }
        }
      };
      auto use_rows = [&](const uint4* buf, int j0, auto n_tag) {
        constexpr int N = decltype(n_tag)::value;
#pragma unroll
        for (int jj = 0; jj < N; ++jj) {
          const uint32_t r = r0 + (uint32_t)(j0 + jj) * RPL;
#pragma unroll
          for (int k = 0; k < G; ++k)
            if ((uint32_t)k < g) acc[k] = xor_and(acc[k], buf[jj], w_mask[k * 64 + r]);
        }
      };
      // The rest of the step's loads (the ChaCha registers are free now).
      // 128-B rows: two halves, each issued before the previous batch is
      // consumed.  Wider rows: chunks of 8 (holding more of them in flight
      // makes the kernel spill).
      constexpr int REST = NL - PF;
      if constexpr (REST == 0) {
        use_rows(dat, 0, std::integral_constant<int, PF>{});
      } else if constexpr (REST <= 8) {
        constexpr int H = REST / 2 > 0 ? (REST % 2 == 0 ? REST / 2 : REST) : REST;
        uint4 ma[H];
        load_rows(ma, PF, std::integral_constant<int, H>{});
        use_rows(dat, 0, std::integral_constant<int, PF>{});
        if constexpr (H < REST) {
          uint4 mb[REST - H];
          load_rows(mb, PF + H, std::integral_constant<int, REST - H>{});
          use_rows(ma, PF, std::integral_constant<int, H>{});
          use_rows(mb, PF + H, std::integral_constant<int, REST - H>{});
        } else {
          use_rows(ma, PF, std::integral_constant<int, H>{});
        }
      } else {
        use_rows(dat, 0, std::integral_constant<int, PF>{});
        constexpr int CH2 = 8;
        static_assert(REST % CH2 == 0, "load chunks must tile the step");
#pragma unroll 1
        for (int j0 = PF; j0 < NL; j0 += CH2) {
          uint4 more[CH2];
          load_rows(more, j0, std::integral_constant<int, CH2>{});
          use_rows(more, j0, std::integral_constant<int, CH2>{});
        }
      }
      __syncwarp();
    }
    };
    if constexpr (OWN) {
      if (full)
        run_own(std::true_type{});
      else
        run_own(std::false_type{});
    } else {
      if (full)
        run_steps(std::true_type{});
      else
        run_steps(std::false_type{});
    }
  }
  if (cur_seg >= 0) flush(p.seg[cur_seg], cur_group);
  if constexpr (!OWN) {
    // Cross-block reduction of the wide-row instantiations: the CTA XORs its
    // warps' partial rows (written by this CTA, visible after the barrier;
    // plain loads, not the read-only path) and folds the result into the
    // zeroed shares with 64-bit XOR atomics.  XOR is associative and
    // commutative, so the shares do not depend on the order.  (The own-rows
    // instantiations leave this to reduce_kernel: the extra code changes
    // their register allocation and costs 0.5% on the 31-bit pass, far more
    // than the reduction launch it saves.)
    __syncthreads();
    const uint4* const cta_part = p.partial + (uint64_t)blockIdx.x * nw * p.cols;
    for (uint32_t c = threadIdx.x; c < p.cols; c += blockDim.x) {
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      for (uint32_t w = 0; w < nw; ++w) v = xor4(v, cta_part[(size_t)w * p.cols + c]);
      xor_out(p.out + c, v);
    }
  }
}

// Whether scan_warp_kernel<G, VT> reduces its partial rows into the shares
// itself (wide rows) or leaves them to reduce_kernel (own-rows scan).
bool warp_reduces_in_kernel(int G, uint32_t VT) { return (uint32_t)G * VT > 2u; }

// out[c] ^= XOR over the nparts partial rows (launch_reduce zeroes out first).
// Block (x, y) = cpb columns x (kThreads / cpb) slices over the partial rows
// [y * per_block, (y + 1) * per_block); slices combine in shared memory and
// each block folds its result into out with XOR atomics.
__global__ void __launch_bounds__(kThreads) reduce_kernel(const uint4* __restrict__ partial,
                                                          uint32_t nparts, uint32_t cols,
                                                          uint32_t per_block, uint4* __restrict__ out) {
  __shared__ uint4 red[kThreads];
  const uint32_t cpb = cols < 32u ? cols : 32u;
  const uint32_t slices = kThreads / cpb;
  const uint32_t cl = threadIdx.x % cpb, sl = threadIdx.x / cpb;
  const uint32_t c = blockIdx.x * cpb + cl;
  const uint32_t j0 = blockIdx.y * per_block;
  const uint32_t j1 = min(nparts, j0 + per_block);
  uint4 v = make_uint4(0u, 0u, 0u, 0u);
  if (c < cols && sl < slices)
    for (uint32_t j = j0 + sl; j < j1; j += slices) v = xor4(v, partial[(size_t)j * cols + c]);
  red[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < cpb && c < cols) {
    uint4 r = make_uint4(0u, 0u, 0u, 0u);
    for (uint32_t s = 0; s < slices; ++s) r = xor4(r, red[s * cpb + threadIdx.x]);
    xor_out(out + c, r);
  }
}

// ChaChaKey::eval (dpf.rs:103-142) of one index: the d-level path walk.
__device__ __forceinline__ uint4 eval_leaf(const KeyDev* __restrict__ K, uint64_t x) {
  uint4 s = __ldg(&K->root_seed);
  uint32_t t = __ldg(&K->root_t);
  const uint32_t d = __ldg(&K->domain_bits);
  for (uint32_t lvl = 0; lvl < d; ++lvl) {
    uint4 Lc, Rc;
    uint32_t tl, tr;
    expand_cw_g(s, t, K, lvl, Lc, tl, Rc, tr);
    const uint32_t bit = (uint32_t)(x >> (d - 1 - lvl)) & 1u;
    s = bit ? Rc : Lc;
    t = bit ? tr : tl;
  }
  return leaf_mask_g(s, t, K);
}

// Pending epoch delta of a table folded into the shares of the pass
// (scan_delta_for_gpu, crates/morphogen-server/src/scan.rs:434-485, in row
// mode): out[col_j] ^= XOR_e diff_e & eval_j(row_e) for every job j (a key
// scanned over this table).  One thread per entry evaluates its row; each
// 16-byte position is XOR-reduced across the warp with shuffles, then across
// the CTA in shared memory, and the CTA's result is XORed into the share
// with one atomic per word (XOR is order-independent, so the result is
// deterministic).  The entry count is read on the device so that pushes are
// seen by replayed graphs.
__global__ void __launch_bounds__(kThreads) delta_kernel(const KeyDev* __restrict__ keys, const uint2* __restrict__ jobs,
                                                         const uint64_t* __restrict__ idx, const uint4* __restrict__ diffs,
                                                         const uint32_t* __restrict__ count, uint32_t V, uint64_t first,
                                                         uint4* __restrict__ out) {
  __shared__ uint4 s_acc[MG_MAX_ROW_BYTES / 16];
  const uint32_t n = *count;
  const uint64_t e0 = (uint64_t)blockIdx.x * kThreads;
  if (e0 >= n) return;  // uniform per CTA
  const uint2 job = jobs[blockIdx.y];
  const KeyDev* __restrict__ K = keys + job.x;
  for (uint32_t v = threadIdx.x; v < V; v += kThreads) s_acc[v] = make_uint4(0u, 0u, 0u, 0u);
  const uint64_t e = e0 + threadIdx.x;
  const bool live = e < n;
  const uint4 m = live ? eval_leaf(K, first + idx[e]) : make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t v = 0; v < V; ++v) {
    uint4 c = live ? diffs[e * V + v] : make_uint4(0u, 0u, 0u, 0u);
    c.x &= m.x; c.y &= m.y; c.z &= m.z; c.w &= m.w;
#pragma unroll
    for (uint32_t off = 16; off >= 1; off >>= 1) {
      c.x ^= __shfl_xor_sync(0xFFFFFFFFu, c.x, off);
      c.y ^= __shfl_xor_sync(0xFFFFFFFFu, c.y, off);
      c.z ^= __shfl_xor_sync(0xFFFFFFFFu, c.z, off);
      c.w ^= __shfl_xor_sync(0xFFFFFFFFu, c.w, off);
    }
    if (lane == 0 && (c.x | c.y | c.z | c.w)) {
      atomicXor(&s_acc[v].x, c.x);
      atomicXor(&s_acc[v].y, c.y);
      atomicXor(&s_acc[v].z, c.z);
      atomicXor(&s_acc[v].w, c.w);
    }
  }
  __syncthreads();
  for (uint32_t v = threadIdx.x; v < V; v += kThreads) {
    const uint4 a = s_acc[v];
    if (a.x | a.y | a.z | a.w) {
      unsigned int* o = reinterpret_cast<unsigned int*>(out + job.y + v);
      atomicXor(o + 0, a.x);
      atomicXor(o + 1, a.y);
      atomicXor(o + 2, a.z);
      atomicXor(o + 3, a.w);
    }
  }
}

// SplitMix64 output `w` of the stream seeded with `seed` (Steele, Lea, Flood 2014).
__device__ __forceinline__ uint64_t splitmix_word(uint64_t seed, uint64_t w) {
  uint64_t z = seed + (w + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void fill_splitmix_kernel(uint2* __restrict__ dst, uint64_t words, uint64_t seed, uint64_t word0) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
    const uint64_t z = splitmix_word(seed, word0 + w);
    dst[w] = make_uint2((uint32_t)z, (uint32_t)(z >> 32));
  }
}

// dst[i] = src[i] for n 16-byte words, and zero[i] = 0 for nz.  Used
// inside the one-call path's graph to move the keys in (clearing the shares
// at the same time) and the shares out through the pinned host buffers'
// device-mapped addresses: a kernel node of a few hundred threads finishes
// sooner than a copy-engine transfer of a few KB.
__global__ void copy_u4_kernel(const uint4* __restrict__ src, uint4* __restrict__ dst, uint32_t n,
                               uint4* __restrict__ zero, uint32_t nz) {
  const uint32_t m = n > nz ? n : nz;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    if (i < n) dst[i] = src[i];
    if (i < nz) zero[i] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// table[row_idx[e]] ^= diff[e]; XOR atomics make duplicate rows in one batch
// order-independent.
__global__ void xor_rows_kernel(uint4* __restrict__ table, uint32_t V, const uint64_t* __restrict__ idx,
                                const uint4* __restrict__ diffs, uint64_t n) {
  const uint64_t total = n * V;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const uint64_t e = i / V;
    const uint32_t ln = (uint32_t)(i % V);
    const uint4 dv = diffs[i];
    unsigned int* t = reinterpret_cast<unsigned int*>(table + idx[e] * V + ln);
    atomicXor(t + 0, dv.x);
    atomicXor(t + 1, dv.y);
    atomicXor(t + 2, dv.z);
    atomicXor(t + 3, dv.w);
  }
}

// ChaChaKey::eval (dpf.rs:103-142) at n indices, one thread per index.
__global__ void eval_points_kernel(const KeyDev* __restrict__ key, const uint64_t* __restrict__ idx,
                                   uint64_t n, uint4* __restrict__ out) {
  __shared__ KeyDev sk;
  {
    const uint4* src = reinterpret_cast<const uint4*>(key);
    uint4* dst = reinterpret_cast<uint4*>(&sk);
    for (uint32_t i = threadIdx.x; i < sizeof(KeyDev) / 16; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t x = idx[i];
    uint4 s = sk.root_seed;
    uint32_t t = sk.root_t;
    const uint32_t d = sk.domain_bits;
    for (uint32_t lvl = 0; lvl < d; ++lvl) {
      uint4 Lc, Rc;
      uint32_t tl, tr;
      expand_cw(s, t, sk, lvl, Lc, tl, Rc, tr);
      const uint32_t bit = (uint32_t)(x >> (d - 1 - lvl)) & 1u;
      s = bit ? Rc : Lc;
      t = bit ? tr : tl;
    }
    out[i] = leaf_mask(s, t, sk);
  }
}

// PRG-only ceiling: every thread chains `iters` node expansions (left child,
// t folded in) with no memory traffic -- the best the ChaCha8 code above can
// do on this GPU, the ALU roofline of the scan kernel.
__global__ void __launch_bounds__(256) prg_peak_kernel(uint32_t* __restrict__ out, uint32_t iters) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint4 s = make_uint4(tid, tid * 0x9E3779B9u, ~tid, 0x01234567u);
  uint32_t acc = 0;
  for (uint32_t i = 0; i < iters; ++i) {
    uint4 L, R;
    uint32_t tl, tr;
    prg_expand(s, L, R, tl, tr);
    s = make_uint4(L.x ^ R.w, L.y ^ tl, L.z ^ tr, L.w ^ R.x);
    acc += R.y;
  }
  out[tid] = s.x ^ s.y ^ s.z ^ s.w ^ acc;
}

// ---- host-side launchers --------------------------------------------------

// The dynamic shared memory limit of a kernel (cudaFuncAttributeMax-
// DynamicSharedMemorySize) belongs to the kernel function on its device, for
// the whole process: every context, workspace and the allocation-free entry
// point see the same value.  It is therefore kept here as one high-water mark
// per (device, kernel) under one mutex and only ever raised, so that a caller
// preparing a small launch can never lower the limit under another caller's
// larger launch.
namespace {
std::mutex g_smem_mu;
std::map<std::pair<int, const void*>, size_t> g_smem_limit;

cudaError_t raise_smem_limit(const void* fn, size_t smem) {
  int dev = 0;
  if (cudaError_t e = cudaGetDevice(&dev)) return e;
  std::lock_guard<std::mutex> lk(g_smem_mu);
  size_t& have = g_smem_limit[{dev, fn}];
  if (have >= smem) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) have = smem;
  return e;
}
}  // namespace

cudaError_t prg_peak_shape(int sms, uint32_t* blocks, uint32_t* threads) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, prg_peak_kernel, 256, 0);
  if (e != cudaSuccess) return e;
  *threads = 256;
  *blocks = (uint32_t)(per_sm > 0 ? per_sm : 1) * (uint32_t)sms * 4;
  return cudaSuccess;
}

cudaError_t launch_prg_peak(uint32_t* out, uint32_t iters, uint32_t blocks, uint32_t threads,
                            cudaStream_t st) {
  prg_peak_kernel<<<blocks, threads, 0, st>>>(out, iters);
  return cudaGetLastError();
}

size_t scan_smem_bytes(int G, uint32_t slots) {
  return (size_t)G * (sizeof(KeyDev) + 2 * kThreads * 16 + (size_t)slots * kThreads * 17);
}

template <int G>
static cudaError_t launch_scan_t(const ScanParams& p, uint32_t grid, size_t smem, cudaStream_t st) {
  scan_kernel<G><<<grid, kThreads, smem, st>>>(p);
  return cudaGetLastError();
}

template <int G>
static cudaError_t prepare_t(size_t smem) {
  return raise_smem_limit(reinterpret_cast<const void*>(scan_kernel<G>), smem);
}

template <int G>
static int occupancy_t(size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, scan_kernel<G>, kThreads, smem) != cudaSuccess)
    return 0;
  return n;
}

#define MG_G_DISPATCH(G_, EXPR1, EXPR2, EXPR3, EXPR4, EXPR8) \
  switch (G_) {                                              \
    case 1: return EXPR1;                                    \
    case 2: return EXPR2;                                    \
    case 3: return EXPR3;                                    \
    case 4: return EXPR4;                                    \
    case 8: return EXPR8;                                    \
    default: break;                                          \
  }

bool scan_g_supported(int G) { return G == 1 || G == 2 || G == 3 || G == 4 || G == 8; }

cudaError_t scan_prepare(int G, size_t smem) {
  MG_G_DISPATCH(G, prepare_t<1>(smem), prepare_t<2>(smem), prepare_t<3>(smem), prepare_t<4>(smem),
                prepare_t<8>(smem));
  return cudaErrorInvalidValue;
}

int scan_occupancy(int G, size_t smem) {
  MG_G_DISPATCH(G, occupancy_t<1>(smem), occupancy_t<2>(smem), occupancy_t<3>(smem),
                occupancy_t<4>(smem), occupancy_t<8>(smem));
  return 0;
}

cudaError_t launch_scan(int G, const ScanParams& p, uint32_t grid, size_t smem, cudaStream_t st) {
  MG_G_DISPATCH(G, launch_scan_t<1>(p, grid, smem, st), launch_scan_t<2>(p, grid, smem, st),
                launch_scan_t<3>(p, grid, smem, st), launch_scan_t<4>(p, grid, smem, st),
                launch_scan_t<8>(p, grid, smem, st));
  return cudaErrorInvalidValue;
}

cudaError_t launch_reduce(const uint4* partial, uint32_t nparts, uint32_t cols, uint4* out,
                          cudaStream_t st, bool out_zeroed) {
  if (cols == 0) return cudaSuccess;
  if (!out_zeroed)
    if (cudaError_t e = cudaMemsetAsync(out, 0, (size_t)cols * 16, st)) return e;
  const uint32_t cpb = cols < 32u ? cols : 32u;
  const uint32_t slices = kThreads / cpb;
  const uint32_t per_block = slices * 4;  // at most 4 partial rows per thread
  const dim3 grid((cols + cpb - 1) / cpb, nparts ? (nparts + per_block - 1) / per_block : 1);
  reduce_kernel<<<grid, kThreads, 0, st>>>(partial, nparts, cols, per_block, out);
  return cudaGetLastError();
}

cudaError_t launch_copy_u4(const void* src, void* dst, uint32_t n, cudaStream_t st, void* zero, uint32_t nz) {
  const uint32_t m = n > nz ? n : nz;
  if (m == 0) return cudaSuccess;
  const uint32_t blocks = (m + kThreads - 1) / kThreads < 32u ? (m + kThreads - 1) / kThreads : 32u;
  copy_u4_kernel<<<blocks, kThreads, 0, st>>>(static_cast<const uint4*>(src), static_cast<uint4*>(dst), n,
                                              static_cast<uint4*>(zero), nz);
  return cudaGetLastError();
}

cudaError_t launch_fill_splitmix(void* dst, uint64_t words, uint64_t seed, uint64_t word0, int sms, cudaStream_t st) {
  if (words == 0) return cudaSuccess;
  uint64_t blocks = (words + 255) / 256;
  const uint64_t cap = (uint64_t)sms * 16;
  if (blocks > cap) blocks = cap;
  fill_splitmix_kernel<<<(unsigned)blocks, 256, 0, st>>>(reinterpret_cast<uint2*>(dst), words, seed, word0);
  return cudaGetLastError();
}

cudaError_t launch_xor_rows(void* table, uint32_t V, const uint64_t* idx, const void* diffs,
                            uint64_t n, int sms, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  uint64_t blocks = (n * V + 255) / 256;
  const uint64_t cap = (uint64_t)sms * 16;
  if (blocks > cap) blocks = cap;
  xor_rows_kernel<<<(unsigned)blocks, 256, 0, st>>>(reinterpret_cast<uint4*>(table), V, idx,
                                                     reinterpret_cast<const uint4*>(diffs), n);
  return cudaGetLastError();
}

cudaError_t launch_eval_points(const KeyDev* key, const uint64_t* idx, uint64_t n, void* out, int sms,
                               cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  uint64_t blocks = (n + 127) / 128;
  const uint64_t cap = (uint64_t)sms * 8;
  if (blocks > cap) blocks = cap;
  eval_points_kernel<<<(unsigned)blocks, 128, 0, st>>>(key, idx, n, reinterpret_cast<uint4*>(out));
  return cudaGetLastError();
}

// ---- warp-path launchers --------------------------------------------------

// Dynamic shared memory of a warp-kernel CTA of nw warps: per warp, G keys'
// leaf-mask exchange buffers and depth-first stacks.
size_t warp_smem_bytes(int G, uint32_t VT, uint32_t slots, uint32_t nw) {
  (void)VT;
  return (size_t)nw * G * (64 * 16 + (size_t)slots * 32 * 17);
}

bool warp_vt_supported(uint32_t V) { return V == 1 || V == 2 || V == 4 || V == 8 || V == 16 || V == 32; }

template <int G, int VT>
static cudaError_t warp_prepare_t(size_t smem) {
  return raise_smem_limit(reinterpret_cast<const void*>(scan_warp_kernel<G, VT>), smem);
}
template <int G, int VT>
static int warp_occupancy_t(size_t smem, uint32_t nw) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, scan_warp_kernel<G, VT>, (int)(nw * 32), smem) != cudaSuccess)
    return 0;
  return n;
}
template <int G, int VT>
static cudaError_t warp_launch_t(const WarpScanParams& p, uint32_t grid, uint32_t nw, size_t smem, cudaStream_t st) {
  scan_warp_kernel<G, VT><<<grid, nw * 32, smem, st>>>(p);
  return cudaGetLastError();
}

#define MG_VT_DISPATCH(G_, VT_, FN, ...)                \
  switch (VT_) {                                        \
    case 1: return FN<G_, 1>(__VA_ARGS__);              \
    case 2: return FN<G_, 2>(__VA_ARGS__);              \
    case 4: return FN<G_, 4>(__VA_ARGS__);              \
    case 8: return FN<G_, 8>(__VA_ARGS__);              \
    case 16: return FN<G_, 16>(__VA_ARGS__);            \
    case 32: return FN<G_, 32>(__VA_ARGS__);            \
    default: break;                                     \
  }

#define MG_GVT_DISPATCH(G, VT, FN, FAIL, ...)                 \
  switch (G) {                                                \
    case 1: MG_VT_DISPATCH(1, VT, FN, __VA_ARGS__) break;     \
    case 2: MG_VT_DISPATCH(2, VT, FN, __VA_ARGS__) break;     \
    case 3: MG_VT_DISPATCH(3, VT, FN, __VA_ARGS__) break;     \
    case 4: MG_VT_DISPATCH(4, VT, FN, __VA_ARGS__) break;     \
    default: break;                                           \
  }                                                           \
  return FAIL;

bool warp_g_supported(int G) { return G >= 1 && G <= 4; }

cudaError_t warp_prepare(int G, uint32_t VT, size_t smem) {
  MG_GVT_DISPATCH(G, VT, warp_prepare_t, cudaErrorInvalidValue, smem)
}
int warp_occupancy(int G, uint32_t VT, size_t smem, uint32_t nw) {
  MG_GVT_DISPATCH(G, VT, warp_occupancy_t, 0, smem, nw)
}
cudaError_t launch_scan_warp(int G, uint32_t VT, const WarpScanParams& p, uint32_t grid, uint32_t nw, size_t smem,
                             cudaStream_t st) {
  MG_GVT_DISPATCH(G, VT, warp_launch_t, cudaErrorInvalidValue, p, grid, nw, smem, st)
}

cudaError_t launch_delta(const KeyDev* keys, const uint2* jobs, uint32_t njobs, const uint64_t* idx,
                         const void* diffs, const uint32_t* count, uint32_t capacity, uint32_t V, uint64_t first,
                         uint4* out, cudaStream_t st) {
  if (njobs == 0 || capacity == 0) return cudaSuccess;
  dim3 grid((capacity + kThreads - 1) / kThreads, njobs);
  delta_kernel<<<grid, kThreads, 0, st>>>(keys, jobs, idx, reinterpret_cast<const uint4*>(diffs), count, V, first,
                                          out);
  return cudaGetLastError();
}

cudaError_t launch_frontier(const FrontierStep& f, uint32_t nkeys, cudaStream_t st) {
  if (f.n_in == 0 || nkeys == 0) return cudaSuccess;
  if (f.per == 0 || ((uint64_t)f.per << f.c) > (1ull << kFrontierLevels)) return cudaErrorInvalidValue;
  if (f.walk && (f.per != 1 || f.L_in >= (uint32_t)kMaxLevels)) return cudaErrorInvalidValue;
  dim3 grid((unsigned)((f.n_in + f.per - 1) / f.per), nkeys);
  frontier_kernel<<<grid, kThreads, 0, st>>>(f);
  return cudaGetLastError();
}

}  // namespace mg
