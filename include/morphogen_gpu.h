/*
 * morphogen_gpu.h -- C ABI of the B200 (sm_100a) per-server PIR answer path.
 *
 * One server holds a table of `rows` rows of `row_bytes` bytes (row_bytes a
 * multiple of 16, at most 4096) resident in HBM.  A query key is a ChaCha8
 * GGM DPF key share in the reference's unchanged wire format
 * (ChaChaKey::to_bytes, crates/morphogen-gpu-dpf/src/dpf.rs:259-274).  The
 * server's answer share for a key is
 *
 *     share = XOR_{i < rows} ( row_i AND mask(i) ),  mask(i) = key.eval(i)
 *
 * with the 16-byte DPF output repeated over every 16-byte lane of the row
 * (crates/morphogen-gpu-dpf/src/kernel.rs:1243-1256, generalised from 4096-B
 * pages to R-byte rows; the reference's page mode is row_bytes = 4096).
 *
 * All entry points use C linkage, plain pointers and sizes, return an int
 * status (MG_OK == 0) and never throw.  mg_last_error() returns a
 * thread-local message for the last failing call on the calling thread.
 * A context may be used from several host threads: calls on one context are
 * serialised internally; distinct mg_batch workspaces may be driven from
 * different threads and overlap on the device through their own streams.
 */
#ifndef MORPHOGEN_GPU_H
#define MORPHOGEN_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference surfaces DriverError (mapped to HTTP 500) and
 * GpuDpfError (crates/morphogen-gpu-dpf/src/dpf.rs:9-15). */
enum {
  MG_OK = 0,
  MG_EINVAL = 1,    /* bad argument (null pointer, row_bytes % 16 != 0, ...)    */
  MG_EKEY = 2,      /* malformed key bytes: GpuDpfError::InvalidKeyFormat       */
  MG_ERANGE = 3,    /* index beyond the DPF domain: PageIndexTooLarge, or more
                       rows than 2^domain_bits (kernel.rs:1283-1285)             */
  MG_ENOMEM = 4,    /* device or pinned-host allocation failed                  */
  MG_ECUDA = 5,     /* CUDA runtime error: DriverError                          */
  MG_ETIMEDOUT = 6, /* the pass did not complete before the caller's deadline   */
  MG_ENODEV = 7,    /* no usable sm_100 device                                  */
  MG_EBUSY = 8      /* workspace still owns a pass in flight                    */
};

/* Largest DPF depth the device path accepts.  ChaChaParams::new allows up to
 * 32 levels (dpf.rs:65-79); the reference kernel silently truncates at 25
 * (kernel.rs:45,131-136), this library evaluates all 32. */
#define MG_MAX_DOMAIN_BITS 32
#define MG_MAX_ROW_BYTES 4096

typedef struct mg_context mg_context; /* GpuScanner                      */
typedef struct mg_table mg_table;     /* GpuPageMatrix with R-byte rows  */
typedef struct mg_batch mg_batch;     /* BatchWorkspace (kernel.rs:163-171) */

/* KernelTiming (kernel.rs:1214-1228); whole-pass figures in nanoseconds. */
typedef struct {
  uint64_t h2d_ns;
  uint64_t kernel_ns; /* CUDA-event time of the scan + reduction kernels */
  uint64_t d2h_ns;
  uint64_t total_ns;
} mg_timing;

/* Scan kernels.  CTA: a CTA expands a 2^S-row tile (breadth-first in shared
 * memory, then one depth-first walk per thread); any row size.  WARP: a
 * frontier of tree nodes is computed breadth-first up front and every warp
 * walks 32 x 2^M rows on its own; rows of 16..512 B (power of two). */
enum { MG_KERNEL_AUTO = 0, MG_KERNEL_CTA = 1, MG_KERNEL_WARP = 2 };

/* Launch shape chosen for a pass (first launch; subtree_bits over all). */
typedef struct {
  uint32_t subtree_bits;   /* rows per work item = 2^subtree_bits (CTA: S; warp: M + 5) */
  uint32_t keys_per_cta;   /* keys evaluated together on one work item */
  uint32_t grid;           /* persistent CTAs launched */
  uint32_t items;          /* (tile, key group) work items */
  uint32_t segments;       /* (table, domain) segments in the pass */
  uint32_t smem_bytes;     /* dynamic shared memory per CTA */
  uint32_t kernel;         /* MG_KERNEL_CTA or MG_KERNEL_WARP */
  uint32_t frontier_nodes; /* frontier nodes held for the warp kernel */
  uint32_t kernels;        /* kernel launches per pass (frontier chain, scans, reductions) */
} mg_plan_info;

/* ---- context: GpuScanner::new (kernel.rs:258-465) ------------------------ */
int mg_context_create(int device, mg_context** out);
int mg_context_destroy(mg_context* ctx);
const char* mg_last_error(void);
/* SM count and free/total device memory (admission control). */
int mg_device_info(mg_context* ctx, int* sm_count, uint64_t* free_bytes, uint64_t* total_bytes);

/* ---- tables: GpuPageMatrix (crates/morphogen-gpu-dpf/src/storage.rs) ------ */
/* alloc_empty (storage.rs:89-101): zero-filled rows x row_bytes on the device. */
int mg_table_create(mg_context* ctx, uint64_t rows, uint32_t row_bytes, mg_table** out);
/* A table holding rows [first_row, first_row + rows) of a larger logical
 * table: keys are evaluated at the logical row indices, so the shares of the
 * range tables that partition a table XOR to the share of the whole table
 * (sharding one table over several GPUs: per-GPU shares, then one XOR).  The
 * reference only times this layout (crates/morphogen-gpu-dpf/src/bin/
 * bench_sharded.rs:14-110: a page-range per GPU, scanned from page 0, no
 * combine); here each range answers at its own logical rows. */
int mg_table_create_range(mg_context* ctx, uint64_t first_row, uint64_t rows, uint32_t row_bytes,
                          mg_table** out);
uint64_t mg_table_first_row(const mg_table* table);
int mg_table_destroy(mg_table* table);
/* update_pages (storage.rs:104-124) / new (storage.rs:27-43): host -> device. */
int mg_table_write_rows(mg_table* table, uint64_t first_row, const void* host_rows, uint64_t nrows);
int mg_table_read_rows(const mg_table* table, uint64_t first_row, void* host_rows, uint64_t nrows);
/* Synthetic content: logical byte o (row-range tables start at first_row *
 * row_bytes) = byte (o % 8) of SplitMix64 output o / 8 of the stream seeded
 * with `seed`; generated on the device. */
int mg_table_fill_splitmix(mg_table* table, uint64_t seed);
/* Epoch merge: row_idx[i] ^= diffs[i] for n entries, in place on the device
 * (the GPU half of EpochManager::try_advance, server/epoch.rs:516-545, and
 * the XOR patch of try_build_snapshot_from_entries, server/epoch.rs:118-181).
 * Host arrays; row indices must be < rows. */
int mg_table_xor_rows(mg_table* table, const uint64_t* row_idx, const void* diffs, uint64_t n);
/* ---- epoch delta: DeltaBuffer + scan_delta_for_gpu + epoch merge --------- */
/* A table may hold a device-resident buffer of pending row updates
 * (crates/morphogen-core/src/delta.rs: DeltaEntry{row_idx, diff}).  Every
 * pass over the table folds the pending entries into each key's share:
 * share ^= XOR_e diff_e & eval(row_e) (scan_delta_for_gpu,
 * crates/morphogen-server/src/scan.rs:434-485, in row mode), so answers
 * reflect table XOR delta without touching the table.  mg_table_delta_merge
 * XOR-patches the table with the entries, clears the buffer and advances the
 * epoch (the merge of EpochManager::try_advance,
 * crates/morphogen-server/src/epoch.rs:465-549).  Merge and clear wait for
 * every pass already enqueued on the device; the caller must not enqueue a
 * pass over the table while they run (the reference's matrix lock). */
int mg_table_delta_reserve(mg_table* table, uint32_t capacity);
/* DeltaBuffer::push: append n entries (host arrays, diffs n x row_bytes).
 * MG_ERANGE when the buffer is full or a row index is outside the table. */
int mg_table_delta_push(mg_table* table, const uint64_t* row_idx, const void* diffs, uint32_t n);
uint32_t mg_table_delta_count(const mg_table* table);
int mg_table_delta_clear(mg_table* table);
int mg_table_delta_merge(mg_table* table);
uint64_t mg_table_epoch(const mg_table* table);
uint64_t mg_table_rows(const mg_table* table);
uint32_t mg_table_row_bytes(const mg_table* table);
const void* mg_table_device_ptr(const mg_table* table);

/* ---- keys: ChaChaKey (crates/morphogen-gpu-dpf/src/dpf.rs) ---------------- */
/* Wire length 19 + 18 d + 16 (dpf.rs:287). */
size_t mg_key_size(uint32_t domain_bits);
/* ChaChaKey::from_bytes validation (dpf.rs:277-316) plus d <= 32. */
int mg_key_check(const uint8_t* key, size_t len, uint32_t* domain_bits, uint8_t* party);
/* generate_chacha_dpf_keys (dpf.rs:322-432) with caller-supplied root seeds
 * (the reference draws them from rand::random, dpf.rs:332-333).  key0/key1
 * must each hold mg_key_size(domain_bits) bytes. */
int mg_keygen(uint32_t domain_bits, uint64_t target, const uint8_t root_seed0[16],
              const uint8_t root_seed1[16], uint8_t* key0, uint8_t* key1);

/* ---- one-call scan: GpuScanner::scan / scan_batch (kernel.rs:685-935) ----- */
/* Evaluates nkeys keys in one pass; key i is scanned over tables[i] (tables
 * may repeat and may differ: mixed-size batching).  out_shares receives the
 * shares back to back, share i being row_bytes(tables[i]) bytes.  Keys and
 * shares are host memory; the copies are inside the call.  timeout_ms == 0
 * waits without a deadline; otherwise MG_ETIMEDOUT is returned if the pass
 * has not finished in time (the pass still completes on the device; the
 * context's internal workspace stays busy until it does).  timing may be NULL.
 * A call with the same tables, key depths and shape as the previous call on
 * the context reuses its plan and replays one CUDA graph holding the key
 * upload, the pass and the share download (the first such call captures it);
 * its timing reports that graph's device time as kernel_ns and d2h_ns = 0. */
int mg_scan(mg_context* ctx, const mg_table* const* tables, const uint8_t* const* keys,
            const size_t* key_lens, uint32_t nkeys, uint8_t* out_shares, uint32_t timeout_ms,
            mg_timing* timing);

/* ---- workspaces: BatchWorkspace + scan_batch_opts (kernel.rs:163-171,711-924) */
int mg_batch_create(mg_context* ctx, mg_batch** out);
int mg_batch_destroy(mg_batch* batch);
/* Parse and stage keys, plan the pass, copy the keys to the device on the
 * workspace stream.  Reallocates device buffers only when they grow. */
int mg_batch_set_keys(mg_batch* batch, const mg_table* const* tables, const uint8_t* const* keys,
                      const size_t* key_lens, uint32_t nkeys);
/* Pin the launch shape (0 = let the planner choose). */
int mg_batch_set_shape(mg_batch* batch, uint32_t subtree_bits, uint32_t keys_per_cta);
/* Choose the scan kernel (MG_KERNEL_AUTO by default). */
int mg_batch_set_kernel(mg_batch* batch, int kind);
/* Autotuner: with keys set, time candidate launch shapes (both kernels, work
 * item depth, keys per item) on the device for up to budget_ms (0 = all),
 * check that every shape gives identical shares, keep the fastest for this
 * workload (rows, row size, depth, key count of every segment) in the
 * context -- later passes with the same signature use it unless a shape is
 * pinned -- and re-plan this workspace with it.  best/best_ms may be NULL. */
int mg_batch_autotune(mg_batch* batch, uint32_t budget_ms, mg_plan_info* best, double* best_ms);
/* Enqueue the scan and reduction kernels on `stream` (a cudaStream_t; NULL =
 * the workspace's own stream).  Keys and tables must already be resident.
 * Launch-only: capturable into a CUDA graph by the caller. */
int mg_batch_launch(mg_batch* batch, void* stream);
/* Replay the pass from a CUDA graph captured on first use (same keys layout). */
int mg_batch_launch_graph(mg_batch* batch, void* stream);
/* Device -> host copy of the shares (enqueued on the stream; see mg_batch_sync). */
int mg_batch_read(mg_batch* batch, uint8_t* out_shares, void* stream);
/* Wait for the workspace stream with a deadline (0 = none). */
int mg_batch_sync(mg_batch* batch, uint32_t timeout_ms);
int mg_batch_shares_device(mg_batch* batch, const void** dptr, size_t* bytes);
int mg_batch_plan(mg_batch* batch, mg_plan_info* info);
/* Timing of the last launch on the workspace stream: scan + reduction
 * kernels, and the scan kernels alone (a graph replay is timed as a whole). */
int mg_batch_last_kernel_ns(mg_batch* batch, uint64_t* ns);
int mg_batch_last_scan_ns(mg_batch* batch, uint64_t* ns);

/* ---- measurement (no counterpart in the reference) ------------------------ */
/* ChaCha8 node expansions per second of the device PRG alone (no memory
 * traffic, full occupancy): the integer-ALU ceiling of the scan kernel. */
int mg_prg_peak(mg_context* ctx, uint32_t iters, double* expands_per_s);

/* ---- point evaluation on the device: ChaChaKey::eval (dpf.rs:103-142) ----- */
/* out: n * 16 bytes, out[i] = eval(idx[i]).  Host arrays. */
int mg_eval_points(mg_context* ctx, const uint8_t* key, size_t key_len, const uint64_t* idx,
                   uint64_t n, uint8_t* out);

/* ---- serving loop: continuous batching (network/api/mod.rs:544-838) ------- */
/* A dispatcher thread owns `slots` workspaces (one stream each).  Whenever
 * one is free it folds every request that has arrived into one pass, so
 * requests that arrive while others are on the GPU join the next pass and
 * passes of different workspaces overlap on the device.  A request is
 * admitted when the device memory its keys, frontier and partial rows need
 * fits in free memory minus memory_reserve (or when nothing else runs).
 * Tables and their delta buffers stay resident; for an epoch merge call
 * mg_server_pause (drains in-flight passes), mg_table_delta_merge, then
 * mg_server_resume. */
typedef struct {
  uint32_t slots;             /* concurrent passes (default 2) */
  uint32_t max_keys_per_pass; /* 0 = latency-aware: a pass is closed once its
                                 estimated device time (tree nodes of its keys
                                 over the rate measured on completed passes)
                                 reaches 50 ms; always at least one request */
  uint64_t memory_reserve;    /* device bytes kept free (default 1 GiB) */
} mg_server_config;

typedef struct {
  uint64_t completed;       /* requests answered */
  uint64_t failed;
  uint64_t passes;
  uint64_t keys_completed;  /* keys (DPF evaluations) answered */
  uint32_t pending;         /* requests waiting for a pass */
  uint32_t in_flight;       /* passes on the GPU */
  double wall_s;            /* since create / reset */
  double p50_ms, p95_ms, p99_ms, mean_ms, max_ms;  /* submit -> answered */
} mg_server_stats;

typedef struct mg_server mg_server;
int mg_server_create(mg_context* ctx, const mg_server_config* cfg, mg_server** out);
/* Completes the passes already on the GPU, answers requests not yet
 * dispatched with MG_EBUSY (threads blocked in mg_server_wait wake up and
 * return it), waits for those threads to leave, then frees the server. */
int mg_server_destroy(mg_server* server);
/* Queue one request (its keys, key i over tables[i]); returns its id. */
int mg_server_submit(mg_server* server, const mg_table* const* tables, const uint8_t* const* keys,
                     const size_t* key_lens, uint32_t nkeys, uint64_t* request_id);
/* Wait for a request (0 = no deadline) and copy its shares (back to back).
 * The id is released on return, except on MG_ETIMEDOUT. */
int mg_server_wait(mg_server* server, uint64_t request_id, uint8_t* out_shares, uint32_t timeout_ms,
                   double* latency_ms);
int mg_server_pause(mg_server* server, uint32_t timeout_ms);
int mg_server_resume(mg_server* server);
int mg_server_get_stats(mg_server* server, mg_server_stats* stats);
int mg_server_reset_stats(mg_server* server);

/* ---- allocation-free scan (no counterpart in the reference) -------------- */
/* For callers that cannot call cudaMalloc: the host application or a memory
 * pool owns all device memory (plugins, embedded servers), or cudaMalloc /
 * cudaFree would block on or synchronise the device inside a latency-bound
 * serving loop.  Same result as mg_scan for the same table and keys, but no
 * device or pinned memory is allocated: the parsed keys and the per-CTA
 * partial rows live in one fixed device array of MG_NOALLOC_SCRATCH_BYTES,
 * which every GPU that loads the library holds until the process exits.
 *
 * table_dev: rows x row_bytes in device memory on `device`; out_shares_dev:
 * nkeys * row_bytes of device memory, share i at offset i * row_bytes.  Keys
 * are host bytes in the wire format and must all have the same domain_bits.
 * The work is enqueued on `stream` (a cudaStream_t, NULL = legacy default)
 * and the shares are valid once the stream reaches it.  The parsed keys go
 * to the device by value inside kernel parameters: the call does not wait
 * for the stream, and the caller may reuse its key buffers on return.
 *
 * Limits: nkeys <= MG_NOALLOC_MAX_KEYS, and nkeys * 624 bytes of keys plus
 * (persistent CTAs) x nkeys x row_bytes bytes of partial rows must fit the
 * array; otherwise MG_ERANGE with a message naming the limit.  On B200
 * (at most 592 CTAs) that is nkeys * row_bytes up to about 28 KB.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and enables the kernel's shared memory; make that
 * first call before any stream capture.  All calls on a device share the
 * array: each call clears what it needs, but calls that overlap on the GPU
 * (other streams, or host threads without ordering between them) race and
 * must be serialised by the caller. */
#define MG_NOALLOC_SCRATCH_BYTES (16u << 20)
#define MG_NOALLOC_MAX_KEYS 64
int mg_scan_noalloc(int device, const void* table_dev, uint64_t rows, uint32_t row_bytes,
                    const uint8_t* const* keys, const size_t* key_lens, uint32_t nkeys,
                    void* out_shares_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MORPHOGEN_GPU_H */
