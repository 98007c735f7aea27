//! Raw bindings of include/morphogen_gpu.h: every entry point and every
//! struct, with the header's names and C types.  The safe wrappers in the
//! other modules are what the server uses.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_int, c_void};

pub const MG_OK: c_int = 0;
pub const MG_EINVAL: c_int = 1;
pub const MG_EKEY: c_int = 2;
pub const MG_ERANGE: c_int = 3;
pub const MG_ENOMEM: c_int = 4;
pub const MG_ECUDA: c_int = 5;
pub const MG_ETIMEDOUT: c_int = 6;
pub const MG_ENODEV: c_int = 7;
pub const MG_EBUSY: c_int = 8;

pub const MG_MAX_DOMAIN_BITS: u32 = 32;
pub const MG_MAX_ROW_BYTES: u32 = 4096;
pub const MG_KERNEL_AUTO: c_int = 0;
pub const MG_KERNEL_CTA: c_int = 1;
pub const MG_KERNEL_WARP: c_int = 2;
pub const MG_NOALLOC_SCRATCH_BYTES: u32 = 16 << 20;
pub const MG_NOALLOC_MAX_KEYS: u32 = 64;

#[repr(C)]
pub struct mg_context {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct mg_table {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct mg_batch {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct mg_server {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct mg_timing {
    pub h2d_ns: u64,
    pub kernel_ns: u64,
    pub d2h_ns: u64,
    pub total_ns: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct mg_plan_info {
    pub subtree_bits: u32,
    pub keys_per_cta: u32,
    pub grid: u32,
    pub items: u32,
    pub segments: u32,
    pub smem_bytes: u32,
    pub kernel: u32,
    pub frontier_nodes: u32,
    pub kernels: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct mg_server_config {
    pub slots: u32,
    pub max_keys_per_pass: u32,
    pub memory_reserve: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct mg_server_stats {
    pub completed: u64,
    pub failed: u64,
    pub passes: u64,
    pub keys_completed: u64,
    pub pending: u32,
    pub in_flight: u32,
    pub wall_s: f64,
    pub p50_ms: f64,
    pub p95_ms: f64,
    pub p99_ms: f64,
    pub mean_ms: f64,
    pub max_ms: f64,
}

extern "C" {
    pub fn mg_context_create(device: c_int, out: *mut *mut mg_context) -> c_int;
    pub fn mg_context_destroy(ctx: *mut mg_context) -> c_int;
    pub fn mg_last_error() -> *const c_char;
    pub fn mg_device_info(ctx: *mut mg_context, sm_count: *mut c_int, free_bytes: *mut u64, total_bytes: *mut u64)
        -> c_int;

    pub fn mg_table_create(ctx: *mut mg_context, rows: u64, row_bytes: u32, out: *mut *mut mg_table) -> c_int;
    pub fn mg_table_create_range(ctx: *mut mg_context, first_row: u64, rows: u64, row_bytes: u32,
                                 out: *mut *mut mg_table) -> c_int;
    pub fn mg_table_first_row(table: *const mg_table) -> u64;
    pub fn mg_table_destroy(table: *mut mg_table) -> c_int;
    pub fn mg_table_write_rows(table: *mut mg_table, first_row: u64, host_rows: *const c_void, nrows: u64) -> c_int;
    pub fn mg_table_read_rows(table: *const mg_table, first_row: u64, host_rows: *mut c_void, nrows: u64) -> c_int;
    pub fn mg_table_fill_splitmix(table: *mut mg_table, seed: u64) -> c_int;
    pub fn mg_table_xor_rows(table: *mut mg_table, row_idx: *const u64, diffs: *const c_void, n: u64) -> c_int;
    pub fn mg_table_delta_reserve(table: *mut mg_table, capacity: u32) -> c_int;
    pub fn mg_table_delta_push(table: *mut mg_table, row_idx: *const u64, diffs: *const c_void, n: u32) -> c_int;
    pub fn mg_table_delta_count(table: *const mg_table) -> u32;
    pub fn mg_table_delta_clear(table: *mut mg_table) -> c_int;
    pub fn mg_table_delta_merge(table: *mut mg_table) -> c_int;
    pub fn mg_table_epoch(table: *const mg_table) -> u64;
    pub fn mg_table_rows(table: *const mg_table) -> u64;
    pub fn mg_table_row_bytes(table: *const mg_table) -> u32;
    pub fn mg_table_device_ptr(table: *const mg_table) -> *const c_void;

    pub fn mg_key_size(domain_bits: u32) -> usize;
    pub fn mg_key_check(key: *const u8, len: usize, domain_bits: *mut u32, party: *mut u8) -> c_int;
    pub fn mg_keygen(domain_bits: u32, target: u64, root_seed0: *const u8, root_seed1: *const u8, key0: *mut u8,
                     key1: *mut u8) -> c_int;

    pub fn mg_scan(ctx: *mut mg_context, tables: *const *const mg_table, keys: *const *const u8,
                   key_lens: *const usize, nkeys: u32, out_shares: *mut u8, timeout_ms: u32,
                   timing: *mut mg_timing) -> c_int;

    pub fn mg_batch_create(ctx: *mut mg_context, out: *mut *mut mg_batch) -> c_int;
    pub fn mg_batch_destroy(batch: *mut mg_batch) -> c_int;
    pub fn mg_batch_set_keys(batch: *mut mg_batch, tables: *const *const mg_table, keys: *const *const u8,
                             key_lens: *const usize, nkeys: u32) -> c_int;
    pub fn mg_batch_set_shape(batch: *mut mg_batch, subtree_bits: u32, keys_per_cta: u32) -> c_int;
    pub fn mg_batch_set_kernel(batch: *mut mg_batch, kind: c_int) -> c_int;
    pub fn mg_batch_autotune(batch: *mut mg_batch, budget_ms: u32, best: *mut mg_plan_info, best_ms: *mut f64)
        -> c_int;
    pub fn mg_batch_launch(batch: *mut mg_batch, stream: *mut c_void) -> c_int;
    pub fn mg_batch_launch_graph(batch: *mut mg_batch, stream: *mut c_void) -> c_int;
    pub fn mg_batch_read(batch: *mut mg_batch, out_shares: *mut u8, stream: *mut c_void) -> c_int;
    pub fn mg_batch_sync(batch: *mut mg_batch, timeout_ms: u32) -> c_int;
    pub fn mg_batch_shares_device(batch: *mut mg_batch, dptr: *mut *const c_void, bytes: *mut usize) -> c_int;
    pub fn mg_batch_plan(batch: *mut mg_batch, info: *mut mg_plan_info) -> c_int;
    pub fn mg_batch_last_kernel_ns(batch: *mut mg_batch, ns: *mut u64) -> c_int;
    pub fn mg_batch_last_scan_ns(batch: *mut mg_batch, ns: *mut u64) -> c_int;

    pub fn mg_prg_peak(ctx: *mut mg_context, iters: u32, expands_per_s: *mut f64) -> c_int;
    pub fn mg_eval_points(ctx: *mut mg_context, key: *const u8, key_len: usize, idx: *const u64, n: u64,
                          out: *mut u8) -> c_int;

    pub fn mg_server_create(ctx: *mut mg_context, cfg: *const mg_server_config, out: *mut *mut mg_server) -> c_int;
    pub fn mg_server_destroy(server: *mut mg_server) -> c_int;
    pub fn mg_server_submit(server: *mut mg_server, tables: *const *const mg_table, keys: *const *const u8,
                            key_lens: *const usize, nkeys: u32, request_id: *mut u64) -> c_int;
    pub fn mg_server_wait(server: *mut mg_server, request_id: u64, out_shares: *mut u8, timeout_ms: u32,
                          latency_ms: *mut f64) -> c_int;
    pub fn mg_server_pause(server: *mut mg_server, timeout_ms: u32) -> c_int;
    pub fn mg_server_resume(server: *mut mg_server) -> c_int;
    pub fn mg_server_get_stats(server: *mut mg_server, stats: *mut mg_server_stats) -> c_int;
    pub fn mg_server_reset_stats(server: *mut mg_server) -> c_int;

    pub fn mg_scan_noalloc(device: c_int, table_dev: *const c_void, rows: u64, row_bytes: u32,
                           keys: *const *const u8, key_lens: *const usize, nkeys: u32, out_shares_dev: *mut c_void,
                           stream: *mut c_void) -> c_int;
}

/// The calling thread's message for its last failing call.
pub fn last_error() -> String {
    unsafe {
        let p = mg_last_error();
        if p.is_null() {
            String::new()
        } else {
            std::ffi::CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    }
}
