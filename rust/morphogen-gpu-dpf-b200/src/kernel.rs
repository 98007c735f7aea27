//! GpuScanner with the reference's entry points
//! (crates/morphogen-gpu-dpf/src/kernel.rs:156-1240), each a pass of the
//! sm_100a library: keys parsed and planned by mg_batch_set_keys, scan and
//! reduction kernels launched on the workspace's stream (or replayed from a
//! CUDA graph), shares read back.  The reference's kernel variants
//! (baseline, "optimized" v1/v2/v3, transposed) all map to the one scan
//! here; its v2/v3 kernels do not produce page shares, this path always does.
use std::os::raw::c_void;
use std::sync::atomic::{AtomicUsize, Ordering};
use std::sync::{Arc, Mutex};
use std::time::Instant;

use crate::device::{check, DriverError, GpuDevice};
use crate::dpf::{ChaChaKey, Seed128};
use crate::ffi;
use crate::storage::GpuPageMatrix;

pub use crate::storage::PAGE_SIZE_BYTES;
pub const SUBTREE_SIZE: usize = 2048;
pub const THREADS_PER_BLOCK: usize = 256;
/// Depth evaluated in full on the device (the reference kernel: 25).
pub const MAX_DOMAIN_BITS: usize = 32;
pub const MAX_KERNEL_BATCH_SIZE: usize = 16;
pub const DEFAULT_WORKSPACE_POOL_SIZE: usize = 4;
pub const MAX_WORKSPACE_POOL_SIZE: usize = 8;
pub const GPU_WORKSPACE_POOL_SIZE_ENV: &str = "MORPHOGEN_GPU_WORKSPACE_POOL_SIZE";
pub const KEYS_PER_QUERY: usize = 3;
pub const VERIF_BYTES_PER_KEY: usize = 16;

/// kernel.rs:61-66.
pub fn parse_workspace_pool_size(raw: Option<&str>) -> usize {
    raw.and_then(|v| v.parse::<usize>().ok())
        .filter(|v| *v > 0)
        .map(|v| v.min(MAX_WORKSPACE_POOL_SIZE))
        .unwrap_or(DEFAULT_WORKSPACE_POOL_SIZE)
}

/// kernel.rs:69-72.
pub fn select_workspace_pool_slot(ticket: usize, pool_size: usize) -> usize {
    debug_assert!(pool_size > 0);
    ticket % pool_size
}

/// kernel.rs:75-77.
pub fn clamp_tiled_launch_limit(tile_size: usize) -> usize {
    tile_size.clamp(1, MAX_KERNEL_BATCH_SIZE)
}

/// kernel.rs:80-93: the largest of 16/8/4/2/1 not above the remaining queries.
pub fn select_tiled_launch_batch_size(remaining_queries: usize, tile_size: usize) -> usize {
    let capped = remaining_queries.min(clamp_tiled_launch_limit(tile_size));
    [16, 8, 4, 2].iter().copied().find(|b| capped >= *b).unwrap_or(1)
}

/// kernel.rs:96-105.
pub fn plan_tiled_launch_batch_sizes(total_queries: usize, tile_size: usize) -> Vec<usize> {
    let mut remaining = total_queries;
    let mut plan = Vec::new();
    while remaining > 0 {
        let launch = select_tiled_launch_batch_size(remaining, tile_size);
        plan.push(launch);
        remaining -= launch;
    }
    plan
}

/// kernel.rs:1214-1228 (per-query averages in nanoseconds).
#[derive(Debug, Clone, Default)]
pub struct KernelTiming {
    pub dpf_eval_ns: u64,
    pub xor_accumulate_ns: u64,
    pub h2d_ns: u64,
    pub kernel_ns: u64,
    pub d2h_ns: u64,
    pub total_ns: u64,
}

/// kernel.rs:1231-1240: one share per Cuckoo key.  The verif fields are the
/// reference's Binius outputs, all zero there too (ENABLE_BINIUS is off).
#[derive(Debug, Clone)]
pub struct PirResult {
    pub page0: Vec<u8>,
    pub page1: Vec<u8>,
    pub page2: Vec<u8>,
    pub verif0: Vec<u8>,
    pub verif1: Vec<u8>,
    pub verif2: Vec<u8>,
    pub timing: KernelTiming,
}

impl PirResult {
    fn from_shares(mut shares: Vec<Vec<u8>>, timing: KernelTiming) -> Self {
        let page2 = shares.pop().unwrap_or_default();
        let page1 = shares.pop().unwrap_or_default();
        let page0 = shares.pop().unwrap_or_default();
        let z = vec![0u8; VERIF_BYTES_PER_KEY];
        Self { page0, page1, page2, verif0: z.clone(), verif1: z.clone(), verif2: z, timing }
    }
}

/// One mg_batch: device key buffer, partial rows, shares, stream, graph.
struct Workspace {
    raw: *mut ffi::mg_batch,
}

unsafe impl Send for Workspace {}

impl Workspace {
    fn new(device: &GpuDevice) -> Result<Self, DriverError> {
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::mg_batch_create(device.raw(), &mut raw) })?;
        Ok(Self { raw })
    }

    /// Parse, plan and stage one pass: key i over tables[i].
    fn set_keys(&mut self, tables: &[*const ffi::mg_table], keys: &[Vec<u8>]) -> Result<(), DriverError> {
        let ptrs: Vec<*const u8> = keys.iter().map(|k| k.as_ptr()).collect();
        let lens: Vec<usize> = keys.iter().map(|k| k.len()).collect();
        check(unsafe { ffi::mg_batch_set_keys(self.raw, tables.as_ptr(), ptrs.as_ptr(), lens.as_ptr(), keys.len() as u32) })
    }

    fn launch(&mut self, graph: bool) -> Result<(), DriverError> {
        let stream: *mut c_void = std::ptr::null_mut();
        check(unsafe {
            if graph {
                ffi::mg_batch_launch_graph(self.raw, stream)
            } else {
                ffi::mg_batch_launch(self.raw, stream)
            }
        })
    }

    /// Shares of the last pass, split by the tables' row sizes.
    fn read(&mut self, row_bytes: &[usize]) -> Result<Vec<Vec<u8>>, DriverError> {
        let total: usize = row_bytes.iter().sum();
        let mut out = vec![0u8; total];
        check(unsafe { ffi::mg_batch_read(self.raw, out.as_mut_ptr(), std::ptr::null_mut()) })?;
        let mut res = Vec::with_capacity(row_bytes.len());
        let mut off = 0;
        for rb in row_bytes {
            res.push(out[off..off + rb].to_vec());
            off += rb;
        }
        Ok(res)
    }

    fn last_kernel_ns(&mut self) -> u64 {
        let mut ns = 0u64;
        unsafe {
            ffi::mg_batch_last_kernel_ns(self.raw, &mut ns);
        }
        ns
    }

    fn run(&mut self, tables: &[*const ffi::mg_table], keys: &[Vec<u8>], row_bytes: &[usize], graph: bool)
        -> Result<(Vec<Vec<u8>>, u64), DriverError> {
        self.set_keys(tables, keys)?;
        self.launch(graph)?;
        let shares = self.read(row_bytes)?;
        Ok((shares, self.last_kernel_ns()))
    }
}

impl Drop for Workspace {
    fn drop(&mut self) {
        unsafe {
            ffi::mg_batch_destroy(self.raw);
        }
    }
}

/// kernel.rs:156-171 / 258-465.
pub struct GpuScanner {
    pub device: Arc<GpuDevice>,
    batch_workspace_pool: Vec<Mutex<Option<Workspace>>>,
    next_workspace_slot: AtomicUsize,
}

fn flatten(queries: &[[ChaChaKey; 3]]) -> Vec<Vec<u8>> {
    queries.iter().flat_map(|q| q.iter().map(|k| k.to_bytes())).collect()
}

impl GpuScanner {
    pub fn new(device_ord: usize) -> Result<Self, DriverError> {
        let device = GpuDevice::new(device_ord)?;
        let pool = parse_workspace_pool_size(std::env::var(GPU_WORKSPACE_POOL_SIZE_ENV).ok().as_deref());
        Ok(Self {
            device,
            batch_workspace_pool: (0..pool).map(|_| Mutex::new(None)).collect(),
            next_workspace_slot: AtomicUsize::new(0),
        })
    }

    /// kernel.rs:927-935.
    pub unsafe fn scan(&self, db: &GpuPageMatrix, keys: [&ChaChaKey; 3]) -> Result<PirResult, DriverError> {
        let query = [keys[0].clone(), keys[1].clone(), keys[2].clone()];
        Ok(self.scan_batch(db, &[query])?.into_iter().next().unwrap())
    }

    /// kernel.rs:685-700.
    pub unsafe fn scan_batch(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]])
        -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_opts(db, queries, false, false, false, false, false, MAX_KERNEL_BATCH_SIZE)
    }

    /// kernel.rs:711-924: passes of at most `max_tile_size` queries from the
    /// workspace pool (ticket % pool, as there); optional CUDA-graph replay.
    /// The kernel-variant flags select reference kernels and have no effect.
    #[allow(clippy::too_many_arguments)]
    pub unsafe fn scan_batch_opts(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]], _transposed: bool,
                                  _optimized: bool, _optimized_v2: bool, _optimized_v3: bool, use_cuda_graph: bool,
                                  max_tile_size: usize) -> Result<Vec<PirResult>, DriverError> {
        if queries.is_empty() {
            return Ok(Vec::new());
        }
        let start = Instant::now();
        let ticket = self.next_workspace_slot.fetch_add(1, Ordering::Relaxed);
        let slot = &self.batch_workspace_pool[select_workspace_pool_slot(ticket, self.batch_workspace_pool.len())];
        let mut guard = slot.lock().unwrap();
        if guard.is_none() {
            *guard = Some(Workspace::new(&self.device)?);
        }
        let ws = guard.as_mut().unwrap();
        let mut results = Vec::with_capacity(queries.len());
        let mut kernel_ns = 0u64;
        let mut done = 0;
        for q in plan_tiled_launch_batch_sizes(queries.len(), max_tile_size) {
            let keys = flatten(&queries[done..done + q]);
            let tables = vec![db.raw(); keys.len()];
            let sizes = vec![db.row_bytes(); keys.len()];
            let (shares, ns) = ws.run(&tables, &keys, &sizes, use_cuda_graph)?;
            kernel_ns += ns;
            let mut it = shares.into_iter();
            for _ in 0..q {
                let three: Vec<Vec<u8>> = (0..3).map(|_| it.next().unwrap()).collect();
                results.push(PirResult::from_shares(three, KernelTiming::default()));
            }
            done += q;
        }
        let n = queries.len() as u64;
        let total = start.elapsed().as_nanos() as u64;
        for r in results.iter_mut() {
            r.timing = KernelTiming { dpf_eval_ns: kernel_ns / n, kernel_ns: kernel_ns / n, total_ns: total / n,
                                      ..Default::default() };
        }
        Ok(results)
    }

    /// kernel.rs:940-953.
    pub unsafe fn scan_batch_single_query_multistream_optimized(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]],
                                                                stream_count: usize)
        -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_single_query_multistream_optimized_with_graph(db, queries, stream_count, false)
    }

    /// kernel.rs:955-1097: one pass per query, round-robin over
    /// `stream_count` workspaces whose streams overlap on the device.
    pub unsafe fn scan_batch_single_query_multistream_optimized_with_graph(
        &self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]], stream_count: usize, use_cuda_graph: bool,
    ) -> Result<Vec<PirResult>, DriverError> {
        let streams = stream_count.max(1).min(queries.len().max(1));
        if streams <= 1 {
            return self.scan_batch_opts(db, queries, false, true, false, false, use_cuda_graph, MAX_KERNEL_BATCH_SIZE);
        }
        let mut wss = (0..streams).map(|_| Workspace::new(&self.device)).collect::<Result<Vec<_>, _>>()?;
        let tables = vec![db.raw(); 3];
        let sizes = vec![db.row_bytes(); 3];
        let mut out = Vec::with_capacity(queries.len());
        for chunk in queries.chunks(streams) {
            for (ws, q) in wss.iter_mut().zip(chunk.iter()) {
                ws.set_keys(&tables, &flatten(std::slice::from_ref(q)))?;
                ws.launch(use_cuda_graph)?;
            }
            for ws in wss.iter_mut().take(chunk.len()) {
                let shares = ws.read(&sizes)?;
                let ns = ws.last_kernel_ns();
                out.push(PirResult::from_shares(shares, KernelTiming { dpf_eval_ns: ns, kernel_ns: ns,
                                                                       ..Default::default() }));
            }
        }
        Ok(out)
    }

    /// kernel.rs:1105-1112.
    pub unsafe fn scan_batch_optimized(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]])
        -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_optimized_with_graph(db, queries, false)
    }

    /// kernel.rs:1114-1132.
    pub unsafe fn scan_batch_optimized_with_graph(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]],
                                                  use_cuda_graph: bool) -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_opts(db, queries, false, true, false, false, use_cuda_graph, MAX_KERNEL_BATCH_SIZE)
    }

    /// kernel.rs:1135-1143.
    pub unsafe fn scan_batch_optimized_tiled(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]], tile_size: usize)
        -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_optimized_tiled_with_graph(db, queries, tile_size, false)
    }

    /// kernel.rs:1145-1162.
    pub unsafe fn scan_batch_optimized_tiled_with_graph(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]],
                                                        tile_size: usize, use_cuda_graph: bool)
        -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_opts(db, queries, false, true, false, false, use_cuda_graph, tile_size)
    }

    /// kernel.rs:1171-1193 (the reference's v2 kernel gives no page share;
    /// this runs the same scan as every other entry point).
    pub unsafe fn scan_batch_optimized_v2(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]])
        -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_opts(db, queries, false, true, true, false, false, MAX_KERNEL_BATCH_SIZE)
    }

    /// kernel.rs:1195-1210 (as v2).
    pub unsafe fn scan_batch_optimized_v3(&self, db: &GpuPageMatrix, queries: &[[ChaChaKey; 3]])
        -> Result<Vec<PirResult>, DriverError> {
        self.scan_batch_opts(db, queries, false, true, false, true, false, MAX_KERNEL_BATCH_SIZE)
    }

    /// Mixed-size batching: any (table, key) pairs over several resident
    /// tables in one pass; one share per pair.
    pub unsafe fn scan_multi(&self, items: &[(&GpuPageMatrix, &ChaChaKey)]) -> Result<Vec<Vec<u8>>, DriverError> {
        if items.is_empty() {
            return Ok(Vec::new());
        }
        let tables: Vec<*const ffi::mg_table> = items.iter().map(|(t, _)| t.raw()).collect();
        let keys: Vec<Vec<u8>> = items.iter().map(|(_, k)| k.to_bytes()).collect();
        let sizes: Vec<usize> = items.iter().map(|(t, _)| t.row_bytes()).collect();
        let mut ws = Workspace::new(&self.device)?;
        Ok(ws.run(&tables, &keys, &sizes, false)?.0)
    }

    /// ChaChaKey::eval (dpf.rs:103-142) at each index, on the device (the
    /// point evaluations of scan_delta_for_gpu, scan.rs:434-485).
    pub fn eval_points(&self, key: &ChaChaKey, indices: &[u64]) -> Result<Vec<Seed128>, DriverError> {
        let kb = key.to_bytes();
        let mut out = vec![0u8; indices.len() * 16];
        check(unsafe {
            ffi::mg_eval_points(self.device.raw(), kb.as_ptr(), kb.len(), indices.as_ptr(), indices.len() as u64,
                                out.as_mut_ptr())
        })?;
        Ok(out.chunks(16).map(|c| {
            let mut b = [0u8; 16];
            b.copy_from_slice(c);
            Seed128::from_bytes(&b)
        }).collect())
    }
}

#[cfg(test)]
mod tests {
    use super::*;

    #[test]
    fn workspace_pool_size_parsing() {
        assert_eq!(parse_workspace_pool_size(None), DEFAULT_WORKSPACE_POOL_SIZE);
        assert_eq!(parse_workspace_pool_size(Some("0")), DEFAULT_WORKSPACE_POOL_SIZE);
        assert_eq!(parse_workspace_pool_size(Some("3")), 3);
        assert_eq!(parse_workspace_pool_size(Some("99")), MAX_WORKSPACE_POOL_SIZE);
        assert_eq!(parse_workspace_pool_size(Some("x")), DEFAULT_WORKSPACE_POOL_SIZE);
    }

    #[test]
    fn tiled_plan() {
        assert_eq!(plan_tiled_launch_batch_sizes(7, 16), vec![4, 2, 1]);
        assert_eq!(plan_tiled_launch_batch_sizes(20, 16), vec![16, 4]);
        assert_eq!(plan_tiled_launch_batch_sizes(5, 2), vec![2, 2, 1]);
    }
}
