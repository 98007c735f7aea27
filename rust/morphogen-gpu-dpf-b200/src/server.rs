//! Continuous-batching answer loop (mg_server_*): the GPU half of the
//! reference's /query/page/gpu(/batch) handlers
//! (crates/morphogen-server/src/network/api/mod.rs:544-838).  A handler
//! submits its keys and waits; requests that arrive while others are on the
//! GPU are folded into the next pass, passes of different workspaces overlap
//! on the device.  An epoch merge brackets GpuPageMatrix::delta_merge with
//! pause / resume.
use std::collections::HashMap;
use std::sync::{Arc, Mutex};

use crate::device::{check, DriverError, GpuDevice};
use crate::dpf::ChaChaKey;
use crate::ffi;
use crate::storage::GpuPageMatrix;

pub type ServerStats = ffi::mg_server_stats;

pub struct PirServer {
    _device: Arc<GpuDevice>,
    raw: *mut ffi::mg_server,
    share_bytes: Mutex<HashMap<u64, Vec<usize>>>,
}

unsafe impl Send for PirServer {}
unsafe impl Sync for PirServer {}

impl PirServer {
    /// slots: concurrent passes (0 = 2); max_keys_per_pass: 0 = passes closed
    /// at about 50 ms of measured device time; memory_reserve: device bytes
    /// kept free by admission (0 = 1 GiB).
    pub fn new(device: Arc<GpuDevice>, slots: u32, max_keys_per_pass: u32, memory_reserve: u64)
        -> Result<Self, DriverError> {
        let cfg = ffi::mg_server_config {
            slots,
            max_keys_per_pass,
            memory_reserve: if memory_reserve == 0 { 1 << 30 } else { memory_reserve },
        };
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::mg_server_create(device.raw(), &cfg, &mut raw) })?;
        Ok(Self { _device: device, raw, share_bytes: Mutex::new(HashMap::new()) })
    }

    /// Queue one request (key i over items[i].0); returns its id.
    pub fn submit(&self, items: &[(&GpuPageMatrix, &ChaChaKey)]) -> Result<u64, DriverError> {
        let tables: Vec<*const ffi::mg_table> = items.iter().map(|(t, _)| t.raw()).collect();
        let keys: Vec<Vec<u8>> = items.iter().map(|(_, k)| k.to_bytes()).collect();
        let ptrs: Vec<*const u8> = keys.iter().map(|k| k.as_ptr()).collect();
        let lens: Vec<usize> = keys.iter().map(|k| k.len()).collect();
        let mut id = 0u64;
        check(unsafe {
            ffi::mg_server_submit(self.raw, tables.as_ptr(), ptrs.as_ptr(), lens.as_ptr(), keys.len() as u32, &mut id)
        })?;
        let sizes = items.iter().map(|(t, _)| t.row_bytes()).collect();
        self.share_bytes.lock().unwrap().insert(id, sizes);
        Ok(id)
    }

    /// Wait for a request (timeout_ms = 0: no deadline); its shares and its
    /// submit-to-answer latency in milliseconds.
    pub fn wait(&self, id: u64, timeout_ms: u32) -> Result<(Vec<Vec<u8>>, f64), DriverError> {
        let sizes = self.share_bytes.lock().unwrap().get(&id).cloned().unwrap_or_default();
        let mut out = vec![0u8; sizes.iter().sum()];
        let mut latency = 0f64;
        let rc = unsafe { ffi::mg_server_wait(self.raw, id, out.as_mut_ptr(), timeout_ms, &mut latency) };
        if rc != ffi::MG_ETIMEDOUT {
            self.share_bytes.lock().unwrap().remove(&id);
        }
        check(rc)?;
        let mut shares = Vec::with_capacity(sizes.len());
        let mut off = 0;
        for n in sizes {
            shares.push(out[off..off + n].to_vec());
            off += n;
        }
        Ok((shares, latency))
    }

    /// Stop dispatching and drain the passes on the GPU (for an epoch merge).
    pub fn pause(&self, timeout_ms: u32) -> Result<(), DriverError> {
        check(unsafe { ffi::mg_server_pause(self.raw, timeout_ms) })
    }

    pub fn resume(&self) -> Result<(), DriverError> {
        check(unsafe { ffi::mg_server_resume(self.raw) })
    }

    pub fn stats(&self) -> Result<ServerStats, DriverError> {
        let mut st = ServerStats::default();
        check(unsafe { ffi::mg_server_get_stats(self.raw, &mut st) })?;
        Ok(st)
    }

    pub fn reset_stats(&self) -> Result<(), DriverError> {
        check(unsafe { ffi::mg_server_reset_stats(self.raw) })
    }
}

impl Drop for PirServer {
    fn drop(&mut self) {
        unsafe {
            ffi::mg_server_destroy(self.raw);
        }
    }
}
