//! The device handle and the driver error, standing in for cudarc's
//! `Arc<CudaDevice>` and `DriverError` in the reference's signatures.
use std::os::raw::c_int;
use std::sync::Arc;

use crate::ffi;

/// A failing library call: the MG_E* status and the library's message
/// (the reference maps its cudarc DriverError to HTTP 500).
#[derive(Debug, Clone)]
pub struct DriverError {
    pub code: i32,
    pub message: String,
}

impl DriverError {
    pub(crate) fn last(code: c_int) -> Self {
        Self { code, message: ffi::last_error() }
    }
}

impl std::fmt::Display for DriverError {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "morphogen_gpu error {}: {}", self.code, self.message)
    }
}

impl std::error::Error for DriverError {}

pub(crate) fn check(code: c_int) -> Result<(), DriverError> {
    if code == ffi::MG_OK {
        Ok(())
    } else {
        Err(DriverError::last(code))
    }
}

/// One library context on one GPU (GpuScanner::new's CudaDevice).  Calls on
/// a context are serialised inside the library, so the handle is shared
/// between threads.
pub struct GpuDevice {
    raw: *mut ffi::mg_context,
    ordinal: usize,
}

unsafe impl Send for GpuDevice {}
unsafe impl Sync for GpuDevice {}

impl GpuDevice {
    pub fn new(ordinal: usize) -> Result<Arc<Self>, DriverError> {
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::mg_context_create(ordinal as c_int, &mut raw) })?;
        Ok(Arc::new(Self { raw, ordinal }))
    }

    pub fn ordinal(&self) -> usize {
        self.ordinal
    }

    pub(crate) fn raw(&self) -> *mut ffi::mg_context {
        self.raw
    }

    /// (SM count, free bytes, total bytes) of the device.
    pub fn info(&self) -> Result<(i32, u64, u64), DriverError> {
        let (mut sms, mut free, mut total) = (0 as c_int, 0u64, 0u64);
        check(unsafe { ffi::mg_device_info(self.raw, &mut sms, &mut free, &mut total) })?;
        Ok((sms, free, total))
    }

    /// Node expansions per second of the device ChaCha8 PRG alone.
    pub fn prg_peak(&self) -> Result<f64, DriverError> {
        let mut v = 0f64;
        check(unsafe { ffi::mg_prg_peak(self.raw, 256, &mut v) })?;
        Ok(v)
    }
}

impl Drop for GpuDevice {
    fn drop(&mut self) {
        unsafe {
            ffi::mg_context_destroy(self.raw);
        }
    }
}
