//! B200 (sm_100a) drop-in for the reference's `morphogen-gpu-dpf` crate.
//!
//! Same crate name, types and entry points as
//! crates/morphogen-gpu-dpf/src/lib.rs:20-28 -- `ChaChaKey`, `ChaChaParams`,
//! `GpuDpfError`, `generate_chacha_dpf_keys`, `GpuScanner`, `GpuPageMatrix`,
//! `PirResult`, `KernelTiming` -- so the server's handlers build against it
//! unchanged, except that the device handle is `Arc<GpuDevice>` (the
//! reference's `Arc<CudaDevice>` from cudarc) and errors are `DriverError`
//! from this crate.  Every scan runs in libmorphogen_gpu.so through the C
//! ABI of include/morphogen_gpu.h (module `ffi`), which build.rs builds with
//! nvcc or finds prebuilt.  Differences a caller sees: depths up to 32 are
//! evaluated in full (the reference kernel truncates at 25, kernel.rs:45,
//! 131-136), rows may be any multiple of 16 bytes up to 4096 (`_rows`
//! constructors), and the CPU PRG types of chacha_prg.rs are not exported
//! (point evaluation runs on the device: `GpuScanner::eval_points`).
pub mod device;
pub mod dpf;
pub mod ffi;
pub mod kernel;
pub mod server;
pub mod storage;

pub use device::{DriverError, GpuDevice};
pub use dpf::{generate_chacha_dpf_keys, generate_chacha_dpf_keys_with_seeds, ChaChaKey, ChaChaParams, CorrectionWord,
              GpuDpfError, Seed128};
pub use kernel::{GpuScanner, KernelTiming, PirResult};
pub use server::PirServer;
pub use storage::{ChunkSource, GpuPageMatrix, PAGE_SIZE_BYTES};

/// The allocation-free scan (mg_scan_noalloc) for callers that own all
/// device memory: `table` and `out` are device pointers on `device`, `out`
/// receives keys.len() x row_bytes bytes; `stream` is a cudaStream_t or null.
///
/// # Safety
/// The pointers must be valid device memory of the stated sizes on `device`,
/// and calls that overlap on the GPU must be serialised by the caller.
pub unsafe fn scan_noalloc(device: i32, table: *const std::os::raw::c_void, rows: u64, row_bytes: u32,
                           keys: &[&ChaChaKey], out: *mut std::os::raw::c_void,
                           stream: *mut std::os::raw::c_void) -> Result<(), DriverError> {
    let bytes: Vec<Vec<u8>> = keys.iter().map(|k| k.to_bytes()).collect();
    let ptrs: Vec<*const u8> = bytes.iter().map(|b| b.as_ptr()).collect();
    let lens: Vec<usize> = bytes.iter().map(|b| b.len()).collect();
    device::check(ffi::mg_scan_noalloc(device, table, rows, row_bytes, ptrs.as_ptr(), lens.as_ptr(), bytes.len() as u32,
                                       out, stream))
}
