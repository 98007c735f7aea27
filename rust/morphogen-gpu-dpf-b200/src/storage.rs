//! GpuPageMatrix (crates/morphogen-gpu-dpf/src/storage.rs:18-146) over
//! mg_table: a device-resident table of rows.  The reference's page is a
//! 4096-byte row; the `_rows` constructors take any multiple of 16 up to 4096.
use std::os::raw::c_void;
use std::sync::Arc;

use crate::device::{check, DriverError, GpuDevice};
use crate::ffi;

/// storage.rs:14.
pub const PAGE_SIZE_BYTES: usize = 4096;

/// The chunk view from_chunked_matrix reads (the storage crate's
/// ChunkedMatrix: implement it there with num_chunks / chunk(i).as_slice()).
pub trait ChunkSource {
    fn num_chunks(&self) -> usize;
    fn chunk_bytes(&self, i: usize) -> &[u8];
}

/// Device pointer and length of the resident rows (storage.rs:137-140
/// returns the CudaSlice itself).
#[derive(Clone, Copy, Debug)]
pub struct DeviceSlice {
    pub ptr: *const c_void,
    pub len: usize,
}

pub struct GpuPageMatrix {
    device: Arc<GpuDevice>,
    raw: *mut ffi::mg_table,
    num_pages: usize,
    row_bytes: usize,
}

unsafe impl Send for GpuPageMatrix {}
unsafe impl Sync for GpuPageMatrix {}

impl GpuPageMatrix {
    /// storage.rs:27-43 (panics on a length that is not whole pages, as there).
    pub fn new(device: Arc<GpuDevice>, cpu_data: &[u8]) -> Result<Self, DriverError> {
        Self::new_rows(device, cpu_data, PAGE_SIZE_BYTES)
    }

    pub fn new_rows(device: Arc<GpuDevice>, cpu_data: &[u8], row_bytes: usize) -> Result<Self, DriverError> {
        if cpu_data.len() % row_bytes != 0 {
            panic!("cpu_data length must be multiple of PAGE_SIZE_BYTES");
        }
        let mut m = Self::alloc_empty_rows(device, cpu_data.len() / row_bytes, row_bytes)?;
        m.update_pages(0, cpu_data)?;
        Ok(m)
    }

    /// storage.rs:46-86: chunks uploaded at their byte offsets, the total
    /// padded with zeros to whole pages.
    pub fn from_chunked_matrix<M: ChunkSource + ?Sized>(device: Arc<GpuDevice>, matrix: &M)
        -> Result<Self, DriverError> {
        Self::from_chunked_matrix_rows(device, matrix, PAGE_SIZE_BYTES)
    }

    pub fn from_chunked_matrix_rows<M: ChunkSource + ?Sized>(device: Arc<GpuDevice>, matrix: &M, row_bytes: usize)
        -> Result<Self, DriverError> {
        let total: usize = (0..matrix.num_chunks()).map(|i| matrix.chunk_bytes(i).len()).sum();
        let mut m = Self::alloc_empty_rows(device, (total + row_bytes - 1) / row_bytes, row_bytes)?;
        let mut offset = 0usize;
        for i in 0..matrix.num_chunks() {
            let chunk = matrix.chunk_bytes(i);
            if chunk.len() % row_bytes != 0 {
                let mut padded = chunk.to_vec();
                padded.resize(chunk.len() + row_bytes - chunk.len() % row_bytes, 0);
                m.update_pages(offset / row_bytes, &padded)?;
            } else if !chunk.is_empty() {
                m.update_pages(offset / row_bytes, chunk)?;
            }
            offset += chunk.len();
        }
        Ok(m)
    }

    /// storage.rs:89-101: zero-filled pages.
    pub fn alloc_empty(device: Arc<GpuDevice>, num_pages: usize) -> Result<Self, DriverError> {
        Self::alloc_empty_rows(device, num_pages, PAGE_SIZE_BYTES)
    }

    pub fn alloc_empty_rows(device: Arc<GpuDevice>, num_rows: usize, row_bytes: usize) -> Result<Self, DriverError> {
        Self::alloc_range(device, 0, num_rows, row_bytes)
    }

    /// Rows [first_row, first_row + num_rows) of a larger logical table: the
    /// range answers at its logical rows, so the shares of the ranges that
    /// partition a table XOR to the whole table's share.
    pub fn alloc_range(device: Arc<GpuDevice>, first_row: usize, num_rows: usize, row_bytes: usize)
        -> Result<Self, DriverError> {
        let mut raw = std::ptr::null_mut();
        check(unsafe {
            ffi::mg_table_create_range(device.raw(), first_row as u64, num_rows as u64, row_bytes as u32, &mut raw)
        })?;
        Ok(Self { device, raw, num_pages: num_rows, row_bytes })
    }

    /// storage.rs:104-124 (panics on a bad length or range, as there).
    pub fn update_pages(&mut self, start_page: usize, cpu_pages: &[u8]) -> Result<(), DriverError> {
        if cpu_pages.len() % self.row_bytes != 0 {
            panic!("cpu_pages length must be multiple of PAGE_SIZE_BYTES");
        }
        let n = cpu_pages.len() / self.row_bytes;
        if start_page + n > self.num_pages {
            panic!("Update range exceeds matrix bounds");
        }
        check(unsafe {
            ffi::mg_table_write_rows(self.raw, start_page as u64, cpu_pages.as_ptr() as *const c_void, n as u64)
        })
    }

    /// Synthetic rows: SplitMix64 bytes of `seed`, generated on the device.
    pub fn fill_splitmix(&mut self, seed: u64) -> Result<(), DriverError> {
        check(unsafe { ffi::mg_table_fill_splitmix(self.raw, seed) })
    }

    /// Epoch merge of explicit entries: rows[idx[i]] ^= diffs[i].
    pub fn xor_rows(&mut self, idx: &[u64], diffs: &[u8]) -> Result<(), DriverError> {
        assert_eq!(diffs.len(), idx.len() * self.row_bytes, "one diff row per index");
        check(unsafe { ffi::mg_table_xor_rows(self.raw, idx.as_ptr(), diffs.as_ptr() as *const c_void, idx.len() as u64) })
    }

    /// Device-resident pending delta (DeltaBuffer + scan_delta_for_gpu): every
    /// pass folds it into the shares until delta_merge patches the table.
    pub fn delta_reserve(&mut self, capacity: u32) -> Result<(), DriverError> {
        check(unsafe { ffi::mg_table_delta_reserve(self.raw, capacity) })
    }

    pub fn delta_push(&mut self, idx: &[u64], diffs: &[u8]) -> Result<(), DriverError> {
        assert_eq!(diffs.len(), idx.len() * self.row_bytes, "one diff row per index");
        check(unsafe { ffi::mg_table_delta_push(self.raw, idx.as_ptr(), diffs.as_ptr() as *const c_void, idx.len() as u32) })
    }

    pub fn delta_count(&self) -> u32 {
        unsafe { ffi::mg_table_delta_count(self.raw) }
    }

    pub fn delta_clear(&mut self) -> Result<(), DriverError> {
        check(unsafe { ffi::mg_table_delta_clear(self.raw) })
    }

    pub fn delta_merge(&mut self) -> Result<(), DriverError> {
        check(unsafe { ffi::mg_table_delta_merge(self.raw) })
    }

    pub fn epoch(&self) -> u64 {
        unsafe { ffi::mg_table_epoch(self.raw) }
    }

    pub fn num_pages(&self) -> usize {
        self.num_pages
    }

    pub fn row_bytes(&self) -> usize {
        self.row_bytes
    }

    pub fn first_row(&self) -> usize {
        unsafe { ffi::mg_table_first_row(self.raw) as usize }
    }

    pub fn size_bytes(&self) -> usize {
        self.num_pages * self.row_bytes
    }

    pub fn as_slice(&self) -> DeviceSlice {
        DeviceSlice { ptr: unsafe { ffi::mg_table_device_ptr(self.raw) }, len: self.size_bytes() }
    }

    pub fn device(&self) -> Arc<GpuDevice> {
        self.device.clone()
    }

    pub(crate) fn raw(&self) -> *const ffi::mg_table {
        self.raw
    }
}

impl Drop for GpuPageMatrix {
    fn drop(&mut self) {
        unsafe {
            ffi::mg_table_destroy(self.raw);
        }
    }
}
