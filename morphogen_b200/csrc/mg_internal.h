// mg_internal.h -- launchers shared between the kernels and the C ABI layer.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "mg_device.cuh"

namespace mg {

size_t scan_smem_bytes(int G, uint32_t slots);
bool scan_g_supported(int G);
// Raise (never lower) the kernel's dynamic shared memory limit on the current
// device to at least smem.  The limit is process-wide per device and kernel,
// so every caller goes through this one record (scan_prepare / warp_prepare).
cudaError_t scan_prepare(int G, size_t smem);
int scan_occupancy(int G, size_t smem);
cudaError_t launch_scan(int G, const ScanParams& p, uint32_t grid, size_t smem, cudaStream_t st);
// out = XOR of the partial rows; out is cleared first unless out_zeroed.
cudaError_t launch_reduce(const uint4* partial, uint32_t nparts, uint32_t cols, uint4* out,
                          cudaStream_t st, bool out_zeroed = false);
cudaError_t launch_fill_splitmix(void* dst, uint64_t words, uint64_t seed, uint64_t word0, int sms, cudaStream_t st);
// dst[i] = src[i] for n uint4 (either side may be a pinned host buffer's
// device-mapped address) and zero[i] = 0 for nz uint4.
cudaError_t launch_copy_u4(const void* src, void* dst, uint32_t n, cudaStream_t st, void* zero = nullptr,
                           uint32_t nz = 0);
cudaError_t launch_xor_rows(void* table, uint32_t V, const uint64_t* idx, const void* diffs,
                            uint64_t n, int sms, cudaStream_t st);
cudaError_t launch_eval_points(const KeyDev* key, const uint64_t* idx, uint64_t n, void* out, int sms,
                               cudaStream_t st);

// Warp-independent scan (V uint4 per row in {1,2,4,8,16,32}, G keys per warp
// in 1..4), CTAs of nw warps (kWarps = 16 when the shared memory fits, else 8 or 4).
size_t warp_smem_bytes(int G, uint32_t VT, uint32_t slots, uint32_t nw);
bool warp_vt_supported(uint32_t V);
bool warp_g_supported(int G);
cudaError_t warp_prepare(int G, uint32_t VT, size_t smem);
int warp_occupancy(int G, uint32_t VT, size_t smem, uint32_t nw);
bool warp_reduces_in_kernel(int G, uint32_t VT);
cudaError_t launch_scan_warp(int G, uint32_t VT, const WarpScanParams& p, uint32_t grid, uint32_t nw, size_t smem,
                             cudaStream_t st);
cudaError_t launch_frontier(const FrontierStep& f, uint32_t nkeys, cudaStream_t st);
// Folds a table's pending delta into the shares: jobs[j] = (key slot, first share column).
cudaError_t launch_delta(const KeyDev* keys, const uint2* jobs, uint32_t njobs, const uint64_t* idx,
                         const void* diffs, const uint32_t* count, uint32_t capacity, uint32_t V, uint64_t first,
                         uint4* out, cudaStream_t st);

}  // namespace mg

struct mg_batch;
struct mg_context;

namespace mg {

// True once the workspace's last enqueued work has completed on the device.
bool batch_done(mg_batch* b);
int context_device(const mg_context* ctx);

// Sets the thread-local message returned by mg_last_error().
void set_last_error(const char* msg);

cudaError_t prg_peak_shape(int sms, uint32_t* blocks, uint32_t* threads);
cudaError_t launch_prg_peak(uint32_t* out, uint32_t iters, uint32_t blocks, uint32_t threads,
                            cudaStream_t st);

}  // namespace mg
