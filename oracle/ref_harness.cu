// ref_harness.cu -- TEST INFRASTRUCTURE ONLY: launches the reference's own
// CUDA kernels (crates/morphogen-gpu-dpf/cuda/fused_kernel.cu and
// fused_kernel_optimized.cu, compiled unmodified from the reference tree by
// oracle/ref_build.py into oracle/_ref/) so that tests can compare the
// library's page-mode shares with the reference implementation's, and so
// that bench comparisons can time the reference kernel on the same GPU.
//
// The harness itself is written here: the device key conversion follows
// DpfKeyGpu::from_chacha_key (crates/morphogen-gpu-dpf/src/kernel.rs:126-153)
// and the launch recipe follows GpuScanner::new / scan_batch_opts
// (kernel.rs:293-303,339-349,774-787): grid ceil(pages / 2048), 256 threads,
// dynamic shared memory B*3*4096 + B*3*16 + B*3*32 (+ 256*B*3*16 for the
// baseline kernel), outputs zeroed before the launch.
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace {
constexpr int kRefMaxLevels = 25;   // MAX_DOMAIN_BITS of the reference kernel
constexpr int kPod = 488;           // sizeof(DpfKeyGpu), cuda/fused_kernel.cu:108-118
constexpr int kPage = 4096;
constexpr int kSubtree = 2048;
}  // namespace

struct RefKeyPod;  // the reference's DpfKeyGpu, opaque here

extern "C" __global__ void fused_batch_pir_kernel_1(const uint4*, const RefKeyPod*, uint4*, uint4*, int, int);
extern "C" __global__ void fused_batch_pir_kernel_optimized_1(const uint4*, const RefKeyPod*, uint4*, uint4*, int, int);
extern "C" __global__ void fused_batch_pir_kernel_optimized_2(const uint4*, const RefKeyPod*, uint4*, uint4*, int, int);
extern "C" __global__ void fused_batch_pir_kernel_optimized_4(const uint4*, const RefKeyPod*, uint4*, uint4*, int, int);

static uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// Wire key (dpf.rs:259-274) -> reference device POD (kernel.rs:126-153,
// truncating to 25 levels exactly as the reference does).  Returns 0 or -1.
extern "C" int ref_key_pod(const uint8_t* wire, size_t len, uint8_t* pod) {
  if (len < 35) return -1;
  const uint32_t d = wire[18];
  if (len != 19 + (size_t)d * 18 + 16) return -1;
  std::memset(pod, 0, kPod);
  uint32_t w[4];
  for (int i = 0; i < 4; ++i) w[i] = le32(wire + 4 * i);
  std::memcpy(pod, w, 16);                 // root_seed
  pod[16] = wire[16];                      // root_t
  pod[17] = (uint8_t)d;                    // domain_bits
  const size_t cw_off = 20, tl_off = 20 + 16 * kRefMaxLevels, tr_off = tl_off + kRefMaxLevels;
  const size_t fin_off = tr_off + kRefMaxLevels + 2;
  for (uint32_t l = 0; l < d && l < (uint32_t)kRefMaxLevels; ++l) {
    const uint8_t* c = wire + 19 + 18 * l;
    for (int i = 0; i < 4; ++i) w[i] = le32(c + 4 * i);
    std::memcpy(pod + cw_off + 16 * l, w, 16);
    pod[tl_off + l] = c[16];
    pod[tr_off + l] = c[17];
  }
  const uint8_t* f = wire + 19 + 18 * d;
  for (int i = 0; i < 4; ++i) w[i] = le32(f + 4 * i);
  std::memcpy(pod + fin_off, w, 16);
  return 0;
}

// One launch of the reference kernel over num_pages 4096-byte pages already
// on the device.  kind 0: baseline fused_batch_pir_kernel_1 (batch must be
// 1); kind 1: fused_batch_pir_kernel_optimized_<batch>, batch in {1, 2, 4}.
// pods: batch*3 device keys (host memory).  out: batch*3*4096 bytes (host).
// reps >= 1 launches are timed with CUDA events (*ms = best).  Returns 0, or
// a CUDA error code.
extern "C" int ref_scan(int kind, int batch, const void* db_dev, int num_pages, const uint8_t* pods,
                        uint8_t* out, int reps, float* ms) {
  const int nk = batch * 3;
  size_t smem = (size_t)nk * kPage + (size_t)nk * 16 + (size_t)nk * 32;
  const void* fn = nullptr;
  if (kind == 0 && batch == 1) {
    fn = (const void*)fused_batch_pir_kernel_1;
    smem += 256 * (size_t)nk * 16;
  } else if (kind == 1 && batch == 1) {
    fn = (const void*)fused_batch_pir_kernel_optimized_1;
  } else if (kind == 1 && batch == 2) {
    fn = (const void*)fused_batch_pir_kernel_optimized_2;
  } else if (kind == 1 && batch == 4) {
    fn = (const void*)fused_batch_pir_kernel_optimized_4;
  } else {
    return (int)cudaErrorInvalidValue;
  }
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return (int)e;
  void *d_keys = nullptr, *d_out = nullptr, *d_verif = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const size_t out_bytes = (size_t)nk * kPage;
  if ((e = cudaMalloc(&d_keys, (size_t)nk * kPod)) == cudaSuccess &&
      (e = cudaMalloc(&d_out, out_bytes)) == cudaSuccess &&
      (e = cudaMalloc(&d_verif, (size_t)nk * 16)) == cudaSuccess &&
      (e = cudaMemcpy(d_keys, pods, (size_t)nk * kPod, cudaMemcpyHostToDevice)) == cudaSuccess &&
      (e = cudaEventCreate(&e0)) == cudaSuccess && (e = cudaEventCreate(&e1)) == cudaSuccess) {
    const dim3 grid((unsigned)((num_pages + kSubtree - 1) / kSubtree)), block(256);
    const uint4* db = static_cast<const uint4*>(db_dev);
    const RefKeyPod* keys = static_cast<const RefKeyPod*>(d_keys);
    uint4* o = static_cast<uint4*>(d_out);
    uint4* v = static_cast<uint4*>(d_verif);
    int n = num_pages, b = batch;
    void* args[] = {&db, &keys, &o, &v, &n, &b};
    float best = 1e30f;
    for (int r = 0; r < (reps < 1 ? 1 : reps) && e == cudaSuccess; ++r) {
      if ((e = cudaMemset(d_out, 0, out_bytes)) != cudaSuccess) break;
      if ((e = cudaMemset(d_verif, 0, (size_t)nk * 16)) != cudaSuccess) break;
      cudaEventRecord(e0);
      if ((e = cudaLaunchKernel(fn, grid, block, args, smem, nullptr)) != cudaSuccess) break;
      cudaEventRecord(e1);
      if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (t < best) best = t;
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, out_bytes, cudaMemcpyDeviceToHost);
    if (ms) *ms = best;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (d_keys) cudaFree(d_keys);
  if (d_out) cudaFree(d_out);
  if (d_verif) cudaFree(d_verif);
  return (int)e;
}
