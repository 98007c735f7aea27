// mg_noalloc.cu -- the scan entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc: a host application or memory pool may
// own all device memory (plugins, embedded servers), and in a latency-bound
// serving loop cudaMalloc/cudaFree can block on or synchronise the device
// and stall every other stream.  mg_scan_noalloc serves them: it runs the
// same scan and reduction kernels as mg_scan, with the parsed keys and the
// per-CTA partial rows placed in one file-scope device array of fixed size
// (g_noalloc_scratch) instead of allocated buffers.  The caller passes the
// table and the output buffer, both in device memory it already owns.
//
// The keys reach the array by value, inside the parameters of a small copy
// kernel (up to kStageKeys keys per launch), so no host buffer has to outlive
// the call and no copy from pageable memory makes the host wait for the
// stream.
//
// The array is held by every GPU that loads the library until the process
// exits.  All calls on a device share it and it keeps the last call's
// contents: the scan kernel zeroes its own partial rows before use and the
// reduction overwrites every output byte, so no state leaks from one call
// into the next, but calls that overlap on the GPU (different streams, or
// different host threads without ordering) race on the array.
#include <cstring>
#include <mutex>

#include "mg_internal.h"
#include "morphogen_gpu.h"

namespace {

constexpr size_t kScratchBytes = (size_t)MG_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Host-side state per device: the array's device address (in host code the
// symbol is only a stand-in and must never be passed to a kernel) and the SM
// count.  The scan kernel's shared-memory limit is not kept here: it is
// process-wide per device and raised through mg::scan_prepare, which every
// entry point shares.
struct DeviceSlot {
  bool ready = false;
  unsigned char* scratch = nullptr;
  int sms = 0;
  size_t smem_optin = 0;
};

// Keys per copy launch: 16 x 624 B of kernel parameters.
constexpr uint32_t kStageKeys = 16;
struct KeyStage {
  mg::KeyDev k[kStageKeys];
  uint32_t n;
};

__global__ void stage_keys_kernel(const __grid_constant__ KeyStage s, mg::KeyDev* __restrict__ dst) {
  const uint4* src = reinterpret_cast<const uint4*>(s.k);
  uint4* d = reinterpret_cast<uint4*>(dst);
  const uint32_t words = s.n * (uint32_t)(sizeof(mg::KeyDev) / 16);
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) d[i] = src[i];
}
DeviceSlot g_slots[kMaxDevices];
std::mutex g_mu;

// Errors go to the thread-local message read by mg_last_error().
int noalloc_fail(int code, const char* msg) {
  mg::set_last_error(msg);
  return code;
}

uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// ChaChaKey::from_bytes (dpf.rs:277-316) into the device layout, no heap use.
int parse(const uint8_t* b, size_t len, mg::KeyDev* k) {
  if (!b) return noalloc_fail(MG_EINVAL, "mg_scan_noalloc: null key pointer");
  if (len < 35) return noalloc_fail(MG_EKEY, "mg_scan_noalloc: invalid key format: byte array too short");
  const uint32_t d = b[18];
  if (len != 19 + (size_t)d * 18 + 16)
    return noalloc_fail(MG_EKEY, "mg_scan_noalloc: invalid key format: invalid byte array length");
  if (d > MG_MAX_DOMAIN_BITS)
    return noalloc_fail(MG_ERANGE, "mg_scan_noalloc: key domain_bits exceeds 32");
  std::memset(k, 0, sizeof *k);
  k->root_seed = make_uint4(le32(b), le32(b + 4), le32(b + 8), le32(b + 12));
  k->root_t = b[16];
  k->domain_bits = d;
  size_t off = 19;
  for (uint32_t l = 0; l < d; ++l) {
    k->cw_seed[l] = make_uint4(le32(b + off), le32(b + off + 4), le32(b + off + 8), le32(b + off + 12));
    k->cw_tl[l] = b[off + 16];
    k->cw_tr[l] = b[off + 17];
    off += 18;
  }
  k->final_cw = make_uint4(le32(b + off), le32(b + off + 4), le32(b + off + 8), le32(b + off + 12));
  return MG_OK;
}

// One-time set-up on `device`, which the caller has made current.
int setup(int device, DeviceSlot*& slot) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceSlot& s = g_slots[device];
  if (!s.ready) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr)
      return noalloc_fail(MG_ECUDA, "mg_scan_noalloc: cudaGetSymbolAddress of the static scratch failed");
    int sms = 0, optin = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess)
      return noalloc_fail(MG_ECUDA, "mg_scan_noalloc: cannot query the device");
    s.scratch = static_cast<unsigned char*>(ptr);
    s.sms = sms;
    s.smem_optin = (size_t)optin;
    s.ready = true;
  }
  slot = &s;
  return MG_OK;
}

}  // namespace

extern "C" int mg_scan_noalloc(int device, const void* table_dev, uint64_t rows, uint32_t row_bytes,
                               const uint8_t* const* keys, const size_t* key_lens, uint32_t nkeys,
                               void* out_shares_dev, void* stream) {
  if (!table_dev || !keys || !key_lens || !out_shares_dev)
    return noalloc_fail(MG_EINVAL, "mg_scan_noalloc: null argument");
  if (device < 0 || device >= kMaxDevices) return noalloc_fail(MG_EINVAL, "mg_scan_noalloc: bad device");
  if (nkeys == 0 || nkeys > MG_NOALLOC_MAX_KEYS)
    return noalloc_fail(MG_ERANGE, "mg_scan_noalloc: nkeys must be in [1, MG_NOALLOC_MAX_KEYS]");
  if (row_bytes == 0 || row_bytes % 16 != 0 || row_bytes > MG_MAX_ROW_BYTES)
    return noalloc_fail(MG_EINVAL, "mg_scan_noalloc: row_bytes must be a multiple of 16 in [16, 4096]");
  if (cudaSetDevice(device) != cudaSuccess) return noalloc_fail(MG_ECUDA, "mg_scan_noalloc: cudaSetDevice failed");
  DeviceSlot* slot = nullptr;
  if (int rc = setup(device, slot)) return rc;

  mg::KeyDev staged[MG_NOALLOC_MAX_KEYS];
  for (uint32_t i = 0; i < nkeys; ++i)
    if (int rc = parse(keys[i], key_lens[i], &staged[i])) return rc;
  const uint32_t d = staged[0].domain_bits;
  for (uint32_t i = 1; i < nkeys; ++i)
    if (staged[i].domain_bits != d)
      return noalloc_fail(MG_EINVAL, "mg_scan_noalloc: all keys of one call must share domain_bits");
  if (d < 64 && rows > (1ull << d))
    return noalloc_fail(MG_ERANGE, "mg_scan_noalloc: more rows than domain size");

  // Shape: one key per CTA, the deepest tile (<= 14 levels) giving >= 4 waves.
  const uint32_t V = row_bytes / 16;
  mg::ScanParams p;
  std::memset(&p, 0, sizeof p);
  uint32_t grid = 0;
  size_t smem = 0;
  for (uint32_t S_target = 14;; --S_target) {
    const uint32_t S = S_target < d ? S_target : d;
    const uint32_t U = S >= 1 ? (S - 1 < 8 ? S - 1 : 8) : 0;
    const uint32_t M = S - U;
    const uint32_t slots = M > 2 ? M : 2;
    smem = mg::scan_smem_bytes(1, slots);
    const uint64_t tiles = (rows + (1ull << S) - 1) >> S;
    const uint64_t items = tiles * nkeys;
    int occ = 0;
    if (smem <= slot->smem_optin) {
      if (mg::scan_prepare(1, smem) != cudaSuccess)
        return noalloc_fail(MG_ECUDA, "mg_scan_noalloc: cannot set the kernel's shared memory");
      occ = mg::scan_occupancy(1, smem);
    }
    const uint64_t slots_total = (uint64_t)(occ > 0 ? occ : 1) * slot->sms;
    if ((occ > 0 && items >= 4 * slots_total) || S_target <= 8) {
      if (occ <= 0) return noalloc_fail(MG_EINVAL, "mg_scan_noalloc: no launch shape fits the device");
      mg::Segment& sg = p.seg[0];
      sg.table = static_cast<const uint4*>(table_dev);
      sg.rows = rows;
      sg.item_begin = 0;
      sg.tiles = (uint32_t)tiles;
      sg.groups = nkeys;
      sg.V = V;
      sg.d = d;
      sg.S = S;
      sg.U = U;
      sg.M = M;
      sg.g = 1;
      sg.key_base = 0;
      sg.col_base = 0;
      p.nsegs = 1;
      p.items = items;
      p.cols = nkeys * V;
      p.slots = slots;
      grid = (uint32_t)(items < slots_total ? (items ? items : 1) : slots_total);
      break;
    }
  }

  // Scratch layout: staged keys, then the per-CTA partial rows (256-B aligned).
  const size_t key_bytes = (size_t)nkeys * sizeof(mg::KeyDev);
  const size_t part_off = (key_bytes + 255) / 256 * 256;
  const size_t part_bytes = (size_t)grid * p.cols * 16;
  if (part_off + part_bytes > kScratchBytes)
    return noalloc_fail(MG_ERANGE,
                        "mg_scan_noalloc: keys and partial rows exceed the MG_NOALLOC_SCRATCH_BYTES static scratch "
                        "(reduce nkeys * row_bytes)");
  p.keys = reinterpret_cast<const mg::KeyDev*>(slot->scratch);
  p.partial = reinterpret_cast<uint4*>(slot->scratch + part_off);

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Keys travel by value in the copy kernel's parameters.
  mg::KeyDev* const d_keys = reinterpret_cast<mg::KeyDev*>(slot->scratch);
  for (uint32_t i0 = 0; i0 < nkeys; i0 += kStageKeys) {
    KeyStage ks;
    ks.n = nkeys - i0 < kStageKeys ? nkeys - i0 : kStageKeys;
    std::memcpy(ks.k, staged + i0, ks.n * sizeof(mg::KeyDev));
    stage_keys_kernel<<<1, 256, 0, st>>>(ks, d_keys + i0);
    if (cudaGetLastError() != cudaSuccess) return noalloc_fail(MG_ECUDA, "mg_scan_noalloc: key upload failed");
  }
  if (mg::launch_scan(1, p, grid, smem, st) != cudaSuccess)
    return noalloc_fail(MG_ECUDA, "mg_scan_noalloc: scan launch failed");
  if (mg::launch_reduce(p.partial, grid, p.cols, static_cast<uint4*>(out_shares_dev), st) != cudaSuccess)
    return noalloc_fail(MG_ECUDA, "mg_scan_noalloc: reduction launch failed");
  return MG_OK;
}
