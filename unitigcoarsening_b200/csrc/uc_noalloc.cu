// uc_noalloc.cu — uc_emit_noalloc: unitig line emission that allocates no
// device memory.
//
// Who needs it: callers that cannot call cudaMalloc.  A serving process that
// hands all of a GPU's free memory to its own pool at start-up has nothing
// left for cudaMalloc to give, and its other streams must not stall on the
// device-wide synchronisation cudaMalloc and cudaFree may perform; a plugin
// inside a host framework whose allocator owns the device memory is not
// allowed to allocate behind that allocator's back.  Such a caller can still
// hold packed keys and head/rank arrays (from its own memory) and needs the
// lines spelled.  uc_emit takes its scratch from a context's arenas, which
// are allocated on demand; this variant takes it from one file-scope device
// array instead, sized for at most UC_EMIT_NOALLOC_MAX_KMERS k-mers.
//
// Set-up: the first call on a device (the device current at the call) looks
// the array's address up with cudaGetSymbolAddress and caches it with the
// device's SM count; make that first call before any stream capture.  Every
// call on a device shares the one array, so calls that overlap on the GPU
// (on different streams, or from different host threads) race on it: order
// them on one stream or serialise them.  Each call clears the part that must
// start at zero (the member counts) on its stream before using it.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/uc.h"
#include "uc_pipeline.h"

namespace {

constexpr uint64_t kMaxKmers = UC_EMIT_NOALLOC_MAX_KMERS;
// member counts and line lengths (4 B each), line offsets (8 B), scan block
// sums: 16 MiB + 2.3 KiB at the maximum; the array keeps 64 KiB of slack.
constexpr size_t kScratchBytes = (size_t(16) << 20) + (size_t(64) << 10);
constexpr int kMaxDevices = 64;

struct DeviceSlot {
  std::atomic<void*> ptr{nullptr};
  int sm_count = 0;
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_setup;

void put_err(char* err, size_t err_len, const std::string& msg) {
  if (!err || !err_len) return;
  const size_t m = msg.size() < err_len - 1 ? msg.size() : err_len - 1;
  std::memcpy(err, msg.data(), m);
  err[m] = '\0';
}

}  // namespace

static __device__ __align__(256) unsigned char g_emit_scratch[kScratchBytes];

// Once per device, with that device current: the scratch array's address.
static uc_status setup_device(int dev, void** ptr, int* sms, std::string& msg) {
  void* p = g_slots[dev].ptr.load(std::memory_order_acquire);
  if (p) {
    *ptr = p;
    *sms = g_slots[dev].sm_count;
    return UC_OK;
  }
  std::lock_guard<std::mutex> lock(g_setup);
  p = g_slots[dev].ptr.load(std::memory_order_acquire);
  if (!p) {
    if (uc::emit_scratch_bytes(kMaxKmers) > kScratchBytes) {
      msg = "internal: scratch array smaller than its stated maximum needs";
      return UC_EINTERNAL;
    }
    cudaError_t e = cudaGetSymbolAddress(&p, g_emit_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      msg = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return UC_ECUDA;
    }
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
      cudaGetLastError();
      msg = std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e);
      return UC_ECUDA;
    }
    g_slots[dev].sm_count = n;
    g_slots[dev].ptr.store(p, std::memory_order_release);
  }
  *ptr = p;
  *sms = g_slots[dev].sm_count;
  return UC_OK;
}

extern "C" uc_status uc_emit_noalloc(void* cuda_stream, const uint64_t* d_keys, const uint32_t* d_succ,
                                     const uint32_t* d_head, const uint32_t* d_rank, uint64_t n, int k,
                                     char* d_out, uint64_t cap, uint64_t* out_bytes, char* err, size_t err_len) {
  (void)d_succ;
  put_err(err, err_len, "");
  if (!out_bytes || (n && (!d_keys || !d_head || !d_rank))) {
    put_err(err, err_len, "NULL pointer argument");
    return UC_EINPUT;
  }
  *out_bytes = 0;
  if (n > kMaxKmers) {
    char b[160];
    std::snprintf(b, sizeof b, "n = %llu k-mers exceeds the no-allocation maximum of %llu (UC_EMIT_NOALLOC_MAX_KMERS)",
                  (unsigned long long)n, (unsigned long long)kMaxKmers);
    put_err(err, err_len, b);
    return UC_EINPUT;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    put_err(err, err_len, e != cudaSuccess ? std::string("cudaGetDevice: ") + cudaGetErrorString(e)
                                           : std::string("device id out of range"));
    return UC_ECUDA;
  }
  std::string msg;
  void* scratch = nullptr;
  int sms = 0;
  uc_status s = setup_device(dev, &scratch, &sms, msg);
  if (s != UC_OK) {
    put_err(err, err_len, msg);
    return s;
  }
  uint64_t ob = 0;
  const int r = uc::emit_in(static_cast<cudaStream_t>(cuda_stream), sms, d_keys, d_head, d_rank, n, k, d_out, cap,
                            ob, scratch, msg);
  *out_bytes = ob;
  if (r) {
    if (r == UC_ECUDA) cudaGetLastError();
    put_err(err, err_len, msg);
  }
  return static_cast<uc_status>(r);
}
