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
// Set-up: the first call in a CUDA context (the device current at the call,
// and its primary or current context) looks the array's address up with
// cudaGetSymbolAddress, loads every kernel the emission launches, and caches
// the address with the device's SM count, keyed by the context's unique id.
// CUDA loads modules lazily by default: the array and the kernels take their
// device memory at that first call.  So make the first call, on every device
// and context it will run in, before the caller hands the rest of the
// device's memory to its own pool (or run with CUDA_MODULE_LOADING=EAGER),
// and before any stream capture.  A context that is destroyed and created
// again (cudaDeviceReset) gets a new id, so the next call sets up again.
// Every call in a context shares the one array, so calls that overlap on the
// GPU (on different streams, or from different host threads) race on it:
// order them on one stream or serialise them.  Each call clears the part
// that must start at zero (the member counts) on its stream before using it.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/uc.h"
#include "uc_pipeline.h"

namespace {

constexpr uint64_t kMaxKmers = UC_EMIT_NOALLOC_MAX_KMERS;
// member counts and line lengths (4 B each), line offsets (8 B), scan block
// sums: 16 MiB + 2.3 KiB at the maximum; the array keeps 64 KiB of slack.
constexpr size_t kScratchBytes = (size_t(16) << 20) + (size_t(64) << 10);

// One cache entry per CUDA context that has called: the context's unique id
// (cuCtxGetId), the array's address in it and the device's SM count.
struct Slot {
  unsigned long long ctx_id;
  void* ptr;
  int sm_count;
};
std::vector<Slot> g_slots;
std::mutex g_setup;

using PfnCtxGetCurrent = int (*)(void**);
using PfnCtxGetId = int (*)(void*, unsigned long long*);
PfnCtxGetCurrent g_ctx_current = nullptr;
PfnCtxGetId g_ctx_id = nullptr;
std::once_flag g_entry_once;

// The current context's unique id (driver entry points found through the
// runtime, so the library needs no link to the driver library); false when
// no context is current or the driver lacks them.
bool current_ctx_id(unsigned long long* id) {
  std::call_once(g_entry_once, [] {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_current = reinterpret_cast<PfnCtxGetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_id = reinterpret_cast<PfnCtxGetId>(f);
    cudaGetLastError();
  });
  if (!g_ctx_current || !g_ctx_id) return false;
  void* ctx = nullptr;
  if (g_ctx_current(&ctx) != 0 || !ctx) return false;
  return g_ctx_id(ctx, id) == 0;
}

void put_err(char* err, size_t err_len, const std::string& msg) {
  if (!err || !err_len) return;
  const size_t m = msg.size() < err_len - 1 ? msg.size() : err_len - 1;
  std::memcpy(err, msg.data(), m);
  err[m] = '\0';
}

}  // namespace

static __device__ __align__(256) unsigned char g_emit_scratch[kScratchBytes];

// Once per context, with that context current: the scratch array's address,
// every emission kernel loaded.
static uc_status setup_context(int dev, void** ptr, int* sms, std::string& msg) {
  std::lock_guard<std::mutex> lock(g_setup);
  unsigned long long id = 0;
  bool have_id = current_ctx_id(&id);
  if (have_id) {
    for (const Slot& s : g_slots)
      if (s.ctx_id == id) {
        *ptr = s.ptr;
        *sms = s.sm_count;
        return UC_OK;
      }
  }
  if (uc::emit_scratch_bytes(kMaxKmers) > kScratchBytes) {
    msg = "internal: scratch array smaller than its stated maximum needs";
    return UC_EINTERNAL;
  }
  // the lookup makes the runtime create (or take) the device's context
  void* p = nullptr;
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
  const int r = uc::emit_preload(msg);
  if (r) return static_cast<uc_status>(r);
  if (!have_id) have_id = current_ctx_id(&id);
  // without a context id (a driver without cuCtxGetId) nothing is cached and
  // every call looks the address up again
  if (have_id) g_slots.push_back(Slot{id, p, n});
  *ptr = p;
  *sms = n;
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
  if (e != cudaSuccess) {
    cudaGetLastError();
    put_err(err, err_len, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return UC_ECUDA;
  }
  std::string msg;
  void* scratch = nullptr;
  int sms = 0;
  uc_status s = setup_context(dev, &scratch, &sms, msg);
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
