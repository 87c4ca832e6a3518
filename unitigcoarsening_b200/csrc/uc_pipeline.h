// uc_pipeline.h — host-side pipeline entry points used by the C ABI.
#pragma once
#include <cstdint>
#include <functional>
#include <string>

#include <cuda_runtime.h>

#include "../../include/uc.h"
#include "uc_kernels.cuh"

namespace uc {

// Grow-only device scratch region.
struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  size_t used = 0;
};

// Per-context state: stream, device scratch arenas, counters, tuning.
struct Env {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 148;
  int smem_optin = 232448;  // max dynamic shared memory per block
  size_t budget = 0;
  Arena ar[2];              // 0: per-k-mer arrays, 1: copies/segments/scratch
  char* big_buf = nullptr;  // scratch of oversized tiles (grow only)
  size_t big_cap = 0;
  char* jbuf = nullptr;     // job table and per-job counters (grow only)
  size_t jcap = 0;
  Counters* ctr = nullptr;    // device
  Counters* h_ctr = nullptr;  // pinned host mirror
  static constexpr int NEV = 10;
  cudaEvent_t ev[NEV] = {};
  bool tiles_timed = false;  // ev[8]/ev[9]/ev[5] bracket the warp and block tile kernels
  uc_tuning tune{};
  uint64_t seed = 0x00C0FFEE5EEDull;
  uint32_t launches = 0;    // kernels launched by the last call
  uint32_t graph_nodes = 0; // of which inside CUDA graphs
  // instantiated graphs of the contraction rounds, reused while the round
  // count (the graph's shape) stays the same
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  uint64_t gkey[2] = {0, 0};
  bool use_graphs = true;
  cudaStream_t gstream = nullptr;  // capture stream when the caller's stream is the legacy one
  // pool mode (serving): the arenas are fixed slices of a device pool that a
  // server owns; they never grow, and oversized-tile scratch comes from the
  // back arena's free end
  bool pool = false;
  // whole-job calls (compact_device and the paths built on it) leave the
  // lines in byte order
  bool sorted = false;
  // called by the fused path once the pack kernels are enqueued and ev[1]
  // recorded after them: from then on the job's text is no longer read, so
  // a host pipeline can upload the next job's text into the same buffer
  std::function<void()> after_pack;
  // failure injection (uc_ctx_set_faults); zeros = off
  uc_faults faults{};
  std::string err;

  int fail(int code, const std::string& msg);
  // Every device allocation of a context goes through here, so that
  // faults.fail_alloc_after can make one fail as out of memory.
  cudaError_t dev_malloc(void** p, size_t bytes);
  void* take(int arena, size_t bytes);
  // Make an arena hold `bytes`; only while nothing is taken from it.
  int reserve(int arena, size_t bytes);
  void reset() { ar[0].used = ar[1].used = 0; }
  int read_ctr();
  int check_err(const Counters* h);
};

int parse_header(Env& e, const char* d_text, size_t bytes, uint64_t& n, uint64_t& body);
int pack(Env& e, const char* d_text, size_t bytes, int k, uint64_t* d_keys, uint64_t& n_out);
int minimizers(Env& e, const uint64_t* d_keys, uint64_t n, int k, int l, uint64_t seed,
               const uint32_t* d_table, uint32_t* l1, uint32_t* l2);
int find_edges(Env& e, const uint64_t* d_keys, uint64_t n, int k, int l, uint64_t seed,
               uint32_t* succ, uint32_t* pred);
int contract(Env& e, const uint64_t* d_keys, const uint32_t* succ, const uint32_t* pred, uint64_t n,
             int k, int method, uint32_t* head, uint32_t* rank, uint64_t& ncyc);
int emit(Env& e, const uint64_t* d_keys, const uint32_t* succ, const uint32_t* head,
         const uint32_t* rank, uint64_t n, int k, char* out, uint64_t cap, uint64_t& out_bytes);
int compact_device(Env& e, const char* d_text, size_t bytes, int k, int l, char* out, uint64_t cap,
                   uint64_t& out_bytes, uc_stats* st);
int compact_batch(Env& e, uint32_t njobs, const char* const* texts, const size_t* bytes, int k, int l, char* out,
                  uint64_t out_cap, uint64_t* out_off, uint64_t* out_len, uc_stats* st);
uint64_t output_bound(size_t text_bytes, int k);
// The fused path for one job from host memory in chunks of chunk_lines lines
// (two passes over the text) and tile groups of about group_copies copies,
// for jobs whose text and lines exceed the device budget (0 = defaults).
int compact_streamed(Env& e, const char* h_text, size_t bytes, int k, int l, char* h_out, uint64_t cap,
                     uint64_t& out_bytes, uc_stats* st, uint64_t chunk_lines, uint64_t group_copies);
// Reorder the lines of out[0, bytes) into byte order in place (scratch from
// the back arena).
int sort_lines(Env& e, char* out, uint64_t bytes, int k);
// Upper bound of the front and back arena bytes (reserve slack included)
// that compact_batch needs for these jobs under the current tuning, from the
// text sizes alone: every line holds at least k+1 bytes and at most every
// k-mer is a cross k-mer.
void batch_footprint(const Env& e, uint32_t njobs, const size_t* bytes, int k, int l, size_t& front, size_t& back);
// emit() over caller-provided device scratch of emit_scratch_bytes(n) bytes
// (256-byte aligned) on stream s: the same kernels, no allocation.  Clears
// the member counts it needs at zero itself.
uint64_t emit_scratch_bytes(uint64_t n);
// Loads every kernel emit_in launches.  Under lazy module loading (the CUDA
// default) a kernel's module is loaded, and its device memory taken, at its
// first use; after this call emit_in needs no device memory of its own.
int emit_preload(std::string& err);
int emit_in(cudaStream_t s, int sm_count, const uint64_t* d_keys, const uint32_t* head, const uint32_t* rank,
            uint64_t n, int k, char* out, uint64_t cap, uint64_t& out_bytes, void* scratch, std::string& err);

}  // namespace uc
