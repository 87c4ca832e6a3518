// uc_capi.cu — the extern "C" boundary of libuc.so (declared in include/uc.h).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/uc.h"
#include "uc_pipeline.h"

struct uc_ctx {
  uc::Env env;
  // host-path device buffers (grow only)
  char* io_text = nullptr;
  size_t io_text_cap = 0;
  char* io_out = nullptr;
  size_t io_out_cap = 0;
  // uc_compact_host_many: the upload stream and its completion event
  cudaStream_t up_stream = nullptr;
  cudaEvent_t up_done = nullptr;
  // host jobs beyond the device budget (uc_ctx_set_streaming)
  int stream_mode = UC_STREAM_AUTO;
  uint64_t stream_chunk_lines = 0, stream_group_copies = 0;
};

struct uc_job {
  uc_ctx* ctx = nullptr;
  uc_status status = UC_OK;
  char* result = nullptr;
  size_t len = 0;
  uc_stats stats{};
  int done = 0;
};

namespace {

uc_status as_status(int r) { return static_cast<uc_status>(r); }

uc_status cuda_fail(uc_ctx* c, cudaError_t e, const char* what) {
  cudaGetLastError();
  c->env.err = std::string(what) + ": " + cudaGetErrorString(e);
  return UC_ECUDA;
}


uc_status set_device(uc_ctx* c) {
  const cudaError_t e = cudaSetDevice(c->env.device);
  return e == cudaSuccess ? UC_OK : cuda_fail(c, e, "cudaSetDevice");
}

uc_status grow(uc_ctx* c, char** buf, size_t* cap, size_t want) {
  if (*cap >= want) return UC_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  const size_t sz = want + (want >> 4) + 4096;
  const cudaError_t e = c->env.dev_malloc(reinterpret_cast<void**>(buf), sz);
  if (e != cudaSuccess) {
    *buf = nullptr;
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      c->env.err = "cudaMalloc of " + std::to_string(sz >> 20) + " MiB (job buffers) failed";
      return UC_ENOMEM;
    }
    return cuda_fail(c, e, "cudaMalloc (job buffers)");
  }
  *cap = sz;
  return UC_OK;
}

// Host text in, host lines out (synchronous).
uc_status run_resident(uc_ctx* c, const char* text, size_t bytes, int k, int l, char** out_owned,
                       char* out_user, size_t out_cap, size_t* out_len, uc_stats* st);

// The streamed path (uc::compact_streamed) from host text into dst (out_user,
// or a buffer of the output bound allocated here).
uc_status run_streamed(uc_ctx* c, const char* text, size_t bytes, int k, int l, char** out_owned,
                       char* out_user, size_t out_cap, size_t* out_len, uc_stats* st) {
  // the device copies of the in-memory path are not used here
  if (c->io_text) cudaFree(c->io_text);
  if (c->io_out) cudaFree(c->io_out);
  c->io_text = c->io_out = nullptr;
  c->io_text_cap = c->io_out_cap = 0;
  const uint64_t bound = uc::output_bound(bytes, k);
  char* dst = out_user;
  size_t cap = out_cap;
  if (!dst) {
    dst = static_cast<char*>(std::malloc(bound ? bound : 1));
    if (!dst) {
      c->env.err = "host malloc of the result failed";
      return UC_ENOMEM;
    }
    cap = bound;
  }
  uint64_t ob = 0;
  const int r = uc::compact_streamed(c->env, text, bytes, k, l, dst, cap, ob, st, c->stream_chunk_lines,
                                     c->stream_group_copies);
  if (r) {
    if (!out_user) std::free(dst);
    return as_status(r);
  }
  if (out_owned) *out_owned = dst;
  *out_len = ob;
  return UC_OK;
}

uc_status run_host(uc_ctx* c, const char* text, size_t bytes, int k, int l, char** out_owned,
                   char* out_user, size_t out_cap, size_t* out_len, uc_stats* st) {
  uc_status s = set_device(c);
  if (s) return s;
  if (c->stream_mode == UC_STREAM_ALWAYS) return run_streamed(c, text, bytes, k, l, out_owned, out_user, out_cap,
                                                               out_len, st);
  s = run_resident(c, text, bytes, k, l, out_owned, out_user, out_cap, out_len, st);
  // a job whose arrays do not fit the device (or its budget) beside its
  // text and lines runs streamed, when the text has the fixed line layout
  if ((s == UC_EBUDGET || s == UC_ENOMEM) && c->stream_mode == UC_STREAM_AUTO && !c->env.sorted) {
    const std::string why = c->env.err;
    c->env.reset();
    s = run_streamed(c, text, bytes, k, l, out_owned, out_user, out_cap, out_len, st);
    if (s) c->env.err = why + "; streamed: " + c->env.err;
  }
  return s;
}

uc_status run_resident(uc_ctx* c, const char* text, size_t bytes, int k, int l, char** out_owned,
                       char* out_user, size_t out_cap, size_t* out_len, uc_stats* st) {
  uc_status s = grow(c, &c->io_text, &c->io_text_cap, bytes + 64);
  if (s) return s;
  const uint64_t bound = uc::output_bound(bytes, k);
  s = grow(c, &c->io_out, &c->io_out_cap, bound);
  if (s) return s;
  cudaError_t e = cudaMemcpyAsync(c->io_text, text, bytes, cudaMemcpyHostToDevice, c->env.stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMemcpyAsync H2D");
  uint64_t ob = 0;
  const int r = uc::compact_device(c->env, c->io_text, bytes, k, l, c->io_out, bound, ob, st);
  if (r) return as_status(r);
  char* dst = out_user;
  if (!dst) {
    dst = static_cast<char*>(std::malloc(ob ? ob : 1));
    if (!dst) {
      c->env.err = "host malloc of the result failed";
      return UC_ENOMEM;
    }
  } else if (ob > out_cap) {
    c->env.err = "result buffer too small";
    return UC_EINPUT;
  }
  if (ob) {
    e = cudaMemcpyAsync(dst, c->io_out, ob, cudaMemcpyDeviceToHost, c->env.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->env.stream);
    if (e != cudaSuccess) {
      if (!out_user) std::free(dst);
      return cuda_fail(c, e, "cudaMemcpyAsync D2H");
    }
  }
  if (out_owned) *out_owned = dst;
  *out_len = ob;
  return UC_OK;
}

}  // namespace

extern "C" {

const char* uc_status_str(uc_status s) {
  switch (s) {
    case UC_OK: return "ok";
    case UC_EINPUT: return "invalid input";
    case UC_ENOMEM: return "out of memory";
    case UC_EBUDGET: return "HBM budget exceeded";
    case UC_ETIMEOUT: return "device wait timed out";
    case UC_EINTERNAL: return "internal error";
    case UC_ECUDA: return "CUDA error";
    case UC_EBUSY: return "job not finished";
  }
  return "unknown status";
}

uc_status uc_ctx_create(int device, size_t hbm_budget, uc_ctx** out) {
  if (!out) return UC_EINPUT;
  *out = nullptr;
  uc_ctx* c = new (std::nothrow) uc_ctx();
  if (!c) return UC_ENOMEM;
  c->env.device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    delete c;
    cudaGetLastError();
    return UC_ECUDA;
  }
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, device);
  c->env.sm_count = prop.multiProcessorCount;
  c->env.smem_optin = int(prop.sharedMemPerBlockOptin);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  c->env.budget = hbm_budget ? hbm_budget : size_t(double(fr) * 0.9);
  e = cudaStreamCreateWithFlags(&c->env.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&c->env.ctr, sizeof(uc::Counters));
  if (e == cudaSuccess) e = cudaMallocHost(&c->env.h_ctr, sizeof(uc::Counters));
  for (int i = 0; i < uc::Env::NEV && e == cudaSuccess; ++i) e = cudaEventCreate(&c->env.ev[i]);
  if (e != cudaSuccess) {
    cudaGetLastError();
    uc_ctx_destroy(c);
    return UC_ECUDA;
  }
  c->env.own_stream = true;
  *out = c;
  return UC_OK;
}

uc_status uc_ctx_destroy(uc_ctx* c) {
  if (!c) return UC_OK;
  cudaSetDevice(c->env.device);
  if (c->env.stream) cudaStreamSynchronize(c->env.stream);
  for (auto& a : c->env.ar)
    if (a.base) cudaFree(a.base);
  if (c->env.big_buf) cudaFree(c->env.big_buf);
  if (c->env.jbuf) cudaFree(c->env.jbuf);
  for (auto& g : c->env.gexec)
    if (g) cudaGraphExecDestroy(g);
  if (c->env.gstream) cudaStreamDestroy(c->env.gstream);
  if (c->io_text) cudaFree(c->io_text);
  if (c->io_out) cudaFree(c->io_out);
  if (c->up_done) cudaEventDestroy(c->up_done);
  if (c->up_stream) cudaStreamDestroy(c->up_stream);
  if (c->env.ctr) cudaFree(c->env.ctr);
  if (c->env.h_ctr) cudaFreeHost(c->env.h_ctr);
  for (int i = 0; i < uc::Env::NEV; ++i)
    if (c->env.ev[i]) cudaEventDestroy(c->env.ev[i]);
  if (c->env.own_stream && c->env.stream) cudaStreamDestroy(c->env.stream);
  delete c;
  return UC_OK;
}

uc_status uc_ctx_set_stream(uc_ctx* c, void* stream) {
  if (!c) return UC_EINPUT;
  if (c->env.own_stream && c->env.stream) {
    cudaStreamSynchronize(c->env.stream);
    cudaStreamDestroy(c->env.stream);
  }
  c->env.stream = static_cast<cudaStream_t>(stream);
  c->env.own_stream = false;
  return UC_OK;
}

uc_status uc_ctx_sync(uc_ctx* c) {
  if (!c) return UC_EINPUT;
  const cudaError_t e = cudaStreamSynchronize(c->env.stream);
  return e == cudaSuccess ? UC_OK : cuda_fail(c, e, "cudaStreamSynchronize");
}

uc_status uc_ctx_set_sorted_output(uc_ctx* c, int on) {
  if (!c) return UC_EINPUT;
  c->env.sorted = on != 0;
  return UC_OK;
}

uc_status uc_ctx_set_tuning(uc_ctx* c, const uc_tuning* t) {
  if (!c || !t) return UC_EINPUT;
  if (t->tile_capacity && (t->tile_capacity < 256 || t->tile_capacity > 8192)) {
    c->env.err = "tile_capacity must be in [256, 8192]";
    return UC_EINPUT;
  }
  if (t->tile_threads && t->tile_threads != 256 && t->tile_threads != 512) {
    c->env.err = "tile_threads must be 256 or 512";
    return UC_EINPUT;
  }
  if (t->contract_method != UC_CONTRACT_POINTER_JUMP && t->contract_method != UC_CONTRACT_HEC) {
    c->env.err = "contract_method must be UC_CONTRACT_POINTER_JUMP or UC_CONTRACT_HEC";
    return UC_EINPUT;
  }
  if (t->warp_capacity > 1 && (t->warp_capacity < 32 || t->warp_capacity > 1024 || t->warp_capacity % 32)) {
    c->env.err = "warp_capacity must be 0, 1 or a multiple of 32 in [32, 1024]";
    return UC_EINPUT;
  }
  if (t->load_factor_pct && (t->load_factor_pct < 150 || t->load_factor_pct > 800)) {
    c->env.err = "load_factor_pct must be 0 or in [150, 800]";
    return UC_EINPUT;
  }
  if (t->bucket_fill > 64) {
    c->env.err = "bucket_fill must be 0 or in [1, 64]";
    return UC_EINPUT;
  }
  if (t->bucket_bits > 25) {
    c->env.err = "bucket_bits must be <= 25";
    return UC_EINPUT;
  }
  c->env.tune = *t;
  return UC_OK;
}

uc_status uc_ctx_get_tuning(const uc_ctx* c, uc_tuning* t) {
  if (!c || !t) return UC_EINPUT;
  *t = c->env.tune;
  return UC_OK;
}

uc_status uc_ctx_set_streaming(uc_ctx* c, int mode, uint64_t chunk_lines, uint64_t group_copies) {
  if (!c) return UC_EINPUT;
  if (mode != UC_STREAM_AUTO && mode != UC_STREAM_ALWAYS && mode != UC_STREAM_NEVER) {
    c->env.err = "mode must be UC_STREAM_AUTO, UC_STREAM_ALWAYS or UC_STREAM_NEVER";
    return UC_EINPUT;
  }
  c->stream_mode = mode;
  c->stream_chunk_lines = chunk_lines;
  c->stream_group_copies = group_copies;
  return UC_OK;
}

uc_status uc_ctx_set_faults(uc_ctx* c, const uc_faults* f) {
  if (!c || !f) return UC_EINPUT;
  c->env.faults = *f;
  return UC_OK;
}

const char* uc_last_error(const uc_ctx* c) { return c ? c->env.err.c_str() : "no context"; }

uc_status uc_parse_header(uc_ctx* c, const char* d_text, size_t bytes, uint64_t* n, uint64_t* body) {
  if (!c || !d_text || !n || !body) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  return as_status(uc::parse_header(c->env, d_text, bytes, *n, *body));
}

uc_status uc_pack(uc_ctx* c, const char* d_text, size_t bytes, int k, uint64_t* d_keys, uint64_t* n_out) {
  if (!c || !d_text || !n_out) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  c->env.reset();
  uint64_t n = 0;
  int r = uc::pack(c->env, d_text, bytes, k, d_keys, n);
  c->env.reset();
  *n_out = n;
  return as_status(r);
}

uc_status uc_minimizers(uc_ctx* c, const uint64_t* d_keys, uint64_t n, int k, int l, uint64_t seed,
                        const uint32_t* d_table, uint32_t* d_l1, uint32_t* d_l2) {
  if (!c || (n && (!d_keys || !d_l1 || !d_l2))) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  return as_status(uc::minimizers(c->env, d_keys, n, k, l, seed, d_table, d_l1, d_l2));
}

uc_status uc_find_edges(uc_ctx* c, const uint64_t* d_keys, uint64_t n, int k, int l, uint64_t seed,
                        uint32_t* d_succ, uint32_t* d_pred) {
  if (!c || (n && (!d_keys || !d_succ || !d_pred))) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  c->env.reset();
  const int r = uc::find_edges(c->env, d_keys, n, k, l, seed, d_succ, d_pred);
  c->env.reset();
  return as_status(r);
}

uc_status uc_contract(uc_ctx* c, const uint64_t* d_keys, const uint32_t* d_succ, const uint32_t* d_pred,
                      uint64_t n, int k, int method, uint32_t* d_head, uint32_t* d_rank, uint64_t* n_cycles) {
  if (!c || (n && (!d_keys || !d_succ || !d_pred || !d_head || !d_rank))) return UC_EINPUT;
  if (method != UC_CONTRACT_POINTER_JUMP && method != UC_CONTRACT_HEC) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  c->env.reset();
  uint64_t cyc = 0;
  const int r = uc::contract(c->env, d_keys, d_succ, d_pred, n, k, method, d_head, d_rank, cyc);
  c->env.reset();
  if (n_cycles) *n_cycles = cyc;
  return as_status(r);
}

uc_status uc_emit(uc_ctx* c, const uint64_t* d_keys, const uint32_t* d_succ, const uint32_t* d_head,
                  const uint32_t* d_rank, uint64_t n, int k, char* d_out, uint64_t cap, uint64_t* out_bytes) {
  if (!c || !out_bytes || (n && (!d_keys || !d_head || !d_rank))) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  c->env.reset();
  uint64_t ob = 0;
  const int r = uc::emit(c->env, d_keys, d_succ, d_head, d_rank, n, k, d_out, cap, ob);
  c->env.reset();
  *out_bytes = ob;
  return as_status(r);
}

uint64_t uc_output_bound(size_t text_bytes, int k) { return uc::output_bound(text_bytes, k); }

uc_status uc_compact_device(uc_ctx* c, const char* d_text, size_t bytes, int k, int l, char* d_out, uint64_t cap,
                            uint64_t* out_bytes, uc_stats* stats) {
  if (!c || !d_text || !d_out || !out_bytes) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  uint64_t ob = 0;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  const int r = uc::compact_device(c->env, d_text, bytes, k, l, d_out, cap, ob, stats);
  c->env.reset();
  *out_bytes = ob;
  return as_status(r);
}

// ---- autotuner --------------------------------------------------------

namespace {

struct Knob {
  uint32_t uc_tuning::*field;
  std::vector<uint32_t> values;
};

bool tuning_valid(const uc_tuning& t) {
  return t.warp_capacity <= 1 || t.warp_capacity <= t.tile_capacity;
}

}  // namespace

uc_status uc_autotune(uc_ctx* c, const char* d_text, size_t bytes, int k, int l, int reps, uint32_t max_ms,
                      uc_tuning* best, float* best_ms, uint32_t* trials) {
  if (!c || !d_text || !best) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  const uint64_t bound = uc::output_bound(bytes, k);
  s = grow(c, &c->io_out, &c->io_out_cap, bound);
  if (s) return s;
  if (reps < 1) reps = 3;
  const double limit = max_ms ? double(max_ms) : 60000.0;
  const uc_tuning saved = c->env.tune;
  double spent = 0.0;
  uint32_t n_trials = 0;
  uint64_t ref_bytes = 0;
  bool have_ref = false;
  // median device time of reps runs after one warm-up run
  auto time_one = [&](const uc_tuning& t, float& ms) -> int {
    c->env.tune = t;
    uint64_t ob = 0;
    uc_stats st{};
    int r = uc::compact_device(c->env, d_text, bytes, k, l, c->io_out, bound, ob, &st);
    c->env.reset();
    if (r) return r;
    spent += st.ms_total;
    std::vector<float> v;
    for (int i = 0; i < reps; ++i) {
      r = uc::compact_device(c->env, d_text, bytes, k, l, c->io_out, bound, ob, &st);
      c->env.reset();
      if (r) return r;
      v.push_back(st.ms_total);
      spent += st.ms_total;
    }
    std::sort(v.begin(), v.end());
    ms = v[v.size() / 2];
    ++n_trials;
    if (!have_ref) {
      ref_bytes = ob;
      have_ref = true;
    } else if (ob != ref_bytes) {
      c->env.err = "autotune: a candidate tuning produced a different output size";
      return UC_EINTERNAL;
    }
    return UC_OK;
  };
  uc_tuning cur{};
  cur.tile_capacity = 4096;
  cur.tile_threads = 512;
  cur.load_factor_pct = 200;
  cur.contract_method = UC_CONTRACT_POINTER_JUMP;
  cur.warp_capacity = 256;
  cur.bucket_fill = 8;
  float cur_ms = 0.f;
  int r = time_one(cur, cur_ms);
  if (r) {
    c->env.tune = saved;
    return as_status(r);
  }
  const Knob knobs[] = {
      {&uc_tuning::warp_capacity, {1, 64, 128, 256, 512}},
      {&uc_tuning::bucket_fill, {2, 4, 8, 16, 32}},
      {&uc_tuning::tile_capacity, {1024, 2048, 4096, 8192}},
      {&uc_tuning::tile_threads, {256, 512}},
      {&uc_tuning::load_factor_pct, {150, 200, 300, 400}},
      {&uc_tuning::contract_method, {UC_CONTRACT_POINTER_JUMP, UC_CONTRACT_HEC}},
  };
  // coordinate descent: each knob in turn over its values, the others held;
  // a change must win by 1% to be kept; stop after a pass with no change
  for (int pass = 0; pass < 3 && spent < limit; ++pass) {
    bool changed = false;
    for (const Knob& kn : knobs) {
      for (uint32_t v : kn.values) {
        if (spent >= limit) break;
        if (cur.*(kn.field) == v) continue;
        uc_tuning cand = cur;
        cand.*(kn.field) = v;
        if (!tuning_valid(cand)) continue;
        float ms = 0.f;
        r = time_one(cand, ms);
        if (r == UC_EINTERNAL || r == UC_ECUDA) {
          c->env.tune = saved;
          return as_status(r);
        }
        if (r) continue;  // a candidate that does not fit (budget, shared memory) is skipped
        if (ms < cur_ms * 0.99f) {
          cur = cand;
          cur_ms = ms;
          changed = true;
        }
      }
    }
    if (!changed) break;
  }
  c->env.tune = cur;
  *best = cur;
  if (best_ms) *best_ms = cur_ms;
  if (trials) *trials = n_trials;
  return UC_OK;
}

uint64_t uc_batch_output_bound(int njobs, const size_t* bytes, int k) {
  uint64_t t = 0;
  for (int j = 0; j < njobs; ++j) t += (uc::output_bound(bytes[j], k) + 15) & ~uint64_t(15);
  return t;
}

uc_status uc_compact_batch(uc_ctx* c, int njobs, const char* const* d_texts, const size_t* bytes, int k, int l,
                           char* d_out, uint64_t out_cap, uint64_t* out_off, uint64_t* out_len, uc_stats* stats) {
  if (!c || njobs < 0 || (njobs > 0 && (!d_texts || !bytes || !d_out || !out_off || !out_len))) return UC_EINPUT;
  uc_status s = set_device(c);
  if (s) return s;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  int r = uc::compact_batch(c->env, uint32_t(njobs), d_texts, bytes, k, l, d_out, out_cap, out_off, out_len, stats);
  c->env.reset();
  if (r == UC_EINPUT) {
    // a job with another line layout, or a malformed one: compact the jobs
    // one by one, so that a malformed job is named
    uint64_t base = 0;
    for (int j = 0; j < njobs; ++j) {
      const uint64_t cap = uc::output_bound(bytes[j], k);
      uint64_t ob = 0;
      uc_stats one{};
      r = uc::compact_device(c->env, d_texts[j], bytes[j], k, l, d_out + base, cap, ob, stats ? &one : nullptr);
      c->env.reset();
      if (r) {
        c->env.err = "job " + std::to_string(j) + ": " + c->env.err;
        return as_status(r);
      }
      out_off[j] = base;
      out_len[j] = ob;
      if (stats) {
        stats->n_kmers += one.n_kmers;
        stats->out_bytes += one.out_bytes;
        stats->ms_total += one.ms_total;
      }
      base += (cap + 15) & ~uint64_t(15);
    }
    return UC_OK;
  }
  return as_status(r);
}

uc_status uc_compact_host(uc_ctx* c, const char* text, size_t bytes, int k, int l, char* out, size_t cap,
                          size_t* out_bytes, uc_stats* stats) {
  if (!c || !text || !out || !out_bytes) return UC_EINPUT;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  return run_host(c, text, bytes, k, l, nullptr, out, cap, out_bytes, stats);
}

uc_status uc_compact_host_many(uc_ctx* c, int njobs, const char* const* texts, const size_t* bytes, int k, int l,
                               char* const* outs, const size_t* caps, size_t* out_lens, uc_stats* stats) {
  if (!c || njobs < 0 || (njobs > 0 && (!texts || !bytes || !outs || !caps || !out_lens))) return UC_EINPUT;
  if (njobs == 0) return UC_OK;
  uc_status s = set_device(c);
  if (s) return s;
  size_t tmax = 0;
  uint64_t omax = 0;
  for (int j = 0; j < njobs; ++j) {
    if (!texts[j] && bytes[j]) return UC_EINPUT;
    tmax = std::max(tmax, bytes[j]);
    omax = std::max<uint64_t>(omax, uc::output_bound(bytes[j], k));
  }
  s = grow(c, &c->io_text, &c->io_text_cap, tmax + 64);
  if (s) return s;
  s = grow(c, &c->io_out, &c->io_out_cap, omax);
  if (s) return s;
  cudaError_t e = cudaSuccess;
  if (!c->up_stream) e = cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess && !c->up_done) e = cudaEventCreateWithFlags(&c->up_done, cudaEventDisableTiming);
  if (e != cudaSuccess) return cuda_fail(c, e, "upload stream");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  // job 0's text goes up first; every later one goes up while the job before
  // it is past its pack phase (its text is dead then), on the upload stream
  e = cudaMemcpyAsync(c->io_text, texts[0], bytes[0], cudaMemcpyHostToDevice, c->up_stream);
  if (e == cudaSuccess) e = cudaEventRecord(c->up_done, c->up_stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMemcpyAsync H2D");
  uc_status result = UC_OK;
  cudaError_t hook_err = cudaSuccess;
  for (int j = 0; j < njobs && result == UC_OK; ++j) {
    e = cudaStreamWaitEvent(c->env.stream, c->up_done, 0);
    if (e != cudaSuccess) {
      result = cuda_fail(c, e, "cudaStreamWaitEvent");
      break;
    }
    const int nxt = j + 1;
    c->env.after_pack = [&, nxt] {
      if (nxt >= njobs) return;
      cudaError_t he = cudaStreamWaitEvent(c->up_stream, c->env.ev[1], 0);
      if (he == cudaSuccess)
        he = cudaMemcpyAsync(c->io_text, texts[nxt], bytes[nxt], cudaMemcpyHostToDevice, c->up_stream);
      if (he == cudaSuccess) he = cudaEventRecord(c->up_done, c->up_stream);
      if (he != cudaSuccess && hook_err == cudaSuccess) hook_err = he;
    };
    uint64_t ob = 0;
    uc_stats one{};
    const int r = uc::compact_device(c->env, c->io_text, bytes[j], k, l, c->io_out, omax, ob, &one);
    c->env.after_pack = nullptr;
    if (r) {
      result = as_status(r);
      break;
    }
    if (hook_err != cudaSuccess) {
      result = cuda_fail(c, hook_err, "cudaMemcpyAsync H2D (next job)");
      break;
    }
    if (ob > caps[j]) {
      c->env.err = "result buffer of job " + std::to_string(j) + " too small";
      result = UC_EINPUT;
      break;
    }
    if (ob) {
      // stream order keeps the next job from writing io_out before this copy
      e = cudaMemcpyAsync(outs[j], c->io_out, ob, cudaMemcpyDeviceToHost, c->env.stream);
      if (e != cudaSuccess) {
        result = cuda_fail(c, e, "cudaMemcpyAsync D2H");
        break;
      }
    }
    out_lens[j] = ob;
    if (stats) {
      stats->n_kmers += one.n_kmers;
      stats->out_bytes += ob;
      stats->ms_total += one.ms_total;
      stats->launches += one.launches;
    }
  }
  // the uploads and copies still in flight finish before return
  const cudaError_t e1 = cudaStreamSynchronize(c->up_stream);
  const cudaError_t e2 = cudaStreamSynchronize(c->env.stream);
  if (result == UC_OK && e1 != cudaSuccess) result = cuda_fail(c, e1, "cudaStreamSynchronize");
  if (result == UC_OK && e2 != cudaSuccess) result = cuda_fail(c, e2, "cudaStreamSynchronize");
  return result;
}

uc_status uc_job_submit(uc_ctx* c, const char* text, size_t bytes, int k, int l, uc_job** job) {
  if (!c || !text || !job) return UC_EINPUT;
  uc_job* j = new (std::nothrow) uc_job();
  if (!j) return UC_ENOMEM;
  j->ctx = c;
  j->status = run_host(c, text, bytes, k, l, &j->result, nullptr, 0, &j->len, &j->stats);
  j->done = 1;
  *job = j;
  return j->status;
}

uc_status uc_job_poll(uc_job* j, int* done) {
  if (!j || !done) return UC_EINPUT;
  *done = j->done;
  return UC_OK;
}

uc_status uc_job_wait(uc_job* j) { return j ? j->status : UC_EINPUT; }

uc_status uc_job_result(uc_job* j, char** buf, size_t* len, uc_stats* stats) {
  if (!j || !buf || !len) return UC_EINPUT;
  if (!j->done) return UC_EBUSY;
  if (j->status) return j->status;
  *buf = j->result;
  *len = j->len;
  j->result = nullptr;
  if (stats) *stats = j->stats;
  return UC_OK;
}

uc_status uc_job_release(uc_job* j) {
  if (!j) return UC_OK;
  std::free(j->result);
  delete j;
  return UC_OK;
}

void uc_free(void* p) { std::free(p); }

uc_status uc_compact_file(uc_ctx* c, const char* in_path, int k, int l, const char* out_path, uc_stats* stats) {
  if (!c || !in_path || !out_path) return UC_EINPUT;
  FILE* f = std::fopen(in_path, "rb");
  if (!f) {
    c->env.err = std::string("could not open input file ") + in_path;
    return UC_EINPUT;
  }
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  char* text = nullptr;
  if (cudaMallocHost(&text, size_t(sz > 0 ? sz : 1)) != cudaSuccess) {
    cudaGetLastError();
    std::fclose(f);
    c->env.err = "pinned host buffer for the input";
    return UC_ENOMEM;
  }
  const size_t got = sz > 0 ? std::fread(text, 1, size_t(sz), f) : 0;
  std::fclose(f);
  if (got != size_t(sz > 0 ? sz : 0)) {
    cudaFreeHost(text);
    c->env.err = "short read of the input file";
    return UC_EINPUT;
  }
  char* out = nullptr;
  const size_t cap = size_t(uc::output_bound(got, k));
  if (cudaMallocHost(&out, cap) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeHost(text);
    c->env.err = "pinned host buffer for the output";
    return UC_ENOMEM;
  }
  size_t ob = 0;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  uc_status s = run_host(c, text, got, k, l, nullptr, out, cap, &ob, stats);
  cudaFreeHost(text);
  if (s == UC_OK) {
    FILE* o = std::fopen(out_path, "ab");  // append, as write_to_f does
    if (!o) {
      c->env.err = std::string("could not open output file ") + out_path;
      s = UC_EINPUT;
    } else {
      if (ob && std::fwrite(out, 1, ob, o) != ob) {
        c->env.err = "short write of the output file";
        s = UC_EINPUT;
      }
      std::fclose(o);
    }
  }
  cudaFreeHost(out);
  return s;
}

}  // extern "C"
