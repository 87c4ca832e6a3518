// uc_server.cu — a serving loop over one GPU (uc_server_* in uc.h).
//
// Jobs (k-mer texts in host memory) arrive at any time.  One device pool of
// the configured HBM budget is allocated once; a scheduler thread admits the
// job at the head of the queue when a device lane is idle and a slice of the
// pool big enough for the job's footprint bound is free (first fit).  Small
// jobs queued behind it with the same k and l join it in one batched launch
// (compact_batch: one tile queue over all of them), so arrivals that queue up
// while the GPU is busy are served together.  Each lane is a host thread with
// its own stream, counters and cached CUDA graphs, so admitted jobs overlap
// on the device.  A lane copies its jobs' texts into the slice, runs the fused
// path, copies the lines back into host buffers and returns the slice.
//
// The reference has no serving mode; it runs one file per process
// (driver.cpp:422-662).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/uc.h"
#include "uc_pipeline.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// The count line of a k-mer text in host memory (driver.cpp:296-304).
uint64_t header_count(const char* t, size_t bytes) {
  size_t p = 0;
  while (p < bytes && (t[p] == ' ' || t[p] == '\t' || t[p] == '\r')) ++p;
  uint64_t v = 0;
  while (p < bytes && t[p] >= '0' && t[p] <= '9' && v < (1ull << 40)) v = v * 10 + uint64_t(t[p++] - '0');
  return v;
}

// First-fit allocator over the offsets of one device pool.
class PoolMap {
 public:
  explicit PoolMap(size_t cap) : cap_(cap) { free_[0] = cap; }
  bool alloc(size_t len, size_t& off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= len) {
        off = it->first;
        const size_t rest = it->second - len;
        free_.erase(it);
        if (rest) free_[off + len] = rest;
        used_ += len;
        peak_ = std::max(peak_, used_);
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t len) {
    used_ -= len;
    auto it = free_.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t cap() const { return cap_; }
  size_t peak() const { return peak_; }

 private:
  size_t cap_, used_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;
};

struct SJob {
  uint64_t id = 0;
  const char* text = nullptr;
  size_t bytes = 0;
  int k = 0, l = 0;
  uc_status status = UC_OK;
  std::string err;
  char* result = nullptr;
  size_t len = 0;
  uint64_t n_kmers = 0;
  uint32_t batch = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  bool done = false;
};

struct Work {
  std::vector<SJob*> jobs;
  size_t off = 0, len = 0;               // pool slice
  size_t text_bytes = 0, out_bytes = 0;  // its regions
  size_t front = 0, back = 0;
};

struct Lane {
  uc::Env env;
  std::thread th;
  bool busy = false;
  Work work;
  std::condition_variable cv;
};

}  // namespace

struct uc_server {
  uc_server_config cfg{};
  char* pool = nullptr;
  PoolMap* map = nullptr;
  char* hpool = nullptr;      // pinned host pool for results
  PoolMap* hmap = nullptr;
  std::map<const char*, size_t> hlen;  // result pointer -> its region length
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<SJob*> queue;
  std::map<uint64_t, SJob*> jobs;
  uint64_t next_id = 1;
  std::vector<Lane*> lanes;
  std::thread sched;
  bool stop = false;
  // totals over completed jobs
  std::vector<double> lat_ms;
  uint64_t kmers_done = 0, batches = 0, batched_jobs = 0;
  double t_first = 0, t_last = 0;
};

namespace {

// Footprint of a group of jobs: text copies, output, front and back arenas.
void group_footprint(const uc::Env& env, const std::vector<SJob*>& g, Work& w) {
  std::vector<size_t> bytes;
  w.text_bytes = 0;
  w.out_bytes = 0;
  for (SJob* j : g) {
    bytes.push_back(j->bytes);
    w.text_bytes += align256(j->bytes + 64);
  }
  const int k = g[0]->k, l = g[0]->l;
  w.out_bytes = align256(uc_batch_output_bound(int(g.size()), bytes.data(), k) + 64);
  uc::batch_footprint(env, uint32_t(g.size()), bytes.data(), k, l, w.front, w.back);
  w.front = align256(w.front);
  w.back = align256(w.back);
  w.len = w.text_bytes + w.out_bytes + w.front + w.back;
}

void finish_job(uc_server* s, SJob* j, uc_status st, const std::string& err) {
  j->status = st;
  j->err = err;
  j->t_done = now_s();
  j->done = true;
  if (st == UC_OK) {
    s->lat_ms.push_back((j->t_done - j->t_submit) * 1e3);
    s->kmers_done += j->n_kmers;
    s->t_last = std::max(s->t_last, j->t_done);
  }
}

// Host buffer of a result: a region of the pinned host pool (device to host
// copies at full speed, no page faults), else malloc when the pool is full.
char* host_result(uc_server* s, size_t len) {
  {
    std::lock_guard<std::mutex> lock(s->mu);
    size_t off = 0;
    const size_t a = align256(len);
    if (s->hmap && s->hmap->alloc(a, off)) {
      char* p = s->hpool + off;
      s->hlen[p] = a;
      return p;
    }
  }
  return static_cast<char*>(std::malloc(len));
}

// Caller holds s->mu.
void free_result_locked(uc_server* s, char* p) {
  auto it = s->hlen.find(p);
  if (it != s->hlen.end()) {
    s->hmap->release(size_t(p - s->hpool), it->second);
    s->hlen.erase(it);
  } else {
    std::free(p);
  }
}

void free_result(uc_server* s, char* p) {
  std::lock_guard<std::mutex> lock(s->mu);
  free_result_locked(s, p);
}

// Run one admitted group on a lane (lane thread, no lock held).
void run_work(uc_server* s, Lane& ln) {
  Work& w = ln.work;
  uc::Env& e = ln.env;
  char* base = s->pool + w.off;
  char* d_text = base;
  char* d_out = base + w.text_bytes;
  e.ar[0] = uc::Arena{d_out + w.out_bytes, w.front, 0};
  e.ar[1] = uc::Arena{d_out + w.out_bytes + w.front, w.back, 0};
  const uint32_t nj = uint32_t(w.jobs.size());
  std::vector<const char*> texts(nj);
  std::vector<size_t> bytes(nj);
  size_t o = 0;
  uc_status st = UC_OK;
  std::string err;
  for (uint32_t i = 0; i < nj; ++i) {
    texts[i] = d_text + o;
    bytes[i] = w.jobs[i]->bytes;
    if (bytes[i] && cudaMemcpyAsync(d_text + o, w.jobs[i]->text, bytes[i], cudaMemcpyHostToDevice, e.stream) !=
                        cudaSuccess) {
      st = UC_ECUDA;
      err = std::string("host to device copy: ") + cudaGetErrorString(cudaGetLastError());
    }
    o += align256(bytes[i] + 64);
  }
  std::vector<uint64_t> off(nj), len(nj);
  std::vector<uc_stats> jst(nj);
  std::vector<uc_status> js(nj, UC_OK);
  std::vector<std::string> jerr(nj);
  if (st == UC_OK) {
    int r = UC_OK;
    if (nj > 1) {
      uc_stats bs{};
      r = uc::compact_batch(e, nj, texts.data(), bytes.data(), w.jobs[0]->k, w.jobs[0]->l, d_out, w.out_bytes,
                            off.data(), len.data(), &bs);
      e.reset();
      if (r == UC_OK) {
        for (uint32_t i = 0; i < nj; ++i) jst[i] = bs;
      } else if (r != UC_EINPUT) {
        st = static_cast<uc_status>(r);
        err = e.err;
      }
      // an input the batched path does not take (a layout other than k
      // chars and '\n' per line) or a malformed job: every job runs alone
      // below, so that only a malformed one fails
    }
    if (st == UC_OK && (nj == 1 || r != UC_OK)) {
      // one job, or a batch that the batched path refused: each job alone,
      // one after another, in the same slice
      uint64_t pos = 0;
      for (uint32_t i = 0; i < nj; ++i) {
        uint64_t ob = 0;
        uc_stats one{};
        const uint64_t cap = uc::output_bound(bytes[i], w.jobs[i]->k);
        const int ri = uc::compact_device(e, texts[i], bytes[i], w.jobs[i]->k, w.jobs[i]->l, d_out + pos, cap, ob,
                                          &one);
        e.reset();
        js[i] = static_cast<uc_status>(ri);
        if (ri) jerr[i] = e.err;
        off[i] = pos;
        len[i] = ri ? 0 : ob;
        jst[i] = one;
        pos += (cap + 15) & ~uint64_t(15);
      }
    }
  }
  if (st == UC_OK) {
    for (uint32_t i = 0; i < nj; ++i) {
      if (js[i] != UC_OK || len[i] == 0) continue;
      char* h = host_result(s, len[i]);
      if (!h) {
        js[i] = UC_ENOMEM;
        jerr[i] = "host result buffer";
        continue;
      }
      w.jobs[i]->result = h;
      w.jobs[i]->len = len[i];
      if (cudaMemcpyAsync(h, d_out + off[i], len[i], cudaMemcpyDeviceToHost, e.stream) != cudaSuccess) {
        js[i] = UC_ECUDA;
        jerr[i] = std::string("device to host copy: ") + cudaGetErrorString(cudaGetLastError());
      }
    }
    if (cudaStreamSynchronize(e.stream) != cudaSuccess) {
      st = UC_ECUDA;
      err = std::string("cudaStreamSynchronize: ") + cudaGetErrorString(cudaGetLastError());
    }
  }
  std::lock_guard<std::mutex> lock(s->mu);
  s->map->release(w.off, w.len);
  if (nj > 1) {
    ++s->batches;
    s->batched_jobs += nj;
  }
  for (uint32_t i = 0; i < nj; ++i) {
    SJob* j = w.jobs[i];
    j->n_kmers = header_count(j->text, j->bytes);
    const uc_status fs = (st != UC_OK) ? st : js[i];
    finish_job(s, j, fs, (st != UC_OK) ? err : jerr[i]);
    if (fs != UC_OK && j->result) {
      free_result_locked(s, j->result);
      j->result = nullptr;
      j->len = 0;
    }
  }
  ln.busy = false;
  ln.work = Work{};
  s->cv_sched.notify_all();
  s->cv_done.notify_all();
}

void lane_main(uc_server* s, Lane* ln) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lock(s->mu);
  for (;;) {
    ln->cv.wait(lock, [&] { return s->stop || !ln->work.jobs.empty(); });
    if (ln->work.jobs.empty()) return;  // stopping and idle
    lock.unlock();
    run_work(s, *ln);
    lock.lock();
  }
}

void sched_main(uc_server* s) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lock(s->mu);
  for (;;) {
    if (s->stop) return;
    Lane* idle = nullptr;
    for (Lane* ln : s->lanes)
      if (!ln->busy) {
        idle = ln;
        break;
      }
    if (s->queue.empty() || !idle) {
      s->cv_sched.wait(lock);
      continue;
    }
    SJob* h = s->queue.front();
    std::vector<SJob*> g{h};
    Work w;
    group_footprint(idle->env, g, w);
    if (w.len > s->map->cap()) {
      s->queue.pop_front();
      finish_job(s, h, UC_EBUDGET, "job footprint " + std::to_string(w.len >> 20) + " MiB exceeds the pool");
      s->cv_done.notify_all();
      continue;
    }
    // continuous batching: small jobs queued behind the head with the same
    // k and l join its launch while the group's footprint still fits
    std::vector<size_t> picked;
    if (h->bytes <= s->cfg.batch_bytes && s->cfg.max_batch > 1) {
      for (size_t qi = 1; qi < s->queue.size() && g.size() < size_t(s->cfg.max_batch); ++qi) {
        SJob* j = s->queue[qi];
        if (j->k != h->k || j->l != h->l || j->bytes > s->cfg.batch_bytes) continue;
        g.push_back(j);
        Work w2;
        group_footprint(idle->env, g, w2);
        size_t probe = 0;
        if (w2.len <= s->map->cap() && s->map->alloc(w2.len, probe)) {
          s->map->release(probe, w2.len);
          w = w2;
          picked.push_back(qi);
        } else {
          g.pop_back();
          break;
        }
      }
    }
    if (!s->map->alloc(w.len, w.off)) {
      if (g.size() > 1) {  // fall back to the head alone
        g.resize(1);
        picked.clear();
        group_footprint(idle->env, g, w);
        if (!s->map->alloc(w.len, w.off)) {
          s->cv_sched.wait(lock);  // memory frees when a lane finishes
          continue;
        }
      } else {
        s->cv_sched.wait(lock);
        continue;
      }
    }
    for (auto it = picked.rbegin(); it != picked.rend(); ++it) s->queue.erase(s->queue.begin() + long(*it));
    s->queue.pop_front();
    const double t = now_s();
    for (SJob* j : g) {
      j->t_admit = t;
      j->batch = uint32_t(g.size());
    }
    w.jobs = g;
    idle->work = w;
    idle->busy = true;
    idle->cv.notify_one();
  }
}

void destroy_lane_env(uc::Env& e) {
  if (e.stream) cudaStreamSynchronize(e.stream);
  for (auto& g : e.gexec)
    if (g) cudaGraphExecDestroy(g);
  if (e.gstream) cudaStreamDestroy(e.gstream);
  if (e.jbuf) cudaFree(e.jbuf);
  if (e.ctr) cudaFree(e.ctr);
  if (e.h_ctr) cudaFreeHost(e.h_ctr);
  for (int i = 0; i < uc::Env::NEV; ++i)
    if (e.ev[i]) cudaEventDestroy(e.ev[i]);
  if (e.stream) cudaStreamDestroy(e.stream);
  e = uc::Env{};
}

}  // namespace

uc_status uc_server_create(const uc_server_config* cfg, uc_server** out) {
  if (!cfg || !out) return UC_EINPUT;
  *out = nullptr;
  uc_server* s = new (std::nothrow) uc_server();
  if (!s) return UC_ENOMEM;
  s->cfg = *cfg;
  if (s->cfg.lanes <= 0) s->cfg.lanes = 4;
  if (s->cfg.lanes > 64) s->cfg.lanes = 64;
  if (s->cfg.max_batch <= 0) s->cfg.max_batch = 64;
  if (s->cfg.batch_bytes == 0) s->cfg.batch_bytes = size_t(64) << 20;
  if (cudaSetDevice(s->cfg.device) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return UC_ECUDA;
  }
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  size_t budget = s->cfg.hbm_budget ? s->cfg.hbm_budget : std::min(size_t(160) << 30, size_t(double(fr) * 0.9));
  budget &= ~size_t(255);
  if (cudaMalloc(&s->pool, budget) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return UC_ENOMEM;
  }
  s->cfg.hbm_budget = budget;
  s->map = new PoolMap(budget);
  if (s->cfg.host_budget == 0) s->cfg.host_budget = size_t(16) << 30;
  s->cfg.host_budget &= ~size_t(255);
  if (cudaHostAlloc(&s->hpool, s->cfg.host_budget, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    s->hpool = nullptr;  // results fall back to malloc
  } else {
    s->hmap = new PoolMap(s->cfg.host_budget);
  }
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, s->cfg.device);
  uc_status st = UC_OK;
  for (int i = 0; i < s->cfg.lanes && st == UC_OK; ++i) {
    Lane* ln = new Lane();
    uc::Env& e = ln->env;
    e.device = s->cfg.device;
    e.sm_count = prop.multiProcessorCount;
    e.smem_optin = int(prop.sharedMemPerBlockOptin);
    e.budget = budget;
    e.pool = true;
    e.tune = s->cfg.tuning;
    cudaError_t ce = cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking);
    e.own_stream = true;
    if (ce == cudaSuccess) ce = cudaMalloc(&e.ctr, sizeof(uc::Counters));
    if (ce == cudaSuccess) ce = cudaMallocHost(&e.h_ctr, sizeof(uc::Counters));
    for (int q = 0; q < uc::Env::NEV && ce == cudaSuccess; ++q) ce = cudaEventCreate(&e.ev[q]);
    // job table for the largest batch, allocated once
    const size_t jb = size_t(s->cfg.max_batch) * (sizeof(uc::JobTab) + 4 * 8) + 1024;
    if (ce == cudaSuccess) ce = cudaMalloc(&e.jbuf, jb);
    if (ce == cudaSuccess) e.jcap = jb;
    s->lanes.push_back(ln);
    if (ce != cudaSuccess) {
      cudaGetLastError();
      st = UC_ECUDA;
    }
  }
  if (st != UC_OK) {
    uc_server_destroy(s);
    return st;
  }
  for (Lane* ln : s->lanes) ln->th = std::thread(lane_main, s, ln);
  s->sched = std::thread(sched_main, s);
  *out = s;
  return UC_OK;
}

uc_status uc_server_submit(uc_server* s, const char* text, size_t bytes, int k, int l, uint64_t* ticket) {
  if (!s || (!text && bytes) || !ticket) return UC_EINPUT;
  if (k < 2 || k > 63 || l < 1 || l > 16 || l > k - 1) return UC_EINPUT;
  SJob* j = new (std::nothrow) SJob();
  if (!j) return UC_ENOMEM;
  j->text = text;
  j->bytes = bytes;
  j->k = k;
  j->l = l;
  j->t_submit = now_s();
  std::lock_guard<std::mutex> lock(s->mu);
  j->id = s->next_id++;
  if (s->t_first == 0) s->t_first = j->t_submit;
  s->jobs[j->id] = j;
  s->queue.push_back(j);
  *ticket = j->id;
  s->cv_sched.notify_all();
  return UC_OK;
}

uc_status uc_server_poll(uc_server* s, uint64_t ticket, int* done) {
  if (!s || !done) return UC_EINPUT;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return UC_EINPUT;
  *done = it->second->done ? 1 : 0;
  return UC_OK;
}

uc_status uc_server_wait(uc_server* s, uint64_t ticket, double timeout_s, char** buf, size_t* len,
                         uc_server_job_info* info) {
  if (!s) return UC_EINPUT;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return UC_EINPUT;
  SJob* j = it->second;
  auto ready = [&] { return j->done; };
  if (timeout_s > 0) {
    if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), ready)) return UC_ETIMEOUT;
  } else {
    s->cv_done.wait(lock, ready);
  }
  const uc_status st = j->status;
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->status = st;
    info->batch = j->batch;
    info->n_kmers = j->n_kmers;
    info->queue_ms = (j->t_admit > 0 ? j->t_admit - j->t_submit : 0) * 1e3;
    info->latency_ms = (j->t_done - j->t_submit) * 1e3;
    std::strncpy(info->error, j->err.c_str(), sizeof(info->error) - 1);
  }
  if (buf) {
    *buf = j->result;  // the caller owns it now (uc_server_free)
    j->result = nullptr;
  }
  if (len) *len = j->len;
  if (j->result) free_result_locked(s, j->result);
  s->jobs.erase(it);
  delete j;
  return st;
}

uc_status uc_server_free(uc_server* s, char* buf) {
  if (!s) return UC_EINPUT;
  if (buf) free_result(s, buf);
  return UC_OK;
}

uc_status uc_server_stats(uc_server* s, uc_server_totals* out) {
  if (!s || !out) return UC_EINPUT;
  std::lock_guard<std::mutex> lock(s->mu);
  std::memset(out, 0, sizeof(*out));
  std::vector<double> v = s->lat_ms;
  std::sort(v.begin(), v.end());
  out->jobs_done = v.size();
  out->kmers_done = s->kmers_done;
  out->batches = s->batches;
  out->batched_jobs = s->batched_jobs;
  out->queued = s->queue.size();
  out->pool_bytes = s->map->cap();
  out->pool_peak_bytes = s->map->peak();
  if (!v.empty()) {
    auto pct = [&](double q) { return v[std::min(v.size() - 1, size_t(q * double(v.size() - 1) + 0.5))]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = v.back();
    double t = 0;
    for (double x : v) t += x;
    out->mean_ms = t / double(v.size());
  }
  out->wall_s = (s->t_last > s->t_first) ? s->t_last - s->t_first : 0;
  return UC_OK;
}

uc_status uc_server_destroy(uc_server* s) {
  if (!s) return UC_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    s->cv_sched.notify_all();
    for (Lane* ln : s->lanes) ln->cv.notify_all();
  }
  if (s->sched.joinable()) s->sched.join();
  for (Lane* ln : s->lanes) {
    // a lane finishes the group it holds before it sees the stop flag
    {
      std::lock_guard<std::mutex> lock(s->mu);
      ln->cv.notify_all();
    }
    if (ln->th.joinable()) ln->th.join();
  }
  cudaSetDevice(s->cfg.device);
  for (Lane* ln : s->lanes) {
    destroy_lane_env(ln->env);
    delete ln;
  }
  for (auto& kv : s->jobs) {
    if (kv.second->result) free_result_locked(s, kv.second->result);
    delete kv.second;
  }
  if (s->pool) cudaFree(s->pool);
  delete s->map;
  if (s->hpool) cudaFreeHost(s->hpool);
  delete s->hmap;
  delete s;
  return UC_OK;
}
