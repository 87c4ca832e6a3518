// uc_kernels.cuh — kernel declarations and launch helpers shared by the
// pipeline (uc_pipeline.cu) and the C ABI (uc_capi.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "uc_common.cuh"

namespace uc {

// Device-side counters of one pipeline run (one allocation, zeroed per run).
struct Counters {
  unsigned long long out_cursor;     // bytes of finished lines written
  unsigned long long seg_char_cursor;
  unsigned long long n_copies;
  unsigned long long cycles;
  uint32_t seg_count;
  uint32_t cross_count;
  uint32_t ntiles;
  uint32_t tile_next;
  uint32_t nbig;
  uint32_t active;                   // stitch: active list length
  uint32_t active_next;
  uint32_t err;
  uint32_t work_next;                // level-2 scatter work counter
  uint32_t nwarp, nblock;            // tiles per tier
  uint32_t wtile_next;
  uint32_t count_ovf;                // a 16-bit bucket count wrapped in k_pack
};

// One job of a batch (a single call is a batch of one).  Its k-mers occupy
// keys[koff, koff + n); its buckets are (job << job_bits) | local; its lines
// go to out[obase, obase + ocap); its open segments use ids
// [seg_base, seg_base + seg_cap).
struct JobTab {
  const uint8_t* text;
  unsigned long long tbytes, body, end, n, koff, lb0;  // lb0: first 256-line block
  unsigned long long obase, ocap;
  uint32_t seg_base, seg_cap;
  uint32_t fixed;  // every line is k chars + '\n'
  uint32_t err;    // header/layout problems found on the device
};

struct TileParams {
  const uint64_t* pkeys;        // copies (NW words each, role bits in the last word)
  const uint32_t* plink;        // cross index (fused) or k-mer id (edges)
  const unsigned long long* tile_begin;  // [ntiles + 1] copy offsets
  Counters* ctr;
  const uint32_t* big_list;     // big-tile launch: tile ids
  const uint32_t* wlist;        // warp-tier tile ids
  const uint32_t* blist;        // block-tier tile ids
  uint32_t wcap, wts, wbytes;   // warp tiles: capacity, hash slots, shared bytes per warp
  const JobTab* jobs;
  const uint32_t* tile_job;     // job of each tile
  unsigned long long* jout;     // per-job closed-line cursor (bytes)
  uint32_t* jseg;               // per-job segment cursor
  uint32_t* seg_job;            // job of each segment
  char* big_scratch;
  const unsigned long long* big_off;
  int k;
  uint32_t cap;                 // shared-memory tile capacity (copies)
  uint32_t tslots;              // shared-memory hash slots (power of two >= 2*cap)
  uint32_t lf;                  // hash slots per 100 copies of a tile (150..800)
  int mode;                     // 0 = edges by id, 1 = fused emission
  uint32_t* succ;
  uint32_t* pred;
  char* out;
  unsigned long long out_cap;
  char* segchars;
  unsigned long long segchars_cap;
  uint32_t seg_cap;
  unsigned long long* seg_off;
  uint32_t* seg_len;
  uint32_t* seg_sx;
  uint32_t* seg_ex;
  uint32_t* start_seg;
  uint32_t* end_seg;
};

// Shared memory of one tile: keys plus four 16-bit arrays per copy, and
// 16-bit hash slots.
__host__ __device__ inline size_t tile_bytes(int nw, uint32_t cap, uint32_t tslots) {
  return size_t(cap) * (8u * nw + 8u) + size_t(tslots) * 2u;
}

// Smallest power of two >= x, for x <= 2^31 (callers bound x first); larger
// x returns 2^31 after at most 31 doublings.
__host__ __device__ inline uint32_t pow2_at_least(uint64_t x) {
  uint32_t p = 1;
  for (int i = 0; i < 31 && p < x; ++i) p <<= 1;
  return p;
}

// Carved table of a tile of c copies: the hash slots, and at least 2c
// entries because the table doubles as rank scratch after hashing.
__host__ __device__ inline uint32_t big_slots(uint64_t c, uint32_t lf) {
  const uint64_t want = c * lf / 100;
  return pow2_at_least(want > 2 * c ? want : 2 * c);
}

}  // namespace uc
