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
};

// One open segment of the fused path (written by the tile that finds it): the
// offset of its chars in the segment-char area (low 40 bits) and its job
// (high 24 bits), its copy count, and the cross index through which its line
// continues (NONE where the line ends).  A segment that starts a line keeps
// k - 1 + len chars there; the others keep the len - 1 chars they add (their
// first k-mer ends the segment before).  Segment ids: a segment that starts
// at the S-only copy of cross k-mer x has id x; a segment that starts a line
// (at a P-role copy) takes an id from its job's head pool, after all cross
// indices.
struct __align__(16) SegRec {
  unsigned long long off_job;
  uint32_t len;
  uint32_t next;
};
constexpr int SEG_OFF_BITS = 40;
constexpr unsigned long long SEG_OFF_MASK = (1ull << SEG_OFF_BITS) - 1ull;

// One job of a batch (a single call is a batch of one).  Its k-mers occupy
// keys[koff, koff + n); its buckets are (job << job_bits) | local; its lines
// go to out[obase, obase + ocap); the segments that start its stitched
// lines take head-pool ids [seg_base, seg_base + seg_cap) (after the cross
// indices).
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
  uint32_t* jseg;               // per-job head-pool cursor
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
  SegRec* seg;                  // open segments by id
  uint32_t xcount;              // cross k-mers (the head pool starts there)
};

// Shared memory of one tile: keys plus four 16-bit arrays per copy (sized
// in fours), and 16-bit hash slots.
__host__ __device__ inline size_t tile_bytes(int nw, uint32_t cap, uint32_t tslots) {
  return size_t(cap) * 8u * nw + size_t((cap + 3u) & ~3u) * 8u + size_t(tslots) * 2u;
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
