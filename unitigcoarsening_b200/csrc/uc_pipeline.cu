// uc_pipeline.cu — CUDA kernels of the unitig compactor and the host code
// that sequences them.
//
// Data flow of the fused path (all device resident; a batch of jobs shares
// every launch):
//   text --k_pack (fused minimizers)--> keys[n], (b1,b2)[n], bucket counts
//   --scan/plan--> tiles of whole buckets --k_scatter_coarse/fine--> copies
//   in bucket order --k_tile_warp / k_tile / k_tile_big (persistent; a warp,
//   a CTA, or global scratch per tile)--> finished lines + open segments
//   (one record per segment id: its chars, length and continuation)
//   --stitch (k_walk_emit: each line from its head; list ranking,
//   k_chain_len, k_seg_copy for what the walk leaves)--> cross-tile lines.
// The phase-by-phase entry points (pack, minimizers, find_edges, contract,
// emit) run the same kernels separately.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/uc.h"
#include "uc_kernels.cuh"
#include "uc_pipeline.h"

#include <cuda_pipeline.h>
#include <cub/device/device_radix_sort.cuh>

namespace uc {

// ===================================================================== scan

template <typename Tin, typename Tout>
__global__ void k_scan_reduce(const Tin* __restrict__ in, uint64_t n, Tout* __restrict__ bsum,
                              uint32_t per_block) {
  __shared__ Tout sh[33];
  const uint64_t b0 = uint64_t(blockIdx.x) * per_block;
  Tout acc = 0;
  for (uint64_t i = b0 + threadIdx.x; i < min(n, b0 + per_block); i += blockDim.x) acc += Tout(in[i]);
  Tout total;
  block_excl_scan(acc, sh, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// Exclusive scan of one block's slice, offset by the scanned block sums.
template <typename Tin, typename Tout>
__global__ void k_scan_down(const Tin* __restrict__ in, uint64_t n, Tout* __restrict__ out,
                            const Tout* __restrict__ boff, uint32_t per_block, Tout* total_out) {
  __shared__ Tout sh[33];
  const uint64_t b0 = uint64_t(blockIdx.x) * per_block;
  const uint64_t b1 = min(n, b0 + per_block);
  const uint32_t per_thread = (per_block + blockDim.x - 1) / blockDim.x;
  const uint64_t lo = b0 + uint64_t(threadIdx.x) * per_thread;
  const uint64_t hi = min(b1, lo + per_thread);
  Tout acc = 0;
  for (uint64_t i = lo; i < hi; ++i) acc += Tout(in[i]);
  Tout total;
  Tout pre = block_excl_scan(acc, sh, &total) + boff[blockIdx.x];
  for (uint64_t i = lo; i < hi; ++i) {
    const Tout v = Tout(in[i]);
    out[i] = pre;
    pre += v;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
    out[n] = boff[blockIdx.x] + total;
    if (total_out) *total_out = boff[blockIdx.x] + total;
  }
}

// Exclusive scan in[0..n) -> out[0..n], out[n] = total.  tmp needs
// scan_tmp_elems(n) elements of Tout.
template <typename Tin, typename Tout>
static void scan_excl(const Tin* in, uint64_t n, Tout* out, Tout* tmp, cudaStream_t s,
                      Tout* total_out = nullptr) {
  const uint32_t per_block = 1024 * 8;
  const uint64_t nb = std::max<uint64_t>(1, (n + per_block - 1) / per_block);
  Tout* bsum = tmp;
  Tout* boff = tmp + nb;
  Tout* rest = tmp + 2 * nb + 1;
  k_scan_reduce<Tin, Tout><<<unsigned(nb), 1024, 0, s>>>(in, n, bsum, per_block);
  if (nb == 1) {
    cudaMemsetAsync(boff, 0, sizeof(Tout), s);
  } else {
    scan_excl<Tout, Tout>(bsum, nb, boff, rest, s);
  }
  k_scan_down<Tin, Tout><<<unsigned(nb), 1024, 0, s>>>(in, n, out, boff, per_block, total_out);
}


static uint64_t scan_tmp_elems(uint64_t n) {
  uint64_t t = 0;
  const uint64_t per_block = 1024 * 8;
  for (;;) {
    const uint64_t nb = std::max<uint64_t>(1, (n + per_block - 1) / per_block);
    t += 2 * nb + 1;
    if (nb == 1) break;
    n = nb;
  }
  return t + 8;
}

// ===================================================================== pack

__device__ __forceinline__ uint32_t base_code(uint32_t c) {
  // char_map of compact_kmers (driver.cpp:228-232): A=0 C=1 G=2 T=3, else 0
  return (c == 'C') ? 1u : (c == 'G') ? 2u : (c == 'T') ? 3u : 0u;
}

// SWAR conversion of 4 text bytes (little-endian in x) to 2-bit codes.
// A=0x41 C=0x43 G=0x47 T=0x54 give ((b>>1)^(b>>2))&3 = 0,1,2,3; a byte is
// kept only if rebuilding its letter from that code gives the byte back, so
// every other byte packs as A (the zeroed char_map of compact_kmers,
// driver.cpp:228-232).  Returns the codes of the 4 bytes in bytes 0..3 of the
// result (values 0..3); *nl gets 0x80 in each byte equal to '\n'.
__device__ __forceinline__ uint32_t swar_codes(uint32_t x, uint32_t* nl) {
  const uint32_t t = ((x >> 1) ^ (x >> 2)) & 0x03030303u;
  const uint32_t f = (t << 1) + (((t >> 1) & 0x01010101u) << 1) + (t & (t >> 1) & 0x01010101u) * 11u;
  const uint32_t eq = ~((0x41414141u + f) ^ x);
  const uint32_t ok = ((eq & 0x7F7F7F7Fu) + 0x01010101u) & eq & 0x80808080u;  // 0x80 where byte matches
  const uint32_t z = x ^ 0x0A0A0A0Au;
  *nl = ~(((z & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | z) & 0x80808080u;
  return t & ((ok >> 7) * 3u);
}
// 4 byte-wise codes -> one byte c0 | c1<<2 | c2<<4 | c3<<6
__device__ __forceinline__ uint32_t gather_codes(uint32_t t) { return ((t * 0x41041u) >> 18) & 0xFFu; }

// A block packs 256 consecutive lines per pass.  It first stages the text
// span of those lines in shared memory with 16-byte loads from every thread
// (the whole span in flight at once), inserting a 4-byte gap after every 32
// bytes so that lines 32 bytes apart fall in different banks.  Then each
// thread packs one line, 4 chars per 32-bit SWAR step.  With FUSE the
// prefix/suffix minimizer buckets of every key are computed and counted in the
// same pass (lmin_buckets.h:299-318).
constexpr int PACK_LINES = 256;
constexpr int PACK_SPAN = 18432;                    // staged text bytes per pass
// + 32 words: a (short) line starting at the end of the span reads up to
// k + 4 bytes past its start
constexpr int PACK_WORDS = PACK_SPAN / 4 + PACK_SPAN / 32 + 32;

__device__ __forceinline__ uint32_t pad_word(uint32_t byte_off) { return (byte_off >> 2) + (byte_off >> 5); }

__device__ __forceinline__ uint32_t job_of_block(const JobTab* __restrict__ jobs, uint32_t njobs, uint64_t g) {
  uint32_t lo = 0, hi = njobs;  // last job with lb0 <= g
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].lb0 <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Bucket counts while packing.  The resident path counts copies per group
// of 2^cshift buckets in 32-bit words, at most 2^20 of them (4 MiB, so the
// count reductions stay in L2 at 2^25 buckets); level 3 of the scatter counts
// the buckets of each group itself.  The streamed path (cshift = CNT16)
// counts every bucket in a 16-bit half of a 32-bit word (64 MiB at 2^25
// buckets); a half that wraps shows up as a low total, and the counts are
// then taken again at 32 bits (k_count_buckets).  k_widen16 turns them into
// 32-bit counts.
constexpr uint32_t CNT16 = 32;
constexpr uint32_t COUNT_GROUPS_BITS = 20;
__device__ __forceinline__ void count16(uint32_t* c16, uint32_t b) {
  // a reduction (no value returned, so no wait): a count that wraps its 16
  // bits carries into its neighbour or out of the word, which shows up on
  // the host as a total below the copies the pack counted (k-mers plus cross
  // k-mers), and the counts are then taken again at 32 bits
  atomicAdd(c16 + (b >> 1), 1u << ((b & 1u) * 16u));
}
__global__ void k_widen16(const uint32_t* __restrict__ c16, uint64_t M, uint32_t* __restrict__ counts) {
  for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < M; b += uint64_t(gridDim.x) * blockDim.x)
    counts[b] = (c16[b >> 1] >> ((b & 1u) * 16u)) & 0xFFFFu;
}

__global__ void k_count_buckets(const uint32_t* __restrict__ b1, const uint32_t* __restrict__ b2, uint64_t n,
                                uint32_t* __restrict__ counts) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t a = b1[i], b = b2[i];
    atomicAdd(counts + a, 1u);
    if (a != b) atomicAdd(counts + b, 1u);
  }
}

// MULTI: the block's job comes from the job table (batches); otherwise the
// one job is a kernel parameter, read from the constant bank.
// KC, LC: k and l fixed at compile time (0: taken from the arguments), so
// that the per-word and per-l-mer loops of the common shapes unroll with
// constant shifts.
template <int NW, bool FUSE, bool MULTI, int KC = 0, int LC = 0>
__global__ void __launch_bounds__(256) k_pack(const JobTab* __restrict__ jobs, const JobTab one, uint32_t njobs,
                                              uint64_t nblocks,
                                              const unsigned long long* __restrict__ starts, int k_arg,
                                              uint64_t* __restrict__ keys, uint32_t* err, int l_arg, uint64_t seed,
                                              uint32_t jb, uint32_t* __restrict__ b1, uint32_t* __restrict__ b2,
                                              uint32_t* __restrict__ counts, uint32_t cshift,
                                              uint32_t* __restrict__ jcross) {
  __shared__ uint32_t buf[PACK_WORDS];
  __shared__ uint32_t s_cross;
  const int k = KC ? KC : k_arg;
  const int l = LC ? LC : l_arg;
  uint32_t bad = 0;
  const uint32_t stride = uint32_t(k) + 1;
  uint64_t kmask_hi;
  if constexpr (NW == 1) kmask_hi = (k >= 32) ? ~0ull : ((1ull << (2 * k)) - 1ull);
  else kmask_hi = (2 * k - 64 >= 64) ? ~0ull : ((1ull << ((2 * k - 64) & 63)) - 1ull);
  for (uint64_t g = blockIdx.x; g < nblocks; g += gridDim.x) {
    const uint32_t j = MULTI ? job_of_block(jobs, njobs, g) : 0u;
    const uint8_t* text = MULTI ? jobs[j].text : one.text;
    const uint64_t tbytes = MULTI ? jobs[j].tbytes : one.tbytes;
    const uint64_t body = MULTI ? jobs[j].body : one.body;
    const uint64_t end = MULTI ? jobs[j].end : one.end;
    const uint64_t n = MULTI ? jobs[j].n : one.n;
    const uint64_t koff = MULTI ? jobs[j].koff : one.koff;
    const uint64_t b0 = (g - (MULTI ? jobs[j].lb0 : one.lb0)) * PACK_LINES;
    const uintptr_t tb = reinterpret_cast<uintptr_t>(text);
    const uint32_t cnt = uint32_t((n - b0) < PACK_LINES ? (n - b0) : PACK_LINES);
    const uint64_t s0 = starts ? uint64_t(starts[b0]) : body + b0 * stride;
    const uint64_t s1 = (b0 + cnt < n) ? (starts ? uint64_t(starts[b0 + cnt]) : body + (b0 + cnt) * stride) : end;
    const uintptr_t A0 = (tb + s0) & ~uintptr_t(15);
    const uint64_t span = (tb + s1) - A0;
    const bool staged = span + 16 <= PACK_SPAN;
    if (threadIdx.x == 0) s_cross = 0;
    if (staged) {
      const uint32_t nch = uint32_t((span + 15) / 16);
      for (uint32_t c = threadIdx.x; c < nch; c += blockDim.x) {
        const uintptr_t a = A0 + 16u * c;
        uint4 v;
        if (a >= tb && a + 16 <= tb + tbytes) {
          v = __ldcs(reinterpret_cast<const uint4*>(a));  // read once: evict first
        } else {
          uint32_t w[4] = {0x0A0A0A0Au, 0x0A0A0A0Au, 0x0A0A0A0Au, 0x0A0A0A0Au};
          for (int q = 0; q < 16; ++q) {
            const uintptr_t x = a + q;
            if (x >= tb && x < tb + tbytes) {
              const uint32_t byte = *reinterpret_cast<const uint8_t*>(x);
              w[q >> 2] = (w[q >> 2] & ~(0xFFu << (8 * (q & 3)))) | (byte << (8 * (q & 3)));
            }
          }
          v = make_uint4(w[0], w[1], w[2], w[3]);
        }
        const uint32_t wi = pad_word(16u * c);  // 4 words, never split by a gap
        buf[wi] = v.x;
        buf[wi + 1] = v.y;
        buf[wi + 2] = v.z;
        buf[wi + 3] = v.w;
      }
    }
    __syncthreads();
    const uint32_t t = threadIdx.x;
    uint32_t mycross = 0;
    if (t < cnt) {
      const uint64_t line = b0 + t;
      const uint64_t s = starts ? uint64_t(starts[line]) : body + line * stride;
      Key<NW> key;
#pragma unroll
      for (int w = 0; w < NW; ++w) key.w[w] = 0;
      bool lbad = false;
      const bool check_term = !starts && line + 1 < n;
      bool fast = false;
      if (staged) {
        const uint32_t off = uint32_t((tb + s) - A0);     // line start in the staged span
        const uint32_t lim = uint32_t((tb + s1) - A0);    // end of the staged lines
        lbad |= (off + uint32_t(k) > lim);
        const uint32_t sh = 8u * (off & 3u);
        const uint32_t base = off & ~3u;
        // fast form: codes of 4 bytes in 3 operations, then one check that
        // every byte is the letter its code spells ("ACGT"[code]); a line
        // with any other byte among its k chars (a non-ACGT letter or a line
        // break) is packed again by the exact form below
        {
          uint32_t cur = buf[pad_word(base)];
          uint32_t mism = 0;
          const int nfull = k / 4;
#pragma unroll 4
          for (int jw = 0; jw <= nfull; ++jw) {
            const uint32_t nxt = buf[pad_word(base + 4u * (jw + 1))];
            const uint32_t x = __funnelshift_r(cur, nxt, sh);
            cur = nxt;
            const int c0 = 4 * jw;
            // the last word holds k % 4 chars and the line break
            const uint32_t inmask = (jw < nfull) ? 0xFFFFFFFFu : ((1u << (8 * (k - c0))) - 1u);
            const uint32_t g = gather_codes(((x >> 1) ^ (x >> 2)) & 0x03030303u);
            mism |= (ascii4(g) ^ x) & inmask;
            if (check_term && jw == nfull) lbad |= ((x >> (8 * (k - c0))) & 0xFFu) != '\n';
            // codes past char k-1 fall under kmask_hi below; a word never
            // straddles the two key words (32 is a multiple of 4)
            const uint64_t gc = uint64_t(g);
            if (NW == 1 || c0 < 32) key.w[0] |= gc << (2 * c0);
            else key.w[NW - 1] |= gc << (2 * (c0 - 32));
          }
          fast = (mism == 0);
        }
      }
      if (staged && !fast) {
#pragma unroll
        for (int w = 0; w < NW; ++w) key.w[w] = 0;
        const uint32_t off = uint32_t((tb + s) - A0);
        const uint32_t lim = uint32_t((tb + s1) - A0);
        lbad |= (off + uint32_t(k) > lim);
        const uint32_t sh = 8u * (off & 3u);
        const uint32_t base = off & ~3u;
        uint32_t cur = buf[pad_word(base)];
        const int nwords = (k + 4) / 4;  // covers chars 0..k (k chars + terminator)
#pragma unroll 4
        for (int jw = 0; jw < nwords; ++jw) {
          const uint32_t nxt = buf[pad_word(base + 4u * (jw + 1))];
          const uint32_t x = __funnelshift_r(cur, nxt, sh);
          cur = nxt;
          uint32_t nl;
          const uint32_t tc = swar_codes(x, &nl);
          const int c0 = 4 * jw;
          const uint32_t inmask = (c0 + 4 <= k) ? 0xFFFFFFFFu : (c0 >= k ? 0u : (0xFFFFFFFFu >> (8 * (c0 + 4 - k))));
          lbad |= (nl & inmask) != 0;
          if (check_term && c0 <= k && k < c0 + 4) {
            const uint32_t tbyte = (x >> (8 * (k - c0))) & 0xFFu;
            lbad |= (tbyte != '\n');
          }
          const uint64_t gc = uint64_t(gather_codes(tc & inmask));
          if (NW == 1 || c0 < 32) key.w[0] |= gc << (2 * c0);
          else key.w[NW - 1] |= gc << (2 * (c0 - 32));
        }
      } else if (!staged) {
        for (int c = 0; c <= k; ++c) {
          const uint64_t pos = s + c;
          const uint32_t ch = (pos < end) ? uint32_t(__ldg(text + pos)) : uint32_t('\n');
          if (c < k) {
            lbad |= (ch == '\n') || (pos >= end);
            const uint64_t code = base_code(ch);
            if (c < 32) key.w[0] |= code << (2 * c);
            else key.w[NW - 1] |= code << (2 * (c - 32));
          } else if (check_term && ch != '\n') {
            lbad = true;
          }
        }
      }
      key.w[NW - 1] &= kmask_hi;
      if (lbad) bad = 1;
      // keys and bucket ids stream out with evict-first stores, so that the
      // text and them do not push the bucket counts out of L2
      if constexpr (NW == 1) __stcs(reinterpret_cast<unsigned long long*>(keys) + koff + line,
                                    static_cast<unsigned long long>(key.w[0]));
      else st_key<NW>(keys, koff + line, key);
      if constexpr (FUSE) {
        uint32_t a, b;
        lmins<NW>(key, k, l, seed, nullptr, a, b);
        const uint32_t jp = j << jb;
        a = jp | bucket_of(a, jb);
        b = jp | bucket_of(b, jb);
        __stcs(b1 + koff + line, a);
        __stcs(b2 + koff + line, b);
        if (counts) {  // (the streamed path's second pass only needs the buckets)
          if (cshift == CNT16) {
            count16(counts, a);
            if (a != b) count16(counts, b);
          } else {
            // one 32-bit count per group of 2^cshift buckets (a reduction)
            atomicAdd(counts + (a >> cshift), 1u);
            if (a != b) atomicAdd(counts + (b >> cshift), 1u);
          }
          mycross = (a != b) ? 1u : 0u;
        }
      }
    }
    if constexpr (FUSE) {
      mycross = __reduce_add_sync(0xFFFFFFFFu, mycross);
      if ((threadIdx.x & 31) == 0 && mycross) atomicAdd(&s_cross, mycross);
    }
    __syncthreads();
    if (FUSE && threadIdx.x == 0 && s_cross && jcross) atomicAdd(jcross + j, s_cross);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(err, starts ? ERR_LINE : ERR_LAYOUT);
}

// Header and end of every job's text (batches of more than one job): the
// count line, the first k-mer line, the end of the last line, and whether
// every line is k chars + '\n'.  One thread per job.
__global__ void k_headers(JobTab* __restrict__ jobs, uint32_t njobs, int k) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  JobTab J = jobs[j];
  const uint8_t* t = J.text;
  const uint64_t bytes = J.tbytes;
  uint64_t p = 0;
  while (p < bytes && (t[p] == ' ' || t[p] == '\t' || t[p] == '\r')) ++p;
  uint32_t e = 0;
  uint64_t v = 0;
  if (p >= bytes || t[p] < '0' || t[p] > '9') e = 1;
  while (!e && p < bytes && t[p] >= '0' && t[p] <= '9') {
    v = v * 10 + uint64_t(t[p] - '0');
    if (v > 0x7FFFFFFEull) e = 1;
    ++p;
  }
  while (p < bytes && t[p] != '\n') ++p;
  const uint64_t body = (p < bytes) ? p + 1 : bytes;
  uint64_t end = bytes;
  while (end > body && (t[end - 1] == '\n' || t[end - 1] == '\r')) --end;
  J.n = e ? 0 : v;
  J.body = body;
  J.end = end;
  J.err = e;
  const uint64_t stride = uint64_t(k) + 1;
  J.fixed = (!e && ((J.n == 0 && end == body) || (J.n > 0 && end - body == J.n * stride - 1))) ? 1u : 0u;
  jobs[j] = J;
}

// Line starts for the general layout: '\n' positions in [body, end).
__global__ void k_count_nl(const uint8_t* __restrict__ text, uint64_t body, uint64_t end,
                           uint32_t* __restrict__ cnt, uint32_t chunk) {
  const uint64_t c0 = body + uint64_t(blockIdx.x) * chunk;
  const uint64_t c1 = min(end, c0 + chunk);
  uint32_t acc = 0;
  for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) acc += (text[i] == '\n');
  acc = __reduce_add_sync(0xFFFFFFFFu, acc);
  __shared__ uint32_t sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += sh[w];
    cnt[blockIdx.x] = t;
  }
}

__global__ void k_write_starts(const uint8_t* __restrict__ text, uint64_t body, uint64_t end,
                               const unsigned long long* __restrict__ off, uint32_t chunk,
                               unsigned long long* __restrict__ starts, uint64_t nlines) {
  const uint64_t c0 = body + uint64_t(blockIdx.x) * chunk;
  const uint64_t c1 = min(end, c0 + chunk);
  if (blockIdx.x == 0 && threadIdx.x == 0) starts[0] = body;
  // serial within a warp-strided pass: each thread scans a sub-range in order
  const uint32_t per = (chunk + blockDim.x - 1) / blockDim.x;
  const uint64_t lo = c0 + uint64_t(threadIdx.x) * per;
  const uint64_t hi = min(c1, lo + per);
  uint32_t mine = 0;
  for (uint64_t i = lo; i < hi; ++i) mine += (text[i] == '\n');
  __shared__ uint32_t sc[33];
  uint32_t tot;
  uint64_t r = off[blockIdx.x] + block_excl_scan(mine, sc, &tot);
  for (uint64_t i = lo; i < hi; ++i) {
    if (text[i] == '\n') {
      ++r;
      if (r < nlines) starts[r] = i + 1;
    }
  }
}

// ============================================================== minimizers

template <int NW>
__global__ void k_lmin(const uint64_t* __restrict__ keys, uint64_t n, int k, int l, uint64_t seed,
                       const uint32_t* __restrict__ table, uint32_t* __restrict__ l1,
                       uint32_t* __restrict__ l2) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t a, b;
    lmins<NW>(ld_key<NW>(keys, i), k, l, seed, table, a, b);
    l1[i] = a;
    l2[i] = b;
  }
}

// Minimizers -> prefix bucket b1 and suffix bucket b2, counted per bucket
// (find_l_minimizer "calc lmins" + "count lmins", lmin_buckets.h:299-318).
template <int NW>
__global__ void __launch_bounds__(256) k_lmin_count(const uint64_t* __restrict__ keys, uint64_t n,
                                                    int k, int l, uint64_t seed, uint32_t bbits,
                                                    uint32_t* __restrict__ b1, uint32_t* __restrict__ b2,
                                                    uint32_t* __restrict__ counts) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t a, b;
    lmins<NW>(ld_key<NW>(keys, i), k, l, seed, nullptr, a, b);
    a = bucket_of(a, bbits);
    b = bucket_of(b, bbits);
    b1[i] = a;
    b2[i] = b;
    atomicAdd(counts + a, 1u);
    if (a != b) atomicAdd(counts + b, 1u);
  }
}

// ============================================================ tile planning

// Tiles pack consecutive whole buckets, next fit: each thread walks a run of
// `runlen` buckets (a multiple of 16) and starts a new tile at the run's
// first bucket, at a job's first bucket, and wherever the next bucket would
// take the tile past `cap` copies.  A tile of several buckets therefore
// holds at most `cap` copies; a bucket larger than `cap` sits alone.  Counts
// and flags move 16 at a time (the arrays start 256-byte aligned).
__global__ void k_tile_flags(const uint32_t* __restrict__ counts, uint32_t m, uint32_t cap, uint32_t jb,
                             uint32_t runlen, uint32_t* __restrict__ flag) {
  const uint32_t nruns = (m + runlen - 1) / runlen;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nruns; r += gridDim.x * blockDim.x) {
    const uint32_t b0 = r * runlen, b1 = min(m, b0 + runlen);
    uint32_t run = 0;
    for (uint32_t c0 = b0; c0 < b1; c0 += 16) {
      const bool full = c0 + 16 <= b1;
      uint32_t c[16], f[16];
      if (full) {
        const uint4* src = reinterpret_cast<const uint4*>(counts + c0);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const uint4 x = src[v];
          c[4 * v] = x.x;
          c[4 * v + 1] = x.y;
          c[4 * v + 2] = x.z;
          c[4 * v + 3] = x.w;
        }
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) c[q] = (c0 + q < b1) ? counts[c0 + q] : 0u;
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const uint32_t b = c0 + uint32_t(q);
        const bool st = (b == b0) || ((b >> jb) != ((b - 1) >> jb)) || (run + c[q] > cap);
        f[q] = st;
        run = st ? c[q] : run + c[q];
      }
      if (full) {
        uint4* dst = reinterpret_cast<uint4*>(flag + c0);
#pragma unroll
        for (int v = 0; v < 4; ++v) dst[v] = make_uint4(f[4 * v], f[4 * v + 1], f[4 * v + 2], f[4 * v + 3]);
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (c0 + q < b1) flag[c0 + q] = f[q];
      }
    }
  }
}

__global__ void k_tile_write(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ fidx,
                             const unsigned long long* __restrict__ off, uint32_t m, uint32_t jb,
                             unsigned long long* __restrict__ tile_begin, uint32_t* __restrict__ tile_job,
                             Counters* ctr) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < m; b += gridDim.x * blockDim.x) {
    if (flag[b]) {
      tile_begin[fidx[b]] = off[b];
      tile_job[fidx[b]] = b >> jb;
    }
    if (b == m - 1) {
      const uint32_t nt = fidx[b] + flag[b];
      tile_begin[nt] = off[m];
      ctr->ntiles = nt;
    }
  }
}

// Sort the tiles into tiers by size: warp tiles, block tiles and oversized
// tiles (with the global scratch each one needs).
__global__ void k_classify(const unsigned long long* __restrict__ tile_begin, Counters* ctr, uint32_t wcap,
                           uint32_t cap, uint32_t* __restrict__ wlist, uint32_t* __restrict__ blist,
                           uint32_t* __restrict__ big_list, unsigned long long* __restrict__ big_size, int nw,
                           uint32_t lf, uint32_t t0, uint32_t t1) {
  const uint32_t nt = min(ctr->ntiles, t1);
  for (uint32_t t = t0 + blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    const uint64_t c = tile_begin[t + 1] - tile_begin[t];
    // (a tile's line bytes must fit 32-bit offsets: c * 64 < 2^32)
    if (tile_begin[t + 1] < tile_begin[t] || c > (1ull << 26)) {
      atomicOr(&ctr->err, ERR_INTERNAL);
      continue;
    }
    if (c == 0) continue;
    if (c <= wcap) {
      wlist[atomicAdd(&ctr->nwarp, 1u)] = t;
    } else if (c <= cap) {
      blist[atomicAdd(&ctr->nblock, 1u)] = t;
    } else {
      const uint32_t i = atomicAdd(&ctr->nbig, 1u);
      big_list[i] = t;
      const uint64_t ts = big_slots(c, lf);
      big_size[i] = (c * 8ull * nw + ((c + 3ull) & ~3ull) * 16ull + ts * 4ull + 255ull) & ~255ull;
    }
  }
}

// ================================================================= scatter

// Every k-mer goes to its prefix bucket (role P) and, when its suffix
// minimizer lands in another bucket, a second copy goes to that bucket (role
// S) ("partition by lmins" + "write kmers", lmin_buckets.h:357-407).  The two
// copies of a cross k-mer share one cross index; in edges mode every copy
// carries the k-mer's id instead.
//
// Three levels keep the write frontier inside L2 and the global atomics few.
// Level 1 groups each block's copies by coarse partition (high bucket bits,
// at most 256 partitions) in shared memory and writes them out as contiguous
// runs, one reservation per block and partition.  A coarse partition
// occupies exactly the final positions of its buckets, so level 1 writes
// (key, link, bucket) records into the same index range of a staging
// region.  Level 2 groups each partition's records the same way by
// sub-partition (2^sb buckets), into the same index ranges of a second
// region; all blocks take chunks in partition order.  Level 3 gives each
// sub-partition to one block, which places the records inside its range with
// shared-memory cursors per bucket.
// k-mers per level-1 block pass (at most twice as many copies): large chunks
// spread the per-chunk reservations and barriers over more copies; 3072
// 64-bit keys (100 KB of staging, 2 CTAs per SM) beat 2048 (3 CTAs per SM)
// by 6% at 1 Gbp, and 128-bit keys keep 2048 (98 KB)
template <int NW>
__host__ __device__ constexpr int sc_chunk() {
  return NW == 1 ? 3072 : 2048;
}
static_assert(2 * sc_chunk<1>() < 65536 && 2 * sc_chunk<2>() < 65536, "chunk copy counts share a 32-bit scan");

__global__ void k_coarse_init(const unsigned long long* __restrict__ boff, uint32_t fb, uint32_t mc,
                              unsigned long long* __restrict__ ccur) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < mc; j += gridDim.x * blockDim.x)
    ccur[j] = boff[uint64_t(j) << fb];
}

constexpr int COARSE_THREADS = 256;

template <int NW>
__global__ void __launch_bounds__(COARSE_THREADS) k_scatter_coarse(const uint64_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ b1,
                                                        const uint32_t* __restrict__ b2, uint64_t n,
                                                        uint32_t fb, uint32_t mc,
                                                        unsigned long long* __restrict__ ccur,
                                                        uint64_t* __restrict__ rkey, uint32_t* __restrict__ rlink,
                                                        uint32_t* __restrict__ rbkt, int ids_mode, Counters* ctr) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  uint64_t* skey = reinterpret_cast<uint64_t*>(sm_raw);                         // [2*CHUNK*NW]
  constexpr int SC_CHUNK = sc_chunk<NW>();
  uint32_t* slink = reinterpret_cast<uint32_t*>(skey + 2 * SC_CHUNK * NW);      // [2*CHUNK]
  uint32_t* sbkt = slink + 2 * SC_CHUNK;                                        // [2*CHUNK]
  unsigned long long* gbase = reinterpret_cast<unsigned long long*>(sbkt + 2 * SC_CHUNK);  // [mc]
  uint32_t* hist = reinterpret_cast<uint32_t*>(gbase + mc);                     // [mc]
  uint32_t* lofs = hist + mc;                                                   // [mc + 1]
  __shared__ uint32_t sc[33];
  for (uint64_t c0 = uint64_t(blockIdx.x) * SC_CHUNK; c0 < n; c0 += uint64_t(gridDim.x) * SC_CHUNK) {
    const uint32_t cn = uint32_t((n - c0) < uint64_t(SC_CHUNK) ? (n - c0) : uint64_t(SC_CHUNK));
    // every load of the chunk is issued at once; the values stay in registers
    constexpr int PT = SC_CHUNK / COARSE_THREADS;
    Key<NW> kk[PT];
    uint32_t aa[PT], bb[PT];
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const uint32_t t = uint32_t(q) * COARSE_THREADS + threadIdx.x;
      if (t < cn) {
        kk[q] = ld_key<NW>(keys, c0 + t);
        aa[q] = b1[c0 + t];
        bb[q] = b2[c0 + t];
      }
    }
    for (uint32_t j = threadIdx.x; j < mc; j += blockDim.x) hist[j] = 0;
    __syncthreads();
    // count copies per coarse partition; bit q of cmask marks a cross k-mer
    uint32_t cmask = 0;
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const uint32_t t = uint32_t(q) * COARSE_THREADS + threadIdx.x;
      if (t < cn) {
        atomicAdd(hist + (aa[q] >> fb), 1u);
        if (aa[q] != bb[q]) {
          atomicAdd(hist + (bb[q] >> fb), 1u);
          cmask |= 1u << q;
        }
      }
    }
    __syncthreads();
    // local offsets (scan over the partitions), this thread's first cross
    // index within the chunk, and global reservations.  One scan carries both
    // sums: the copy count in the low half (<= 2 * chunk < 2^16) and the
    // cross count in the high half (<= chunk).  The chunk's cross indices are reserved with a
    // single atomic: a counter shared by every block of the grid serialises
    // in L2, so one reservation per warp and k-mer slot would bound the kernel.
    uint32_t xpre;
    {
      const uint32_t per = (mc + blockDim.x - 1) / blockDim.x;
      const uint32_t j0 = min(mc, threadIdx.x * per), j1 = min(mc, j0 + per);
      uint32_t acc = 0;
      for (uint32_t j = j0; j < j1; ++j) acc += hist[j];
      uint32_t tot;
      const uint32_t both = block_excl_scan(acc | (uint32_t(__popc(cmask)) << 16), sc, &tot);
      uint32_t pre = both & 0xFFFFu;
      xpre = both >> 16;
      for (uint32_t j = j0; j < j1; ++j) {
        const uint32_t h = hist[j];
        lofs[j] = pre;
        gbase[j] = h ? atomicAdd(ccur + j, (unsigned long long)h) : 0ull;
        pre += h;
        hist[j] = 0;
      }
      if (threadIdx.x == 0) {
        lofs[mc] = tot & 0xFFFFu;
        const uint32_t xt = tot >> 16;
        sc[32] = (!ids_mode && xt) ? atomicAdd(&ctr->cross_count, xt) : 0u;
      }
    }
    __syncthreads();
    xpre += sc[32];
    // place every copy in its partition's run of the staging area
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const uint32_t t = uint32_t(q) * COARSE_THREADS + threadIdx.x;
      const bool live = t < cn;
      uint32_t a = 0, b = 0;
      Key<NW> key;
#pragma unroll
      for (int w = 0; w < NW; ++w) key.w[w] = 0;
      if (live) {
        key = kk[q];
        a = aa[q];
        b = bb[q];
      }
      const bool cross = (cmask >> q) & 1u;
      const uint32_t x = (!ids_mode && cross) ? xpre + __popc(cmask & ((1u << q) - 1u)) : NONE;
      if (live) {
        const uint32_t link = ids_mode ? uint32_t(c0 + t) : x;
        Key<NW> kp = key;
        kp.w[NW - 1] |= ROLE_P | (cross ? 0ull : ROLE_S);
        const uint32_t sp = lofs[a >> fb] + atomicAdd(hist + (a >> fb), 1u);
        st_key<NW>(skey, sp, kp);
        slink[sp] = link;
        sbkt[sp] = a;
        if (cross) {
          Key<NW> ks = key;
          ks.w[NW - 1] |= ROLE_S;
          const uint32_t sq = lofs[b >> fb] + atomicAdd(hist + (b >> fb), 1u);
          st_key<NW>(skey, sq, ks);
          slink[sq] = link;
          sbkt[sq] = b;
        }
      }
    }
    __syncthreads();
    // write the runs out: consecutive slots of a partition are consecutive
    // global positions
    const uint32_t total = lofs[mc];
    for (uint32_t sl = threadIdx.x; sl < total; sl += blockDim.x) {
      const uint32_t bk = sbkt[sl];
      const uint32_t part = bk >> fb;
      const uint64_t pos = gbase[part] + (sl - lofs[part]);
      st_key<NW>(rkey, pos, ld_key<NW>(skey, sl));
      rlink[pos] = slink[sl];
      rbkt[pos] = bk;
    }
    __syncthreads();
  }
}

// Level 2: within each coarse partition the staged records are grouped again
// by sub-partition (2^sb consecutive buckets, a few thousand copies), the way
// level 1 groups by partition: a block takes a chunk of one partition's
// staged records, counts them per sub-partition in shared memory, reserves
// one run per sub-partition (one global atomic per run, a few records each
// instead of one per record) and writes its records out as contiguous runs.
// Chunks never span partitions (their list comes from k_mid_items), so the
// counts index one partition's sub-partitions.  All blocks take chunks in
// partition order and reserve at the same cursors, so the runs of the
// chunks in flight stay next to each other: the write frontier is one
// partition's cursors and stays inside L2.  (Reserving for ranges of
// several chunks per block instead gives every block its own frontier:
// 1024 partly written runs per block, more than L2 holds at 1 Gbp.)
constexpr int MID_CHUNK = 4096;    // staged records per level-2 chunk
constexpr int MID_MAX_BINS = 1024; // sub-partitions per coarse partition
constexpr int SUB_MAX_BITS = 8;    // buckets per sub-partition: at most 2^8
constexpr int MID_THREADS = 512;

// Chunk list of level 2: item_start[p] = first chunk of coarse partition p
// (partition p holds the staged records [boff[p << fb], boff[(p+1) << fb])).
__global__ void k_mid_items(const unsigned long long* __restrict__ boff, uint32_t fb, uint32_t mc,
                            uint32_t* __restrict__ item_start) {
  __shared__ uint32_t sc[33];
  const uint32_t p = threadIdx.x;
  uint32_t items = 0;
  if (p < mc) {
    const unsigned long long lo = boff[uint64_t(p) << fb], hi = boff[uint64_t(p + 1) << fb];
    items = uint32_t((hi - lo + MID_CHUNK - 1) / MID_CHUNK);
  }
  uint32_t tot;
  const uint32_t pre = block_excl_scan(items, sc, &tot);
  if (p < mc) item_start[p] = pre;
  if (p == 0) item_start[mc] = tot;
}

template <int NW>
__global__ void __launch_bounds__(MID_THREADS, NW == 1 ? 2 : 1) k_scatter_mid(
    const uint64_t* __restrict__ rkey, const uint32_t* __restrict__ rlink, const uint32_t* __restrict__ rbkt,
    const unsigned long long* __restrict__ goff, uint32_t cg, const uint32_t* __restrict__ item_start, uint32_t fb,
    uint32_t sb, uint32_t mc, unsigned long long* __restrict__ scur, uint64_t* __restrict__ okey,
    uint32_t* __restrict__ olink, uint32_t* __restrict__ obkt, Counters* ctr) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  uint64_t* skey = reinterpret_cast<uint64_t*>(sm_raw);                              // [MID_CHUNK*NW]
  uint32_t* slink = reinterpret_cast<uint32_t*>(skey + MID_CHUNK * NW);              // [MID_CHUNK]
  uint32_t* sbkt = slink + MID_CHUNK;                                                // [MID_CHUNK]
  unsigned long long* gbase = reinterpret_cast<unsigned long long*>(sbkt + MID_CHUNK);  // [nb]
  const uint32_t nb = 1u << (fb - sb);
  uint32_t* hist = reinterpret_cast<uint32_t*>(gbase + nb);                          // [nb]
  uint32_t* lofs = hist + nb;                                                        // [nb + 1]
  uint32_t* istart = lofs + nb + 1;                                                  // [mc + 1]
  __shared__ uint32_t sc[33];
  __shared__ uint32_t s_t, s_p;
  for (uint32_t j = threadIdx.x; j <= mc; j += blockDim.x) istart[j] = item_start[j];
  __syncthreads();
  const uint32_t nitems = istart[mc];
  constexpr int PT = MID_CHUNK / MID_THREADS;
  // the bins this thread scans and reserves
  const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
  const uint32_t j0 = min(nb, threadIdx.x * per), j1 = min(nb, j0 + per);
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t t = atomicAdd(&ctr->work_next, 1u);
      uint32_t lo = 0, hi = mc;  // the partition p with istart[p] <= t < istart[p + 1]
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (istart[mid] <= t) lo = mid;
        else hi = mid;
      }
      s_t = t;
      s_p = lo;
    }
    __syncthreads();
    const uint32_t t = s_t, p = s_p;
    __syncthreads();
    if (t >= nitems) break;
    // (goff: offsets of count groups of 2^cg buckets; partition p starts at
    // group p << (fb - cg))
    const unsigned long long pend = goff[uint64_t(p + 1) << (fb - cg)];
    const unsigned long long c0 = goff[uint64_t(p) << (fb - cg)] + uint64_t(t - istart[p]) * MID_CHUNK;
    const uint32_t cn = uint32_t(min(pend - c0, (unsigned long long)MID_CHUNK));
    const uint32_t sub0 = p << (fb - sb);  // first sub-partition of partition p
    // the chunk's records, all loads issued at once (in registers), and the
    // counts per sub-partition
    uint32_t bb[PT], ll[PT];
    Key<NW> kk[PT];
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const uint32_t i = uint32_t(q) * MID_THREADS + threadIdx.x;
      if (i < cn) {
        bb[q] = rbkt[c0 + i];
        kk[q] = ld_key<NW>(rkey, c0 + i);
        ll[q] = rlink[c0 + i];
      } else {
        bb[q] = 0u;
      }
    }
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) hist[j] = 0;
    __syncthreads();
    // a record outside partition p would be a broken staging order: flag it
    // and leave it out rather than index past the counts
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const uint32_t i = uint32_t(q) * MID_THREADS + threadIdx.x;
      if (i < cn) {
        const uint32_t bin = (bb[q] >> sb) - sub0;
        if (bin < nb) atomicAdd(hist + bin, 1u);
        else atomicOr(&ctr->err, ERR_INTERNAL);
      }
    }
    __syncthreads();
    // local offsets and one reservation per non-empty sub-partition
    {
      uint32_t acc = 0;
      for (uint32_t j = j0; j < j1; ++j) acc += hist[j];
      uint32_t tot;
      uint32_t pre = block_excl_scan(acc, sc, &tot);
      for (uint32_t j = j0; j < j1; ++j) {
        const uint32_t h = hist[j];
        lofs[j] = pre;
        gbase[j] = h ? atomicAdd(scur + sub0 + j, (unsigned long long)h) : 0ull;
        pre += h;
        hist[j] = 0;
      }
      if (threadIdx.x == 0) lofs[nb] = tot;
    }
    __syncthreads();
    // place every record in its sub-partition's run of the staging area
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      const uint32_t i = uint32_t(q) * MID_THREADS + threadIdx.x;
      const uint32_t bin = (bb[q] >> sb) - sub0;
      if (i < cn && bin < nb) {
        const uint32_t sl = lofs[bin] + atomicAdd(hist + bin, 1u);
        st_key<NW>(skey, sl, kk[q]);
        slink[sl] = ll[q];
        sbkt[sl] = bb[q];
      }
    }
    __syncthreads();
    const uint32_t placed = lofs[nb];
    for (uint32_t sl = threadIdx.x; sl < placed; sl += blockDim.x) {
      const uint32_t bk = sbkt[sl];
      const uint32_t bin = (bk >> sb) - sub0;
      const uint64_t pos = gbase[bin] + (sl - lofs[bin]);
      st_key<NW>(okey, pos, ld_key<NW>(skey, sl));
      olink[pos] = slink[sl];
      obkt[pos] = bk;
    }
    __syncthreads();
  }
}

// Level 3: one block owns a sub-partition (2^sb buckets, whole count
// groups of the pack).  With count groups (cout given) it counts its
// records per bucket in shared memory, takes the buckets' offsets from a
// block scan and writes every bucket's count (and offset, to bout) for the
// tile plan; otherwise goff holds every bucket's offset.  It then places
// each record at its bucket's offset plus a rank from a shared-memory
// cursor: no global atomics.  A sub-partition of at most
// `cap` records is assembled in shared memory and written out as one
// contiguous range; a larger one (a large repeat bucket) is placed straight
// into global memory.  Blocks take sub-partitions from a counter.
template <int NW>
__global__ void __launch_bounds__(512, 2) k_scatter_sub(const uint64_t* __restrict__ ikey,
                                                     const uint32_t* __restrict__ ilink,
                                                     const uint32_t* __restrict__ ibkt,
                                                     const unsigned long long* __restrict__ goff, uint32_t gsh,
                                                     uint32_t sb, uint32_t nsub, uint32_t cap,
                                                     uint64_t* __restrict__ pkeys, uint32_t* __restrict__ plink,
                                                     uint32_t* __restrict__ cout, unsigned long long* __restrict__ bout,
                                                     Counters* ctr) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  uint64_t* skey = reinterpret_cast<uint64_t*>(sm_raw);        // [cap * NW]
  uint32_t* slink = reinterpret_cast<uint32_t*>(skey + size_t(cap) * NW);  // [cap]
  __shared__ unsigned long long s_off[1 << SUB_MAX_BITS];
  __shared__ uint32_t s_cur[1 << SUB_MAX_BITS];
  __shared__ uint32_t s_sp;
  __shared__ uint32_t sc[33];
  const uint32_t nbk = 1u << sb;  // <= 2^SUB_MAX_BITS <= blockDim.x
  // records per thread and pass: their loads are in flight together (two
  // CTAs per SM fit the registers)
  constexpr int PER = NW == 1 ? 8 : 4;
  for (;;) {
    if (threadIdx.x == 0) s_sp = atomicAdd(&ctr->work_next, 1u);
    __syncthreads();
    const uint32_t sp = s_sp;
    if (sp >= nsub) break;
    const uint64_t b0 = uint64_t(sp) << sb;
    const unsigned long long lo = goff[uint64_t(sp) << gsh], hi = goff[uint64_t(sp + 1) << gsh];
    // known: goff holds every bucket's offset (no count groups)
    const bool known = cout == nullptr;
    for (uint32_t j = threadIdx.x; j < nbk; j += blockDim.x) {
      if (known) s_off[j] = goff[b0 + j];
      s_cur[j] = 0;
    }
    __syncthreads();
    const bool staged = hi - lo <= cap;
    // the first PER x blockDim records stay in registers from the count to
    // their placement; the rest are counted from their bucket ids and
    // loaded again to be placed
    uint32_t bk[PER];
    Key<NW> kk[PER];
    uint32_t ln[PER];
    auto load = [&](unsigned long long i0) {
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const unsigned long long i = i0 + uint64_t(q) * blockDim.x + threadIdx.x;
        bk[q] = 0xFFFFFFFFu;
        if (i < hi) {
          bk[q] = ibkt[i];
          kk[q] = ld_key<NW>(ikey, i);
          ln[q] = ilink[i];
        }
      }
    };
    auto place = [&](unsigned long long i0) {
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const unsigned long long i = i0 + uint64_t(q) * blockDim.x + threadIdx.x;
        if (i < hi) {
          const uint32_t lb = bk[q] - uint32_t(b0);
          if (lb >= nbk) {  // not this sub-partition's: a broken order upstream
            atomicOr(&ctr->err, ERR_INTERNAL);
            continue;
          }
          const uint64_t pos = s_off[lb] + atomicAdd(s_cur + lb, 1u);
          if (staged) {
            st_key<NW>(skey, pos - lo, kk[q]);
            slink[pos - lo] = ln[q];
          } else {
            st_key<NW>(pkeys, pos, kk[q]);
            plink[pos] = ln[q];
          }
        }
      }
    };
    const uint64_t batch = uint64_t(blockDim.x) * PER;
    load(lo);
    if (!known) {
      // the sub-partition's counts per bucket (records of another
      // sub-partition are flagged when placed)
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const uint32_t lb = bk[q] - uint32_t(b0);
        if (lb < nbk) atomicAdd(s_cur + lb, 1u);
      }
      for (unsigned long long i0 = lo + batch; i0 < hi; i0 += batch) {
        uint32_t bq[PER];
#pragma unroll
        for (int q = 0; q < PER; ++q) {
          const unsigned long long i = i0 + uint64_t(q) * blockDim.x + threadIdx.x;
          bq[q] = (i < hi) ? ibkt[i] : 0xFFFFFFFFu;
        }
#pragma unroll
        for (int q = 0; q < PER; ++q) {
          const uint32_t lb = bq[q] - uint32_t(b0);
          if (lb < nbk) atomicAdd(s_cur + lb, 1u);
        }
      }
      __syncthreads();
      {
        const uint32_t cnt = threadIdx.x < nbk ? s_cur[threadIdx.x] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(cnt, sc, &tot);
        if (threadIdx.x < nbk) {
          s_off[threadIdx.x] = lo + ex;
          s_cur[threadIdx.x] = 0;
          cout[b0 + threadIdx.x] = cnt;
          if (bout) bout[b0 + threadIdx.x] = lo + ex;
        }
      }
      __syncthreads();
    }
    place(lo);
    for (unsigned long long i0 = lo + batch; i0 < hi; i0 += batch) {
      load(i0);
      place(i0);
    }
    __syncthreads();
    if (staged) {
      const uint32_t cnt = uint32_t(hi - lo);
      for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) {
        st_key<NW>(pkeys, lo + t, ld_key<NW>(skey, t));
        plink[lo + t] = slink[t];
      }
    }
    __syncthreads();  // the staging area, s_off / s_cur / s_sp are reused
  }
}

// ==================================================================== tiles

// List-ranking entries: (pointer, distance) in one 64-bit word.
__device__ __forceinline__ unsigned long long pk(uint32_t p, uint32_t o) {
  return (static_cast<unsigned long long>(o) << 32) | p;
}
__device__ __forceinline__ uint32_t pk_p(unsigned long long v) { return uint32_t(v); }
__device__ __forceinline__ uint32_t pk_o(unsigned long long v) { return uint32_t(v >> 32); }
// A head's own entry carries HEAD_BIT in its pointer, so "reached a head" is
// a property of the target entry, not a self-pointer (which a pointer running
// around a cycle can also produce).  Entry counts stay below 2^31.
constexpr uint32_t HEAD_BIT = 0x80000000u;
__device__ __forceinline__ uint32_t ptr_of(unsigned long long v) { return pk_p(v) & ~HEAD_BIT; }
__device__ __forceinline__ bool is_head_entry(unsigned long long v) { return (pk_p(v) & HEAD_BIT) != 0; }


// In-tile indices: 16-bit for shared-memory tiles (capacity <= 32766), 32-bit
// for oversized tiles worked in global scratch.  The top bit of A marks a
// shared prefix ("nullified", assembler.h:138-144) during the edge passes and
// a cycle copy during the cycle cut.
template <typename IT>
struct Ix;
template <>
struct Ix<uint16_t> {
  static constexpr uint32_t NONE = 0xFFFFu, DUP = 0x8000u, CNONE = 0x7FFFu;
};
template <>
struct Ix<uint32_t> {
  static constexpr uint32_t NONE = 0xFFFFFFFFu, DUP = 0x80000000u, CNONE = 0x7FFFFFFFu;
};

// 32-bit atomics on the word holding a 16-bit element; counters stay below
// 2^15 so no carry reaches the neighbouring element.
__device__ __forceinline__ uint32_t* word_of(uint16_t* p, uint32_t& sh) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  sh = uint32_t(a & 2u) * 8u;
  return reinterpret_cast<uint32_t*>(a & ~uintptr_t(3));
}
__device__ __forceinline__ void at_or(uint16_t* p, uint32_t v) {
  uint32_t sh;
  uint32_t* w = word_of(p, sh);
  atomicOr(w, v << sh);
}
__device__ __forceinline__ void at_or(uint32_t* p, uint32_t v) { atomicOr(p, v); }
__device__ __forceinline__ void at_inc(uint16_t* p) {
  uint32_t sh;
  uint32_t* w = word_of(p, sh);
  atomicAdd(w, 1u << sh);
}
__device__ __forceinline__ void at_inc(uint32_t* p) { atomicAdd(p, 1u); }
__device__ __forceinline__ uint32_t at_cas(uint16_t* p, uint32_t cmp, uint32_t val) {
  return atomicCAS(reinterpret_cast<unsigned short*>(p), static_cast<unsigned short>(cmp),
                   static_cast<unsigned short>(val));
}
__device__ __forceinline__ uint32_t at_cas(uint32_t* p, uint32_t cmp, uint32_t val) { return atomicCAS(p, cmp, val); }

template <int NW, typename IT>
struct TileMem {
  uint64_t* key;  // [cap * NW], role bits in the last word
  IT* A;          // suffix-lookup candidate | DUP  -> local successor
  IT* B;          // in-count                       -> scratch
  IT* P;          // who                            -> local predecessor -> segment id
  IT* Q;          // rank pointer / scratch
  IT* T;          // hash slots [ts >= 2*cap]       -> ranks / scratch
  uint32_t ts;
};

template <int NW, typename IT>
__device__ __forceinline__ TileMem<NW, IT> carve(char* base, uint32_t cap, uint32_t ts) {
  TileMem<NW, IT> m;
  const uint32_t cap4 = (cap + 3u) & ~3u;  // the index arrays in fours (vector initialisation)
  m.key = reinterpret_cast<uint64_t*>(base);
  m.A = reinterpret_cast<IT*>(m.key + size_t(cap) * NW);
  m.B = m.A + cap4;
  m.P = m.B + cap4;
  m.Q = m.P + cap4;
  m.T = m.Q + cap4;
  m.ts = ts;
  return m;
}

template <int NW, typename IT>
__device__ __forceinline__ Key<NW> skey(const TileMem<NW, IT>& m, uint32_t i) {
  Key<NW> k;
#pragma unroll
  for (int w = 0; w < NW; ++w) k.w[w] = m.key[size_t(i) * NW + w];
  return k;
}

struct U3 {
  unsigned long long a, b, c;
};
__device__ __forceinline__ U3 u3_add(U3 x, U3 y) { return U3{x.a + y.a, x.b + y.b, x.c + y.c}; }
__device__ __forceinline__ U3 u3_shfl_up(U3 v, int o) {
  return U3{__shfl_up_sync(0xFFFFFFFFu, v.a, o), __shfl_up_sync(0xFFFFFFFFu, v.b, o),
            __shfl_up_sync(0xFFFFFFFFu, v.c, o)};
}
// Exclusive block scan of three counters at once.
__device__ __forceinline__ U3 block_excl_scan3(U3 v, U3* sc, U3* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  U3 inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const U3 t = u3_shfl_up(inc, o);
    if (lane >= o) inc = u3_add(inc, t);
  }
  if (lane == 31) sc[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    U3 s = (lane < nw) ? sc[lane] : U3{0, 0, 0};
    U3 si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const U3 t = u3_shfl_up(si, o);
      if (lane >= o) si = u3_add(si, t);
    }
    if (lane < nw) sc[lane] = U3{si.a - s.a, si.b - s.b, si.c - s.c};
    if (lane == nw - 1) sc[32] = si;
  }
  __syncthreads();
  const U3 base = sc[wid];
  *total = sc[32];
  const U3 r{base.a + inc.a - v.a, base.b + inc.b - v.b, base.c + inc.c - v.c};
  __syncthreads();
  return r;
}

// Reserve a tile's closed-line bytes, open-segment chars and segment ids.
__device__ __forceinline__ int reserve_space(const TileParams& p, uint32_t job, const U3& tot,
                                             unsigned long long* b) {
  const JobTab& J = p.jobs[job];
  b[0] = tot.a ? atomicAdd(p.jout + job, tot.a) : 0ull;
  b[1] = tot.b ? atomicAdd(&p.ctr->seg_char_cursor, tot.b) : 0ull;
  b[2] = tot.c ? atomicAdd(p.jseg + job, uint32_t(tot.c)) : 0u;
  if (b[0] + tot.a > J.ocap || b[1] + tot.b > p.segchars_cap || b[2] + tot.c > J.seg_cap) {
    atomicOr(&p.ctr->err, ERR_CAPACITY);
    return 0;
  }
  b[0] += J.obase;
  b[2] += J.seg_base;
  return 1;
}

// Thread-group policies: a tile is worked by a whole block or by one warp.
struct BlockGroup {
  static __device__ __forceinline__ uint32_t rank() { return threadIdx.x; }
  static __device__ __forceinline__ uint32_t size() { return blockDim.x; }
  static __device__ __forceinline__ void sync() { __syncthreads(); }
  static __device__ __forceinline__ int sync_or(int v) { return __syncthreads_or(v); }
  static __device__ __forceinline__ U3 scan3(U3 v, U3* total) {
    __shared__ U3 sc[33];
    return block_excl_scan3(v, sc, total);
  }
  // The leader reserves output space for the tile; false if a bound was hit.
  static __device__ __forceinline__ bool reserve(const TileParams& p, uint32_t job, const U3& tot,
                                                 unsigned long long* base) {
    __shared__ unsigned long long s_base[3];
    __shared__ int s_ok;
    if (threadIdx.x == 0) s_ok = reserve_space(p, job, tot, s_base);
    __syncthreads();
    base[0] = s_base[0];
    base[1] = s_base[1];
    base[2] = s_base[2];
    const int ok = s_ok;
    __syncthreads();
    return ok;
  }
};

struct WarpGroup {
  static __device__ __forceinline__ uint32_t rank() { return threadIdx.x & 31u; }
  static __device__ __forceinline__ uint32_t size() { return 32u; }
  static __device__ __forceinline__ void sync() { __syncwarp(); }
  static __device__ __forceinline__ int sync_or(int v) { return __any_sync(0xFFFFFFFFu, v); }
  // a warp tile's totals fit 32 bits (at most 256 copies)
  static __device__ __forceinline__ U3 scan3(U3 v, U3* total) {
    const int lane = threadIdx.x & 31;
    uint32_t a = uint32_t(v.a), b = uint32_t(v.b), c = uint32_t(v.c);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t ta = __shfl_up_sync(0xFFFFFFFFu, a, o), tb = __shfl_up_sync(0xFFFFFFFFu, b, o),
                     tc = __shfl_up_sync(0xFFFFFFFFu, c, o);
      if (lane >= o) {
        a += ta;
        b += tb;
        c += tc;
      }
    }
    *total = U3{__shfl_sync(0xFFFFFFFFu, a, 31), __shfl_sync(0xFFFFFFFFu, b, 31), __shfl_sync(0xFFFFFFFFu, c, 31)};
    return U3{a - uint32_t(v.a), b - uint32_t(v.b), c - uint32_t(v.c)};
  }
  static __device__ __forceinline__ bool reserve(const TileParams& p, uint32_t job, const U3& tot,
                                                 unsigned long long* base) {
    unsigned long long b[3] = {0, 0, 0};
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = reserve_space(p, job, tot, b);
    base[0] = __shfl_sync(0xFFFFFFFFu, b[0], 0);
    base[1] = __shfl_sync(0xFFFFFFFFu, b[1], 0);
    base[2] = __shfl_sync(0xFFFFFFFFu, b[2], 0);
    return __shfl_sync(0xFFFFFFFFu, ok, 0);
  }
};

// Pointer-jumping rounds over (px, rx) with second buffers (py, ry); the
// result lands in (ptr, rnk).  Starts point at themselves with rank 0.
template <typename G, typename IT>
__device__ void jump_rounds(uint32_t c, IT* px, IT* rx, IT* py, IT* ry, IT*& ptr, IT*& rnk) {
  uint32_t rounds = 1;
  for (uint32_t lim = 1; lim < c; lim <<= 1) ++rounds;
  for (uint32_t r = 0; r < rounds; ++r) {
    int changed = 0;
    for (uint32_t i = G::rank(); i < c; i += G::size()) {
      const uint32_t p = px[i];
      const uint32_t np = px[p];
      py[i] = IT(np);
      ry[i] = IT(uint32_t(rx[i]) + uint32_t(rx[p]));
      changed |= (np != p);
    }
    IT* t = px; px = py; py = t;
    t = rx; rx = ry; ry = t;
    if (!G::sync_or(changed)) break;
  }
  ptr = px;
  rnk = rx;
}

// KC: k fixed at compile time (0: p.k), so that the masks, shifts and
// spelling loops of the common shapes are constants.
template <int NW, typename IT, typename G, int KC = 0>
__device__ void process_tile(const TileParams& p, const TileMem<NW, IT>& m, uint64_t beg, uint32_t c,
                             uint32_t job) {
  constexpr uint32_t NONE_I = Ix<IT>::NONE, DUP_I = Ix<IT>::DUP, CNONE_I = Ix<IT>::CNONE;
  constexpr uint32_t OPEN_S = NONE_I - 1u;  // an open segment that starts at an S-only copy
  const int k = KC ? KC : p.k;
  const PrefMask pm = pref_mask(k);
  // this tile's hash slots: the power of two above c * lf / 100, at most the
  // carved table (32-bit arithmetic for shared-memory tiles, c <= 8192)
  uint32_t ts;
  {
    const uint32_t want = (sizeof(IT) == 2) ? (c * p.lf) / 100u : uint32_t((uint64_t(c) * p.lf) / 100u);
    const uint32_t x = want > c ? want : c + 1u;
    ts = 1u << (32 - __clz(x - 1u));
    ts = ts < m.ts ? ts : m.ts;
  }
  const uint32_t tmask = ts - 1;
  // ---- stage the tile's keys (async copies), initialise the work arrays
  if constexpr (sizeof(IT) == 2) {
    // shared-memory tile: asynchronous copies overlap the initialisation
    for (uint32_t i = G::rank(); i < c; i += G::size())
      __pipeline_memcpy_async(m.key + size_t(i) * NW, p.pkeys + (beg + i) * NW, 8 * NW);
    __pipeline_commit();
  } else {
    for (uint32_t i = G::rank(); i < c; i += G::size()) {
      const Key<NW> x = ld_key<NW>(p.pkeys, beg + i);
#pragma unroll
      for (int w = 0; w < NW; ++w) m.key[size_t(i) * NW + w] = x.w[w];
    }
  }
  if constexpr (sizeof(IT) == 2) {
    // four 16-bit entries per store (carve sizes the arrays in fours)
    uint64_t* A4 = reinterpret_cast<uint64_t*>(m.A);
    uint64_t* B4 = reinterpret_cast<uint64_t*>(m.B);
    uint64_t* P4 = reinterpret_cast<uint64_t*>(m.P);
    for (uint32_t i = G::rank(); i < (c + 3u) >> 2; i += G::size()) {
      A4[i] = 0x7FFF7FFF7FFF7FFFull;  // CNONE
      B4[i] = 0ull;
      P4[i] = ~0ull;                  // NONE
    }
    if (ts >= 4) {
      uint64_t* T4 = reinterpret_cast<uint64_t*>(m.T);
      for (uint32_t i = G::rank(); i < (ts >> 2); i += G::size()) T4[i] = ~0ull;
    } else {
      for (uint32_t i = G::rank(); i < ts; i += G::size()) m.T[i] = IT(NONE_I);
    }
  } else {
    for (uint32_t i = G::rank(); i < c; i += G::size()) {
      m.A[i] = IT(CNONE_I);
      m.B[i] = 0;
      m.P[i] = IT(NONE_I);
    }
    for (uint32_t i = G::rank(); i < ts; i += G::size()) m.T[i] = IT(NONE_I);
  }
  if constexpr (sizeof(IT) == 2) __pipeline_wait_prior(0);
  G::sync();
  // ---- prefix table of the P copies (generate_hashmap, assembler.h:120-150):
  // one slot per distinct (k-1)-prefix; a prefix held by two copies marks the
  // slot's copy DUP ("nullified")
  for (uint32_t i = G::rank(); i < c; i += G::size()) {
    const Key<NW> x = skey(m, i);
    if (!(roles(x) & ROLE_P)) continue;
    const Key<NW> pf = prefix_of(x, pm);
    uint32_t h = key_hash(pf) & tmask;
    for (uint32_t probe = 0; probe <= tmask; ++probe) {
      const uint32_t cur = at_cas(m.T + h, NONE_I, i);
      if (cur == NONE_I) break;
      if (key_eq(prefix_of(skey(m, cur), pm), pf)) {
        at_or(m.A + cur, DUP_I);
        break;
      }
      h = (h + 1) & tmask;
    }
  }
  G::sync();
  // ---- suffix lookups of the S copies (find_vtx_from_edge, assembler.h:89-111)
  // and in-degree counts ("count edges", assembler.h:180-188)
  for (uint32_t i = G::rank(); i < c; i += G::size()) {
    const Key<NW> x = skey(m, i);
    if (!(roles(x) & ROLE_S)) continue;
    const Key<NW> sf = suffix_of(x, pm);
    uint32_t h = key_hash(sf) & tmask;
    uint32_t cand = CNONE_I;
    for (uint32_t probe = 0; probe <= tmask; ++probe) {
      const uint32_t cur = m.T[h];
      if (cur == NONE_I) break;
      if (key_eq(prefix_of(skey(m, cur), pm), sf)) {
        if (!(uint32_t(m.A[cur]) & DUP_I)) cand = cur;
        break;
      }
      h = (h + 1) & tmask;
    }
    if (cand != CNONE_I) {
      at_inc(m.B + cand);
      m.P[cand] = IT(i);
    }
    m.A[i] = IT((uint32_t(m.A[i]) & DUP_I) | cand);
  }
  G::sync();
  // ---- kept edges: u->v iff v is u's unique successor and u is v's only
  // predecessor ("write edges", assembler.h:189-197); rank init alongside
  for (uint32_t i = G::rank(); i < c; i += G::size()) {
    const uint32_t cand = uint32_t(m.A[i]) & CNONE_I;
    const uint32_t s = (cand != CNONE_I && m.B[cand] == 1u) ? cand : NONE_I;
    const uint32_t q = (m.B[i] == 1u) ? uint32_t(m.P[i]) : NONE_I;
    m.A[i] = IT(s);
    m.P[i] = IT(q);
    m.Q[i] = IT(q == NONE_I ? i : q);
    m.T[i] = IT(q == NONE_I ? 0u : 1u);
  }
  G::sync();
  if (p.mode == 0) {
    for (uint32_t i = G::rank(); i < c; i += G::size()) {
      const uint64_t r = roles(skey(m, i));
      const uint32_t id = p.plink[beg + i];
      if (r & ROLE_S) p.succ[id] = (m.A[i] == NONE_I) ? NONE : p.plink[beg + m.A[i]];
      if (r & ROLE_P) p.pred[id] = (m.P[i] == NONE_I) ? NONE : p.plink[beg + m.P[i]];
    }
    return;
  }
  // ---- local segments: list ranking by pointer jumping
  IT *ptr, *rnk;
  jump_rounds<G, IT>(c, m.Q, m.T, m.B, m.T + c, ptr, rnk);
  // ---- local cycles (every copy has a local predecessor): cut each at its
  // smallest key, then rank again
  int cyc = 0;
  for (uint32_t i = G::rank(); i < c; i += G::size()) {
    // a path copy points at its start (no predecessor); a cycle copy at
    // another cycle copy.  Cycle copies have a successor, so A = index | DUP.
    if (m.P[ptr[i]] != NONE_I) {
      m.A[i] = IT(uint32_t(m.A[i]) | DUP_I);
      cyc = 1;
    }
  }
  if (G::sync_or(cyc)) {
    IT *lx = m.T, *jx = m.T + c, *ly = m.B, *jy = m.Q;
    for (uint32_t i = G::rank(); i < c; i += G::size()) {
      lx[i] = IT(i);
      jx[i] = IT(m.P[i] == NONE_I ? i : uint32_t(m.P[i]));
    }
    G::sync();
    uint32_t rounds = 1;
    for (uint32_t lim = 1; lim < c; lim <<= 1) ++rounds;
    for (uint32_t r = 0; r < rounds; ++r) {
      for (uint32_t i = G::rank(); i < c; i += G::size()) {
        const uint32_t j = jx[i];
        const uint32_t a = lx[i], b = lx[j];
        ly[i] = IT(key_lt(skey(m, b), skey(m, a)) ? b : a);
        jy[i] = jx[j];
      }
      G::sync();
      IT* t = lx; lx = ly; ly = t;
      t = jx; jx = jy; jy = t;
    }
    // after ceil(log2 c)+1 rounds a cycle copy's label covers its whole cycle:
    // exactly one copy per cycle (the smallest key) is its own label; the edge
    // into it is cut, path copies are untouched
    auto on_cycle = [](uint32_t a) { return a != NONE_I && (a & DUP_I); };
    for (uint32_t i = G::rank(); i < c; i += G::size()) {
      if (on_cycle(m.A[i]) && lx[i] == i) {
        const uint32_t q = m.P[i];
        m.A[q] = IT(NONE_I);
        m.P[i] = IT(NONE_I);
      }
    }
    G::sync();
    for (uint32_t i = G::rank(); i < c; i += G::size()) {
      const uint32_t a = m.A[i];
      if (on_cycle(a)) m.A[i] = IT(a & ~DUP_I);
      const uint32_t q = m.P[i];
      m.Q[i] = IT(q == NONE_I ? i : q);
      m.T[i] = IT(q == NONE_I ? 0u : 1u);
    }
    G::sync();
    jump_rounds<G, IT>(c, m.Q, m.T, m.B, m.T + c, ptr, rnk);
  }
  // every copy now reaches a segment start.  Free arrays: the pair not
  // holding (ptr, rnk) keeps each start's byte offset (lo/hi halves), P its
  // local segment id.
  IT* lo_a = (ptr == m.Q) ? m.B : m.Q;
  IT* hi_a = (rnk == m.T) ? m.T + c : m.T;
  // ---- emission: closed segments (start has role P, end has role S) are
  // whole unitigs; the others are stitched across tiles.  Open segments that
  // start at a P-role copy start a stitched line: they take head-pool ids;
  // the others start at an S-only copy and take its cross index.
  // A warp tile first packs its segment ends into a list (in A, which only
  // marked the ends from here on), so that the per-segment loops keep every
  // lane busy; a block tile walks its copies and skips the others.  Each
  // thread's lines are contiguous in the tile's output, in the order the
  // thread visits them (the order of lines is free).
  constexpr bool WARP = std::is_same<G, WarpGroup>::value;
  uint32_t nend = c;
  if constexpr (WARP) {
    const uint32_t lane = G::rank();
    nend = 0;
    for (uint32_t base = 0; base < c; base += 32) {
      const uint32_t i = base + lane;
      const bool e = i < c && m.A[i] == NONE_I;
      const uint32_t mask = __ballot_sync(0xFFFFFFFFu, e);
      __syncwarp();  // the reads of this chunk before any write into it
      if (e) m.A[nend + __popc(mask & ((1u << lane) - 1u))] = IT(i);
      nend += uint32_t(__popc(mask));
    }
    __syncwarp();
  }
  // the segment end visited at step j (NONE_I: not an end)
  auto end_at = [&](uint32_t j) -> uint32_t {
    if constexpr (WARP) return m.A[j];
    else return m.A[j] == NONE_I ? j : NONE_I;
  };
  U3 mine{0, 0, 0};
  for (uint32_t j = G::rank(); j < nend; j += G::size()) {
    const uint32_t i = end_at(j);
    if (i == NONE_I) continue;
    const uint32_t s = ptr[i];
    const uint32_t len = uint32_t(rnk[i]) + 1;
    const bool starts_p = (roles(skey(m, s)) & ROLE_P) != 0;
    const bool closed = starts_p && (roles(skey(m, i)) & ROLE_S);
    if (closed) mine.a += uint64_t(k) + len;
    else { mine.b += starts_p ? uint64_t(k) - 1 + len : uint64_t(len) - 1; mine.c += starts_p ? 1 : 0; }
  }
  U3 tot;
  U3 pre = G::scan3(mine, &tot);
  unsigned long long s_base[3];
  if (!G::reserve(p, job, tot, s_base)) return;
  const unsigned long long cbase = s_base[0], obase = s_base[1], sbase = s_base[2];
  // per segment (the lane that sized it): its offset (kept at its start for
  // the per-copy pass), its first k-mer in full (a segment that starts at an
  // S-only copy keeps only the chars it adds to its line: that k-mer ends
  // the segment before), then its line break or, for an open segment, its
  // record.  The cross indices the record needs are loaded first, so that
  // they arrive while the rest is worked out.
  for (uint32_t j = G::rank(); j < nend; j += G::size()) {
    const uint32_t i = end_at(j);
    if (i == NONE_I) continue;
    const uint32_t s = ptr[i];
    const Key<NW> ks = skey(m, s);
    const uint64_t re = roles(skey(m, i));
    const bool starts_p = (roles(ks) & ROLE_P) != 0;
    const bool p_only = (re & ROLE_S) == 0;
    const bool closed = starts_p && !p_only;
    const uint32_t xs = starts_p ? NONE : p.plink[beg + s];  // this segment's id (S-only start)
    const uint32_t xe = p_only ? p.plink[beg + i] : NONE;   // the next segment's id
    const uint32_t r = rnk[i];
    const uint32_t len = r + 1;
    uint64_t loc;
    uint32_t sid;
    if (closed) {
      loc = pre.a;
      sid = NONE_I;
      pre.a += uint64_t(k) + len;
    } else {
      loc = pre.b;
      sid = starts_p ? uint32_t(pre.c) : OPEN_S;
      pre.b += starts_p ? uint64_t(k) - 1 + len : uint64_t(len) - 1;
      if (starts_p) pre.c += 1;
    }
    m.P[s] = IT(sid);
    if constexpr (sizeof(IT) == 2) {
      lo_a[s] = IT(loc & 0xFFFFu);
      hi_a[s] = IT(loc >> 16);
    } else {
      lo_a[s] = IT(loc);
    }
    char* dst = closed ? (p.out + cbase + loc) : (p.segchars + obase + loc);
    if (sid != OPEN_S) spell_key<NW>(dst, ks, k);
    if (closed) {
      dst[k + r] = '\n';
    } else {
      // the segment's record under its id; a segment that ends at the P-only
      // copy of cross k-mer xe continues in segment xe
      const uint32_t g = starts_p ? p.xcount + uint32_t(sbase) + sid : xs;
      SegRec rec;
      rec.off_job = (obase + loc) | (static_cast<unsigned long long>(job) << SEG_OFF_BITS);
      rec.len = len;
      rec.next = xe;
      p.seg[g] = rec;
    }
  }
  G::sync();
  // every later copy of a segment adds its last char
  for (uint32_t i = G::rank(); i < c; i += G::size()) {
    const uint32_t r = rnk[i];
    if (r == 0) continue;
    const uint32_t s = ptr[i];
    uint64_t loc = lo_a[s];
    if constexpr (sizeof(IT) == 2) loc |= uint64_t(hi_a[s]) << 16;
    const uint32_t sid = m.P[s];
    char* dst = (sid == NONE_I) ? (p.out + cbase + loc) : (p.segchars + obase + loc);
    dst[(sid == OPEN_S ? 0u : uint32_t(k)) + r - 1] = acgt(key_char(skey(m, i), k - 1));
  }
}

// Persistent tile kernels.  Warp tiles (<= warp capacity copies): every warp
// of a CTA owns a slice of shared memory and takes the next warp tile from a
// global counter, with warp-level synchronisation only.  Block tiles (up to
// the tile capacity): the whole CTA works one tile.  Larger tiles go to
// k_tile_big.
template <int NW, int KC>
__global__ void __launch_bounds__(256) k_tile_warp(TileParams p) {
  extern __shared__ __align__(16) char smem[];
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const TileMem<NW, uint16_t> m = carve<NW, uint16_t>(smem + size_t(wid) * p.wbytes, p.wcap, p.wts);
  const uint32_t nt = p.ctr->nwarp;
  uint32_t j = 0;
  if (lane == 0) j = atomicAdd(&p.ctr->wtile_next, 1u);
  j = __shfl_sync(0xFFFFFFFFu, j, 0);
  while (j < nt) {
    uint32_t jn = 0;  // the next tile's index is in flight while this tile is worked
    if (lane == 0) jn = atomicAdd(&p.ctr->wtile_next, 1u);
    const uint32_t t = p.wlist[j];
    const uint64_t beg = p.tile_begin[t];
    const uint32_t c = uint32_t(p.tile_begin[t + 1] - beg);
    process_tile<NW, uint16_t, WarpGroup, KC>(p, m, beg, c, p.tile_job[t]);
    __syncwarp();
    j = __shfl_sync(0xFFFFFFFFu, jn, 0);
  }
}

template <int NW, int KC>
__global__ void __launch_bounds__(512) k_tile(TileParams p) {
  extern __shared__ __align__(16) char smem[];
  __shared__ uint32_t s_t;
  const TileMem<NW, uint16_t> m = carve<NW, uint16_t>(smem, p.cap, p.tslots);
  const uint32_t nt = p.ctr->nblock;
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(&p.ctr->tile_next, 1u);
    __syncthreads();
    const uint32_t j = s_t;
    __syncthreads();
    if (j >= nt) break;
    const uint32_t t = p.blist[j];
    const uint64_t beg = p.tile_begin[t];
    const uint32_t c = uint32_t(p.tile_begin[t + 1] - beg);
    process_tile<NW, uint16_t, BlockGroup, KC>(p, m, beg, c, p.tile_job[t]);
    __syncthreads();
  }
}

// One CTA per oversized tile, working in global scratch.
template <int NW>
__global__ void __launch_bounds__(1024) k_tile_big(TileParams p) {
  const uint32_t t = p.big_list[blockIdx.x];
  const uint64_t beg = p.tile_begin[t];
  const uint64_t c = p.tile_begin[t + 1] - beg;
  const uint32_t ts = big_slots(c, p.lf);
  const TileMem<NW, uint32_t> m = carve<NW, uint32_t>(p.big_scratch + p.big_off[blockIdx.x], uint32_t(c), ts);
  process_tile<NW, uint32_t, BlockGroup>(p, m, beg, uint32_t(c), p.tile_job[t]);
}

// ================================================================= stitch
//
// Open segments continue through cross k-mers: the segment that ends at the
// P-only copy of cross k-mer x is followed by segment x (the one that starts
// at x's S-only copy); both hold x, so every later segment of a line drops
// its first k chars (write_unitigs4, compact.h:59-112), and the tiles keep
// only the chars it adds.  The tiles write each segment's record under its
// id.  The common case is one kernel (k_walk_emit): a thread per line head
// walks its line twice, once for its length, then, after one output
// reservation per job and warp, to copy the segments' chars into one
// contiguous line.  Lines longer than WALK_CAP segments and cycles (no
// head) go through list ranking (pointer jumping from the first state
// rebuilt from the records, or HEC), line lengths at the heads
// (k_chain_len), one reservation per line (k_line_reserve) and a copy per
// segment (k_seg_copy).

// The chars a segment adds to its line: all k - 1 + len for a line's first
// segment (a head-pool id), len - 1 for the others.
__device__ __forceinline__ uint32_t seg_w(uint32_t s, uint32_t len, uint32_t nx, int k) {
  return s < nx ? len - 1u : uint32_t(k) - 1u + len;
}

// First of c consecutive slots for each thread of a block that appends to a
// shared list: one atomic per block.  A list counter that every block of the
// grid bumps serialises in L2, so per-warp appends would bound a pass that
// appends most of its elements.  Every thread of the block must call it;
// sc holds 33 values.
__device__ __forceinline__ uint32_t block_append(uint32_t* count, uint32_t c, uint32_t* sc) {
  uint32_t tot;
  const uint32_t pre = block_excl_scan(c, sc, &tot);  // ends with a barrier after every read of sc
  if (threadIdx.x == 0) sc[32] = tot ? atomicAdd(count, tot) : 0u;
  __syncthreads();
  const uint32_t b = sc[32] + pre;
  __syncthreads();  // sc is reused by the next call
  return b;
}

// X[v] = (start pointer, weight distance); heads point at themselves.
__global__ void __launch_bounds__(256) k_rank_init(const uint32_t* __restrict__ prev, const uint32_t* __restrict__ w,
                            uint64_t n, const Counters* ctr, unsigned long long* __restrict__ X,
                            uint32_t* __restrict__ act, uint32_t* act_count) {
  __shared__ uint32_t sc[33];
  const uint64_t N = ctr ? uint64_t(ctr->seg_count) : n;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  // whole blocks iterate together (block_append needs every thread)
  for (uint64_t s0 = uint64_t(blockIdx.x) * blockDim.x; s0 < N; s0 += stride) {
    const uint64_t s = s0 + threadIdx.x;
    bool tail = false;
    if (s < N) {
      const uint32_t pv = prev[s];
      if (pv == NONE) {
        X[s] = pk(uint32_t(s) | HEAD_BIT, 0);
      } else {
        X[s] = pk(pv, w ? w[pv] : 1u);
        tail = true;
      }
    }
    const uint32_t slot = block_append(act_count, tail ? 1u : 0u, sc);
    if (tail) act[slot] = uint32_t(s);
  }
}

// One round of asynchronous pointer jumping over the active list (act ==
// nullptr: the first round, over the ids [0, *act_count)).  Entries are
// (pointer, distance) pairs in one 64-bit word, so a concurrent reader
// always sees a consistent pair; the list keeps the entries whose pointer
// does not yet reach a head.  Any mix of first-state entries (predecessor,
// its chars) and final ones (head, chars before) is a valid state.
__global__ void __launch_bounds__(256) k_rank_round(unsigned long long* __restrict__ X, const uint32_t* __restrict__ act,
                             const uint32_t* act_count, uint32_t* __restrict__ act_out,
                             uint32_t* act_out_count) {
  __shared__ uint32_t sc[33];
  const uint32_t na = *act_count;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  // whole blocks iterate together (block_append needs every thread)
  for (uint64_t j0 = uint64_t(blockIdx.x) * blockDim.x; j0 < na; j0 += stride) {
    const uint64_t j = j0 + threadIdx.x;
    bool keep = false;
    uint32_t s = 0;
    if (j < na) {
      s = act ? act[j] : uint32_t(j);
      const unsigned long long v = reinterpret_cast<volatile unsigned long long*>(X)[s];
      const unsigned long long u = reinterpret_cast<volatile unsigned long long*>(X)[ptr_of(v)];
      if (!is_head_entry(u)) {  // not yet pointing at a head
        const unsigned long long nv = pk(ptr_of(u), pk_o(v) + pk_o(u));
        reinterpret_cast<volatile unsigned long long*>(X)[s] = nv;
        const unsigned long long z = reinterpret_cast<volatile unsigned long long*>(X)[ptr_of(nv)];
        keep = !is_head_entry(z);
      }
    }
    const uint32_t slot = block_append(act_out_count, keep ? 1u : 0u, sc);
    if (keep) act_out[slot] = s;
  }
}

// ---- the line walk
constexpr uint32_t WALK_CAP = 1024;                // segments a line walk follows
constexpr int WALK_REG = 4;                         // later segments a walk keeps in registers
constexpr unsigned long long LINE_WALKED = ~0ull;  // line base of a line k_walk_emit wrote
constexpr uint32_t JOB_NONE = 0xFFFFFFFFu;

// Reserves want bytes of job's output for each lane of a warp (every lane
// calls; a lane with want 0 or job JOB_NONE takes nothing) with one atomic
// per job present in the warp.  The lanes of one job must be consecutive,
// apart from lanes that take nothing (head-pool ids lie in job order).
// Returns the lane's offset in its job's output.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long* jout, uint32_t job,
                                                           unsigned long long want) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long inc = want;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long v = __shfl_up_sync(0xFFFFFFFFu, inc, d);
    if (lane >= uint32_t(d)) inc += v;
  }
  const uint32_t grp = __match_any_sync(0xFFFFFFFFu, job);
  const uint32_t first = uint32_t(__ffs(grp)) - 1u, last = 31u - uint32_t(__clz(grp));
  const unsigned long long before = __shfl_sync(0xFFFFFFFFu, inc - want, first);
  const unsigned long long total = __shfl_sync(0xFFFFFFFFu, inc, last) - before;
  unsigned long long base = 0;
  if (lane == first && job != JOB_NONE && total) base = atomicAdd(jout + job, total);
  base = __shfl_sync(0xFFFFFFFFu, base, first);
  return base + (inc - want - before);
}

// One thread writes one line: whole aligned 4-byte words as they fill, and
// byte by byte the bytes of its first and last words (which it shares with
// the neighbouring lines, or which lie outside the output buffer: the
// buffer may start at any byte).  Positions are addresses.
struct LineOut {
  uintptr_t p;   // next byte of the line
  uintptr_t p0;  // its first byte
  uint32_t acc;  // the bytes of the word at p & ~3 below p
};

// 4 bytes at any alignment from two aligned words (the segment chars'
// allocation ends with slack, so the second word is inside it)
__device__ __forceinline__ uint32_t load4u(const char* src) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = 8u * uint32_t(a & 3u);
  return sh ? __funnelshift_r(w[0], w[1], sh) : w[0];
}

// Appends bytes [0, n) of v (n <= 4 - (p & 3)) and stores the word they fill.
__device__ __forceinline__ void line_bytes(LineOut& L, uint32_t v, uint32_t n) {
  const uint32_t fill = uint32_t(L.p & 3u);
  const uintptr_t wpos = L.p - fill;
  L.acc |= (n == 4 ? v : (v & ((1u << (8 * n)) - 1u))) << (8 * fill);
  L.p += n;
  if (fill + n == 4) {
    if (wpos >= L.p0) {
      *reinterpret_cast<uint32_t*>(wpos) = L.acc;
    } else {
      for (uint32_t b = uint32_t(L.p0 - wpos); b < 4; ++b) reinterpret_cast<char*>(wpos)[b] = char(L.acc >> (8 * b));
    }
    L.acc = 0;
  }
}

// Appends n bytes from src: up to the destination's next word boundary,
// then whole words from an aligned source stream (one new load per word),
// then the rest.
__device__ __forceinline__ void line_put(LineOut& L, const char* src, uint32_t n) {
  const uint32_t head = min(n, (4u - uint32_t(L.p & 3u)) & 3u);
  if (head) {
    line_bytes(L, load4u(src), head);
    src += head;
    n -= head;
  }
  if (n >= 4) {
    // the destination is word aligned here and the words lie inside the line
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    const uint32_t sh = 8u * uint32_t(a & 3u);
    uint32_t* d = reinterpret_cast<uint32_t*>(L.p);
    const uint32_t nw = n >> 2;
    uint32_t cur = w[0];
    for (uint32_t i = 0; i < nw; ++i) {
      const uint32_t nxt = sh ? w[i + 1] : 0u;
      d[i] = sh ? __funnelshift_r(cur, nxt, sh) : w[i];
      cur = nxt;
    }
    L.p += 4u * nw;
    src += 4u * nw;
    n &= 3u;
  }
  if (n) line_bytes(L, load4u(src), n);
}

// Appends n <= 4 bytes held in v (its low bytes first).
__device__ __forceinline__ void line_put4(LineOut& L, uint32_t v, uint32_t n) {
  const uint32_t take = min(n, 4u - uint32_t(L.p & 3u));
  if (take) line_bytes(L, v, take);
  if (n > take) line_bytes(L, v >> (8 * take), n - take);
}

// The line break, then the bytes of the last word not yet stored.
__device__ __forceinline__ void line_end(LineOut& L) {
  line_bytes(L, uint32_t('\n'), 1);
  const uint32_t fill = uint32_t(L.p & 3u);
  if (fill) {
    const uintptr_t wpos = L.p - fill;
    for (uint32_t b = (wpos >= L.p0 ? 0u : uint32_t(L.p0 - wpos)); b < fill; ++b)
      reinterpret_cast<char*>(wpos)[b] = char(L.acc >> (8 * b));
  }
}

// Every stitched line from its head, one thread per head-pool id: the walk
// follows the line's records for its length (up to WALK_CAP segments after
// the head; the first WALK_REG records stay in registers), the warp
// reserves its lines' bytes, and the walk copies each segment's chars into
// the line (records past the kept ones read again, now mostly in L2).  A line that goes on past WALK_CAP segments is left to the ranking
// path: its head goes to longl.  wst[0] counts the segments of the lines
// written (those with ids below nx), wst[1] the lines left.  cap <=
// WALK_CAP (smaller only to test the ranking path).
__global__ void __launch_bounds__(256) k_walk_emit(uint32_t H, const SegRec* __restrict__ seg, uint32_t nx, int k,
                                                   const JobTab* __restrict__ jobs, unsigned long long* __restrict__ jout,
                                                   const char* __restrict__ segchars, char* __restrict__ out,
                                                   uint32_t cap, uint32_t* __restrict__ longl, uint32_t lcap,
                                                   uint32_t* wst, Counters* ctr) {
  __shared__ uint32_t sc[33];
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  uint32_t walked = 0;
  // whole warps iterate together (warp_reserve needs every lane)
  for (uint64_t h0 = uint64_t(blockIdx.x) * blockDim.x; h0 < H; h0 += stride) {
    const uint64_t h = h0 + threadIdx.x;
    SegRec r{0ull, 0u, NONE};
    if (h < H) r = seg[nx + h];
    const bool live = r.len != 0;
    unsigned long long len = live ? uint64_t(k) - 1u + r.len : 0ull;
    uint32_t s = live ? r.next : NONE, hops = 0;
    // the first WALK_REG later segments stay in registers for the copy
    SegRec c[WALK_REG];
#pragma unroll
    for (int q = 0; q < WALK_REG; ++q) {
      c[q] = SegRec{0ull, 1u, NONE};
      if (s < nx && hops < cap) {
        c[q] = seg[s];
        len += c[q].len - 1u;
        s = c[q].next;
        ++hops;
      }
    }
    while (s < nx && hops < cap) {
      const SegRec q = seg[s];
      len += q.len - 1u;
      s = q.next;
      ++hops;
    }
    const bool done = live && s == NONE;
    const uint32_t job = done ? uint32_t(r.off_job >> SEG_OFF_BITS) : JOB_NONE;
    const unsigned long long o = warp_reserve(jout, job, done ? len + 1u : 0ull);
    if (live && !done) {
      const uint32_t i = atomicAdd(wst + 1, 1u);
      if (i < lcap) longl[i] = uint32_t(h);
      else atomicOr(&ctr->err, ERR_INTERNAL);  // a left line holds more than cap cross ids
    }
    if (done) {
      walked += hops;
      const JobTab& J = jobs[job];
      if (o + len + 1u > J.ocap) {
        atomicOr(&ctr->err, ERR_CAPACITY);
      } else {
        // the kept segments' first words load together (most later
        // segments add no more than 4 chars)
        uint32_t fw[WALK_REG];
#pragma unroll
        for (int q = 0; q < WALK_REG; ++q)
          fw[q] = (uint32_t(q) < hops && c[q].len > 1u) ? load4u(segchars + (c[q].off_job & SEG_OFF_MASK)) : 0u;
        const uintptr_t a = reinterpret_cast<uintptr_t>(out + J.obase + o);
        LineOut L{a, a, 0u};
        line_put(L, segchars + (r.off_job & SEG_OFF_MASK), uint32_t(k) - 1u + r.len);
#pragma unroll
        for (int q = 0; q < WALK_REG; ++q) {
          if (uint32_t(q) < hops) {
            const uint32_t n = c[q].len - 1u;
            if (n <= 4u) line_put4(L, fw[q], n);
            else line_put(L, segchars + (c[q].off_job & SEG_OFF_MASK), n);
          }
        }
        uint32_t t = c[WALK_REG - 1].next;
        for (uint32_t q = WALK_REG; q < hops; ++q) {
          const SegRec g = seg[t];
          line_put(L, segchars + (g.off_job & SEG_OFF_MASK), g.len - 1u);
          t = g.next;
        }
        line_end(L);
      }
    }
  }
  uint32_t tot;
  block_excl_scan(walked, sc, &tot);
  if (threadIdx.x == 0 && tot) atomicAdd(wst, tot);
}

// The ranking's first state from the segment records (when the walk left
// lines or cycles, and for HEC): a line's first segment is a head; segment
// x (x < nx) points at its predecessor, with the chars the predecessor adds.
__global__ void __launch_bounds__(256) k_seg_xinit(uint32_t S, const SegRec* __restrict__ seg, uint32_t nx, int k,
                                                   unsigned long long* __restrict__ X) {
  for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < S; s += uint64_t(gridDim.x) * blockDim.x) {
    const SegRec r = seg[s];
    if (!r.len) continue;
    if (s >= nx) X[s] = pk(uint32_t(s) | HEAD_BIT, 0);
    if (r.next < nx) X[r.next] = pk(uint32_t(s), seg_w(uint32_t(s), r.len, nx, k));
  }
}

__global__ void k_set_u32(uint32_t* p, uint32_t v) { *p = v; }

// Line length of each chain, stored at its head (every live chain has one
// tail, which writes it; the array is zeroed before).  A line's tail starts
// at an S-only copy (a line's first segment always continues).
__global__ void k_chain_len(uint32_t S, const SegRec* __restrict__ seg, const unsigned long long* __restrict__ X,
                            const uint8_t* __restrict__ oncycle, uint32_t nx, int k, uint32_t* __restrict__ linelen,
                            Counters* ctr) {
  constexpr int PER = 4;  // slots per thread and pass: their loads are in flight together
  const uint64_t span = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t s0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s0 < S; s0 += span * PER) {
    SegRec r[PER];
    uint8_t cyc[PER];
    unsigned long long v[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const uint64_t s = s0 + uint64_t(q) * span;
      const bool in = s < S;
      r[q] = in ? seg[s] : SegRec{0ull, 0u, 0u};
      cyc[q] = in ? oncycle[s] : uint8_t(1);
      v[q] = in ? X[s] : 0ull;
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      if (!r[q].len || r[q].next != NONE || cyc[q]) continue;
      const uint32_t h = ptr_of(v[q]);
      const uint32_t s = uint32_t(s0 + uint64_t(q) * span);
      if (h < nx || h >= S) {
        atomicOr(&ctr->err, ERR_INTERNAL);
        continue;
      }
      linelen[h - nx] = pk_o(v[q]) + seg_w(s, r[q].len, nx, k) + 1u;
    }
  }
}

// Each line's base in the output, reserved after the job's lines so far:
// over the heads in list (the lines the walk left), or over all head-pool
// ids (list == nullptr, after HEC ranking: one reservation per job and
// warp).  A head without a length keeps LINE_WALKED, so no segment copies
// into it.
__global__ void __launch_bounds__(256) k_line_reserve(uint32_t n, const uint32_t* __restrict__ list,
                                                      const SegRec* __restrict__ heads,
                                                      const JobTab* __restrict__ jobs,
                                                      unsigned long long* __restrict__ jout,
                                                      const uint32_t* __restrict__ hlen,
                                                      unsigned long long* __restrict__ lbase, Counters* ctr) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  // whole warps iterate together (warp_reserve needs every lane)
  for (uint64_t i0 = uint64_t(blockIdx.x) * blockDim.x; i0 < n; i0 += stride) {
    const uint64_t i = i0 + threadIdx.x;
    uint32_t h = 0, job = JOB_NONE, want = 0;
    if (i < n) {
      h = list ? list[i] : uint32_t(i);
      const SegRec r = heads[h];
      want = r.len ? hlen[h] : 0u;
      if (want) job = uint32_t(r.off_job >> SEG_OFF_BITS);
    }
    // a list's heads come in any job order: one atomic each
    const unsigned long long o = list ? (want ? atomicAdd(jout + job, (unsigned long long)want) : 0ull)
                                      : warp_reserve(jout, job, want);
    if (want) {
      const JobTab& J = jobs[job];
      if (o + want > J.ocap) atomicOr(&ctr->err, ERR_CAPACITY);
      else lbase[h] = J.obase + o;
    }
  }
}

// Copy each segment's chars into its line.  A warp takes 4 x 32 consecutive
// segments: each lane resolves four segments' source, destination and
// length (their records and ranking entries, then their heads' line bases;
// all four gathers in flight together), then groups of 8 lanes copy the
// segments word by word.
__global__ void __launch_bounds__(256) k_seg_copy(
    uint32_t S, const SegRec* __restrict__ seg, const unsigned long long* __restrict__ X,
    const uint8_t* __restrict__ oncycle, uint32_t nx, const unsigned long long* __restrict__ lbase,
    const char* __restrict__ segchars, char* __restrict__ out, int k) {
  constexpr int PER = 4;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = uint64_t(warp) * 32u * PER; base < S; base += uint64_t(nwarps) * 32u * PER) {
    uint64_t dst[PER], src[PER];
    uint32_t nb[PER], last[PER], hd[PER];
    unsigned long long off[PER];
    bool live[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const uint64_t s = base + uint64_t(q) * 32u + uint32_t(lane);
      live[q] = s < S;
      dst[q] = src[q] = 0;
      nb[q] = last[q] = 0;
      hd[q] = 0;
      off[q] = 0;
      if (live[q]) {
        const SegRec r = seg[s];
        const uint8_t cyc = oncycle[s];
        const unsigned long long v = X[s];
        // (a pointer short of a head is flagged by k_chain_len)
        live[q] = r.len != 0 && !cyc && ptr_of(v) >= nx && ptr_of(v) < S;
        if (live[q]) {
          hd[q] = ptr_of(v) - nx;
          off[q] = pk_o(v);
          src[q] = r.off_job & SEG_OFF_MASK;
          nb[q] = seg_w(uint32_t(s), r.len, nx, k);
          last[q] = r.next == NONE;
        }
      }
    }
    // (segments of lines the walk wrote copy nothing)
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      if (!live[q]) continue;
      const unsigned long long lb = lbase[hd[q]];
      if (lb == LINE_WALKED) {
        nb[q] = 0;
        last[q] = 0;
      } else {
        dst[q] = lb + off[q];
      }
    }
    // groups of 8 lanes: group g copies, one after another, the segments
    // resolved by its own 8 lanes.  Each lane of the group stores aligned
    // 4-byte words of the destination, funnel-shifted from the two aligned
    // source words that hold them; the up to 3 bytes before the first
    // aligned word and after the last one go byte by byte.  Source words
    // are read only where they hold a byte of the segment, so they stay in
    // the segment chars' allocation.
    const uint32_t gl = uint32_t(lane) & 7u;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
#pragma unroll 1
      for (int i = 0; i < 8; ++i) {
        const uint64_t d = __shfl_sync(0xFFFFFFFFu, dst[q], i, 8);
        const uint64_t c = __shfl_sync(0xFFFFFFFFu, src[q], i, 8);
        const uint32_t m = __shfl_sync(0xFFFFFFFFu, nb[q], i, 8);
        const uint32_t e = __shfl_sync(0xFFFFFFFFu, last[q], i, 8);
        // bytes before the first aligned word of the destination (the output
        // buffer itself may start at any byte)
        const uint32_t hb = min((4u - uint32_t(reinterpret_cast<uintptr_t>(out + d) & 3u)) & 3u, m);
        const uint32_t nbody = (m - hb) >> 2;
        const uint32_t tb = (m - hb) & 3u;
        const char* sp = segchars + c + hb;
        char* dp = out + d + hb;
        const uint32_t sh = 8u * uint32_t(reinterpret_cast<uintptr_t>(sp) & 3u);
        const uint32_t* sw = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(sp) & ~uintptr_t(3));
        for (uint32_t wi = gl; wi < nbody; wi += 8) {
          const uint32_t w0 = sw[wi];
          const uint32_t v = sh ? __funnelshift_r(w0, sw[wi + 1], sh) : w0;
          reinterpret_cast<uint32_t*>(dp)[wi] = v;
        }
        if (gl < hb) out[d + gl] = segchars[c + gl];
        if (gl >= 4 && gl - 4 < tb) dp[4 * nbody + (gl - 4)] = sp[4 * nbody + (gl - 4)];
        if (gl == 7 && e) out[d + m] = '\n';
      }
    }
  }
}

__global__ void k_mark_cycle(const uint32_t* __restrict__ act, const uint32_t* act_count,
                             uint8_t* __restrict__ oncycle) {
  const uint32_t na = *act_count;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < na; j += gridDim.x * blockDim.x)
    oncycle[act[j]] = 1;
}

// Cycles of segments (rare; they hold only segments that start at S-only
// copies): one thread spells each cycle starting at its smallest k-mer.  The
// cycle's distinct k-mers are the last chars of each segment after its first
// k-mer, read circularly.
template <int NW>
__global__ void k_seg_cycles(Counters* ctr, uint32_t S, const uint32_t* __restrict__ act, uint32_t na,
                             uint8_t* __restrict__ oncycle, const SegRec* __restrict__ seg,
                             const JobTab* __restrict__ jobs, unsigned long long* __restrict__ jout,
                             const char* __restrict__ segchars, char* __restrict__ out, int k) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (uint32_t j = 0; j < na; ++j) {
    const uint32_t s0 = act[j];
    if (oncycle[s0] != 1) continue;
    // total distinct k-mers N and the circular char accessor
    uint64_t N = 0;
    uint32_t s = s0, steps = 0;
    do {
      N += seg[s].len - 1u;
      oncycle[s] = 2;
      s = seg[s].next;
    } while (s != s0 && s < S && ++steps <= S);
    if (s != s0 || N == 0) {
      atomicOr(&ctr->err, ERR_INTERNAL);
      continue;
    }
    // char q of the circular string: segment chars after the first k
    // (q < N and the cycle was walked above, so the loop ends within it)
    auto at = [&](uint64_t q) -> char {
      uint32_t t = s0;
      for (uint32_t guard = 0; guard <= S; ++guard) {
        const SegRec r = seg[t];
        const uint64_t m = r.len - 1u;
        if (q < m) return segchars[(r.off_job & SEG_OFF_MASK) + q];
        q -= m;
        t = r.next;
      }
      return 'A';
    };
    // the k-mer ending at circular position q; find the smallest
    auto kmer_at = [&](uint64_t q) {
      Key<NW> x;
#pragma unroll
      for (int w = 0; w < NW; ++w) x.w[w] = 0;
      for (int c = 0; c < k; ++c) {
        const char ch = at((q + N * 64 - (k - 1) + c) % N);
        const uint64_t code = (ch == 'C') ? 1 : (ch == 'G') ? 2 : (ch == 'T') ? 3 : 0;
        if (c < 32) x.w[0] |= code << (2 * c);
        else if (NW == 2) x.w[NW - 1] |= code << (2 * (c - 32));
      }
      return x;
    };
    uint64_t best = 0;
    Key<NW> bk = kmer_at(0);
    for (uint64_t q = 1; q < N; ++q) {
      const Key<NW> x = kmer_at(q);
      if (key_lt(x, bk)) { bk = x; best = q; }
    }
    const uint64_t len = uint64_t(k) + N;  // k + (N - 1) chars + '\n'
    const uint32_t job = uint32_t(seg[s0].off_job >> SEG_OFF_BITS);
    const unsigned long long o = atomicAdd(jout + job, len);
    if (o + len > jobs[job].ocap) {
      atomicOr(&ctr->err, ERR_CAPACITY);
      return;
    }
    char* dst = out + jobs[job].obase + o;
    for (uint64_t t = 0; t + 1 < len; ++t) dst[t] = at((best + N * 64 - (k - 1) + t) % N);
    dst[len - 1] = '\n';
    atomicAdd(&ctr->cycles, 1ull);
  }
}

// ===================================================== HEC contraction
//
// Heavy-edge coarsening over a set of paths (and rare cycles), restating the
// reference's round loop (coarsen_de_bruijn_full_cycle, coarseners.h:437-485):
// every node with a predecessor wants to merge with it, a head wants its
// successor, an isolated node is a finished chain (coarsen_HEC,
// heuristics.h:224-245); two compare-and-swaps pair a node with its choice or
// let it join the choice's aggregate (parallel_map_construct,
// heuristics.h:106-203, with bounded retries and a singleton fallback instead
// of unbounded spins); aggregates become the next level's nodes
// (coarsen_de_bruijn_graph, coarseners.h:68-92).  Members are ordered by
// walking from the aggregate's first member (instead of the O(m^2) sort of
// transpose_and_sort, coarseners.h:182-235) and their offsets are composed
// top-down (instead of copying member lists, compact_graph.h:55-112).
// Levels live in one node pool; level r occupies [lb[r], lb[r] + ln[r]).
// Kernels read the level sizes on the device, so every round is enqueued
// without host round trips.
constexpr uint32_t HV_UNSET = 0xFFFFFFFFu, HV_LOCK = 0xFFFFFFFEu, HV_FIN = 0xFFFFFFFDu, HV_CYC = 0xFFFFFFFCu;
constexpr uint32_t HP_SENT = 0xFFFFFFFBu;  // coarse node not yet given a first member

struct HecPool {
  uint32_t *prv, *nxt, *wt, *hn, *vc, *agg, *loc, *first0;
  uint32_t* lb;  // [R+1] level base
  uint32_t* ln;  // [R+1] level size
  uint32_t cap;
  Counters* ctr;
};

__global__ void k_hec_level0(HecPool h, const uint32_t* __restrict__ prev, const uint32_t* __restrict__ next,
                             const uint32_t* __restrict__ w, uint64_t n, const Counters* nctr) {
  const uint64_t N = nctr ? uint64_t(nctr->seg_count) : n;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    h.lb[0] = 0;
    h.ln[0] = uint32_t(N);
  }
  for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < N; u += uint64_t(gridDim.x) * blockDim.x) {
    h.prv[u] = prev[u];
    h.nxt[u] = next[u];
    h.wt[u] = w ? w[u] : 1u;
    h.first0[u] = uint32_t(u);
  }
}

// Level 0 from the fused path's segments: next from the records, prev from
// the ranking's first state built from them (k_seg_xinit; ids [0, nx) only:
// a line's first segment has none), weights from the lengths.  Unused head-pool ids have
// length 0 and stay isolated.
__global__ void k_hec_level0_seg(HecPool h, const SegRec* __restrict__ seg, const unsigned long long* __restrict__ X0,
                                 uint64_t S, uint32_t nx, int k) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    h.lb[0] = 0;
    h.ln[0] = uint32_t(S);
  }
  for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < S; u += uint64_t(gridDim.x) * blockDim.x) {
    const SegRec r = seg[u];
    uint32_t pv = NONE, nx_ = NONE, w = 0;
    if (r.len) {
      pv = (u < nx) ? ptr_of(X0[u]) : NONE;
      nx_ = r.next;
      w = seg_w(uint32_t(u), r.len, nx, k);
    }
    h.prv[u] = pv;
    h.nxt[u] = nx_;
    h.wt[u] = w;
    h.first0[u] = uint32_t(u);
  }
}

// choice (hn) per node; isolated nodes are finished chains; a node whose
// predecessor is still the sentinel is a whole cycle collapsed into one
__global__ void k_hec_prep(HecPool h, int r) {
  const uint32_t b = h.lb[r], N = h.ln[r];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const uint32_t u = b + j;
    const uint32_t pv = h.prv[u], nx = h.nxt[u];
    if (pv == HP_SENT) {
      h.hn[u] = NONE;
      h.vc[u] = HV_CYC;
    } else if (pv == u) {  // a one-node cycle
      h.hn[u] = NONE;
      h.vc[u] = HV_CYC;
    } else {
      const uint32_t c = (pv != NONE) ? pv : nx;
      h.hn[u] = c;
      h.vc[u] = (c == NONE) ? HV_FIN : HV_UNSET;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    h.lb[r + 1] = b + N;
    h.ln[r + 1] = 0;
  }
}

// One pass of the two-CAS pairing.  A label is the pool index of the
// aggregate's root.  Pass 1 gives up after 10 tries when u > v (the
// reference's deadlock break, heuristics.h:142-146); pass 2 retries the rest
// a bounded number of times and then leaves u a singleton aggregate.
__global__ void k_hec_match(HecPool h, int r, int pass) {
  const uint32_t b = h.lb[r], N = h.ln[r];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const uint32_t u = b + j;
    const uint32_t v = h.hn[u];
    if (v == NONE) continue;
    if (pass == 2 && atomicAdd(h.vc + u, 0u) != HV_UNSET) continue;
    bool done = false;
    const int limit = (pass == 1) ? 64 : 256;
    for (int it = 0; it < limit && !done; ++it) {
      if (atomicCAS(h.vc + u, HV_UNSET, HV_LOCK) == HV_UNSET) {
        if (atomicCAS(h.vc + v, HV_UNSET, HV_LOCK) == HV_UNSET) {
          atomicExch(h.vc + v, u);
          atomicExch(h.vc + u, u);
          done = true;
        } else {
          const uint32_t lv = atomicAdd(h.vc + v, 0u);
          if (lv < HV_CYC) {  // v already labelled: join its aggregate
            atomicExch(h.vc + u, lv);
            done = true;
          } else {
            atomicExch(h.vc + u, HV_UNSET);  // release and retry
          }
        }
      } else {
        done = true;  // u is labelled (or being labelled) by a neighbour
      }
      if (pass == 1 && it > 10 && u > v) break;
    }
    if (pass == 2 && !done) atomicCAS(h.vc + u, HV_UNSET, u);  // singleton
  }
}

// Roots (label == self) take the next level's pool slots; the root's hn
// holds its new index afterwards.
__global__ void k_hec_roots(HecPool h, int r) {
  const uint32_t b = h.lb[r], N = h.ln[r];
  const uint32_t nb = h.lb[r + 1];
  const int lane = threadIdx.x & 31;
  for (uint32_t j0 = blockIdx.x * blockDim.x; j0 < N; j0 += gridDim.x * blockDim.x) {
    const uint32_t j = j0 + threadIdx.x;
    const uint32_t u = b + j;
    const bool root = (j < N) && (h.vc[u] == u);
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, root);
    uint32_t base = 0;
    if (m) {
      if (lane == __ffs(m) - 1) base = atomicAdd(h.ln + r + 1, uint32_t(__popc(m)));
      base = __shfl_sync(0xFFFFFFFFu, base, __ffs(m) - 1);
    }
    if (root) {
      const uint32_t a = nb + base + __popc(m & ((1u << lane) - 1u));
      if (a >= h.cap) {
        atomicOr(&h.ctr->err, ERR_CAPACITY);
      } else {
        h.hn[u] = a;
        h.prv[a] = HP_SENT;
        h.nxt[a] = NONE;
        h.wt[a] = 0;
        h.first0[a] = NONE;
      }
    }
  }
}

__global__ void k_hec_assign(HecPool h, int r) {
  const uint32_t b = h.lb[r], N = h.ln[r];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const uint32_t u = b + j;
    const uint32_t c = h.vc[u];
    h.agg[u] = (c < HV_CYC) ? h.hn[c] : NONE;
  }
}

// The first member of each aggregate (predecessor outside it) walks its
// members along next: local offsets, total weight, coarse neighbours.
__global__ void k_hec_order(HecPool h, int r) {
  const uint32_t b = h.lb[r], N = h.ln[r];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const uint32_t u = b + j;
    const uint32_t A = h.agg[u];
    if (A == NONE || A >= h.cap) continue;
    const uint32_t pv = h.prv[u];
    if (pv != NONE && h.agg[pv] == A) continue;  // not the first member
    uint32_t off = 0, m = u, last = u;
    for (uint32_t guard = 0; guard < N; ++guard) {
      h.loc[m] = off;
      off += h.wt[m];
      last = m;
      const uint32_t nx = h.nxt[m];
      if (nx == NONE || h.agg[nx] != A) break;
      m = nx;
    }
    h.wt[A] = off;
    h.first0[A] = h.first0[u];
    h.nxt[A] = (h.nxt[last] == NONE) ? NONE : h.agg[h.nxt[last]];
    h.prv[A] = (pv == NONE) ? NONE : h.agg[pv];
  }
}

// Top-down: (head, offset) of every node from its aggregate's, stored in
// (hn, loc).  A finished node is a whole chain headed by its first member; a
// cycle node marks its members with head NONE.
__global__ void k_hec_down(HecPool h, int r) {
  const uint32_t b = h.lb[r], N = h.ln[r];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const uint32_t u = b + j;
    const uint32_t c = h.vc[u];
    uint32_t hd, of;
    if (c == HV_FIN) {
      hd = h.first0[u];
      of = 0;
    } else if (c == HV_CYC) {
      hd = NONE;
      of = 0;
    } else {
      const uint32_t A = h.agg[u];
      hd = (A == NONE || A >= h.cap) ? NONE : h.hn[A];
      of = (hd == NONE) ? 0 : h.loc[A] + h.loc[u];
    }
    h.hn[u] = hd;
    h.loc[u] = of;
  }
}

// Level-0 results into the (pointer | HEAD_BIT, offset) form of the ranking.
__global__ void k_hec_emit(HecPool h, unsigned long long* __restrict__ X, uint8_t* __restrict__ oncycle) {
  const uint32_t N = h.ln[0];
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const uint32_t hd = h.hn[s];
    if (hd == NONE) {
      X[s] = pk(s, 0);
      if (oncycle) oncycle[s] = 1;
    } else {
      X[s] = pk(hd == s ? (hd | HEAD_BIT) : hd, h.loc[s]);
    }
  }
}

__global__ void k_cycle_list(const uint8_t* __restrict__ oncycle, uint64_t n, const Counters* nctr,
                             uint32_t* __restrict__ act, uint32_t* __restrict__ cnt) {
  const uint64_t N = nctr ? uint64_t(nctr->seg_count) : n;
  for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < N; s += uint64_t(gridDim.x) * blockDim.x)
    if (oncycle[s]) act[atomicAdd(cnt, 1u)] = uint32_t(s);
}

__global__ void k_hec_check(HecPool h, int R) {
  if (h.ln[R] != 0) atomicOr(&h.ctr->err, ERR_TIMEOUT);
}

// ======================================================= phase-API helpers

__global__ void k_head_rank(const unsigned long long* __restrict__ X, uint64_t n,
                            uint32_t* __restrict__ head, uint32_t* __restrict__ rank) {
  for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += uint64_t(gridDim.x) * blockDim.x) {
    const unsigned long long x = X[v];
    head[v] = ptr_of(x);
    rank[v] = pk_o(x);
  }
}

// Cycle vertices of the global graph (rare): one thread ranks each cycle from
// its smallest key.
template <int NW>
__global__ void k_vertex_cycles(const uint32_t* __restrict__ act, uint32_t na,
                                const uint32_t* __restrict__ succ, const uint64_t* __restrict__ keys,
                                uint64_t n_all, uint32_t* __restrict__ head, uint32_t* __restrict__ rank,
                                uint8_t* __restrict__ seen, unsigned long long* ncyc) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (uint32_t j = 0; j < na; ++j) {
    const uint32_t v0 = act[j];
    if (seen[v0]) continue;
    uint32_t best = v0;
    Key<NW> bk = ld_key<NW>(keys, v0);
    uint64_t steps = 0;
    uint32_t x = succ[v0];
    for (; x != v0 && x != NONE && steps < n_all; x = succ[x], ++steps) {
      const Key<NW> xk = ld_key<NW>(keys, x);
      if (key_lt(xk, bk)) { bk = xk; best = x; }
    }
    if (x != v0) continue;  // not a cycle: left as ranked
    uint32_t r = 0;
    x = best;
    steps = 0;
    do {
      head[x] = best;
      rank[x] = r++;
      seen[x] = 1;
      x = succ[x];
    } while (x != best && x != NONE && ++steps < n_all);
    ++*ncyc;
  }
}

__global__ void k_count_members(const uint32_t* __restrict__ head, uint64_t n, uint32_t* __restrict__ cnt) {
  for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += uint64_t(gridDim.x) * blockDim.x)
    atomicAdd(cnt + head[v], 1u);
}

__global__ void k_line_len(const uint32_t* __restrict__ head, const uint32_t* __restrict__ cnt,
                           uint64_t n, int k, uint32_t* __restrict__ len) {
  for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += uint64_t(gridDim.x) * blockDim.x)
    len[v] = (head[v] == uint32_t(v)) ? uint32_t(k) + cnt[v] : 0u;
}

// Spell each vertex's chars at its line offset (write_intra_bucket_outputs,
// compact.h:187-208): rank 0 writes the whole k-mer, rank r writes its last
// char at k-1+r, the last member adds '\n'.
template <int NW>
__global__ void k_spell(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ head,
                        const uint32_t* __restrict__ rank, const uint32_t* __restrict__ cnt,
                        const unsigned long long* __restrict__ loff, uint64_t n, int k,
                        char* __restrict__ out) {
  for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
       v += uint64_t(gridDim.x) * blockDim.x) {
    const Key<NW> x = ld_key<NW>(keys, v);
    const uint32_t h = head[v], r = rank[v];
    char* dst = out + loff[h];
    if (r == 0) {
      spell_key<NW>(dst, x, k);
    } else {
      dst[k - 1 + r] = acgt(key_char(x, k - 1));
    }
    if (r + 1 == cnt[h]) dst[k + r] = '\n';
  }
}

// =========================================================== host pipeline

static int grid_for(const Env& e, uint64_t work, int block) {
  const uint64_t want = (work + block - 1) / block;
  const uint64_t cap = uint64_t(e.sm_count) * 16;
  return int(std::max<uint64_t>(1, std::min(want, cap)));
}

#define UC_CK(call)                                                                                  \
  do {                                                                                               \
    cudaError_t _e = (call);                                                                         \
    if (_e != cudaSuccess) return e.fail(UC_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

int Env::fail(int code, const std::string& msg) {
  err = msg;
  return code;
}

cudaError_t Env::dev_malloc(void** p, size_t bytes) {
  if (faults.fail_alloc_after && --faults.fail_alloc_after == 0) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

void* Env::take(int w, size_t bytes) {
  Arena& a = ar[w];
  const size_t o = (a.used + 255) & ~size_t(255);
  if (o + bytes > a.cap) return nullptr;
  a.used = o + bytes;
  return a.base + o;
}

int Env::reserve(int w, size_t bytes) {
  Arena& a = ar[w];
  bytes += size_t(16) << 20;
  if (bytes <= a.cap) return UC_OK;
  if (pool)
    return fail(UC_EBUDGET, "job needs " + std::to_string(bytes >> 20) + " MiB in arena " + std::to_string(w) +
                                ", its pool slice holds " + std::to_string(a.cap >> 20) + " MiB");
  if (a.used) return fail(UC_EINTERNAL, "arena grown while in use");
  const size_t other = ar[1 - w].cap;
  if (bytes + other > budget)
    return fail(UC_EBUDGET, "job needs " + std::to_string((bytes + other) >> 20) + " MiB of scratch, budget " +
                                std::to_string(budget >> 20) + " MiB");
  if (a.base) {
    cudaStreamSynchronize(stream);
    cudaFree(a.base);
    a.base = nullptr;
    a.cap = 0;
  }
  if (dev_malloc(reinterpret_cast<void**>(&a.base), bytes) != cudaSuccess) {
    cudaGetLastError();
    a.base = nullptr;
    return fail(UC_ENOMEM, "cudaMalloc of " + std::to_string(bytes >> 20) + " MiB failed");
  }
  a.cap = bytes;
  return UC_OK;
}

int Env::check_err(const Counters* h) {
  const uint32_t f = h->err;
  if (!f) return UC_OK;
  if (f & ERR_LINE) return fail(UC_EINPUT, "a k-mer line is shorter than k");
  if (f & ERR_COUNT) return fail(UC_EINPUT, "header count differs from the number of lines");
  if (f & ERR_TIMEOUT) return fail(UC_ETIMEOUT, "a bounded device wait ran out");
  if (f & ERR_CAPACITY) return fail(UC_EINTERNAL, "an output bound was exceeded");
  return fail(UC_EINTERNAL, "internal invariant failed (flags " + std::to_string(f) + ")");
}

int Env::read_ctr() {
  Env& e = *this;
  UC_CK(cudaMemcpyAsync(h_ctr, ctr, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
  UC_CK(cudaStreamSynchronize(stream));
  return UC_OK;
}

// Parse the count line: reads the first bytes back to the host.
int parse_header(Env& e, const char* d_text, size_t bytes, uint64_t& n, uint64_t& body) {
  std::vector<char> h;
  size_t want = std::min<size_t>(bytes, 256);
  for (;;) {
    h.resize(want);
    if (want) UC_CK(cudaMemcpyAsync(h.data(), d_text, want, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    size_t p = 0;
    while (p < want && (h[p] == ' ' || h[p] == '\t' || h[p] == '\r')) ++p;
    if (p >= want || h[p] < '0' || h[p] > '9') {
      if (want < bytes && p >= want) {
        want = std::min(bytes, want * 4);
        continue;
      }
      return e.fail(UC_EINPUT, "missing k-mer count header");
    }
    uint64_t v = 0;
    while (p < want && h[p] >= '0' && h[p] <= '9') {
      v = v * 10 + uint64_t(h[p] - '0');
      if (v > 0xFFFFFFFEull) return e.fail(UC_EINPUT, "k-mer count too large");
      ++p;
    }
    while (p < want && h[p] != '\n') ++p;
    if (p >= want && want < bytes) {
      want = std::min(bytes, want * 4);
      continue;
    }
    n = v;
    body = (p < want) ? p + 1 : want;
    return UC_OK;
  }
}

// End of the k-mer lines: trailing '\n' / '\r' bytes are not a line.
static int text_end(Env& e, const char* d_text, size_t bytes, uint64_t body, uint64_t& end) {
  end = bytes;
  char tail[256];
  while (end > body) {
    const size_t take = std::min<uint64_t>(256, end - body);
    UC_CK(cudaMemcpyAsync(tail, d_text + end - take, take, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    size_t j = take;
    while (j > 0 && (tail[j - 1] == '\n' || tail[j - 1] == '\r')) --j;
    end -= (take - j);
    if (j > 0) break;
  }
  return UC_OK;
}

static size_t line_index_bytes(size_t bytes, uint64_t n) {
  const uint64_t nchunks = bytes / (1 << 16) + 2;
  return nchunks * 4 + (nchunks + 1) * 8 + scan_tmp_elems(nchunks) * 8 + (n + 1) * 8 + 8 * 256;
}

struct FuseArgs {
  int l = 0;
  uint64_t seed = 0;
  uint32_t jb = 0;
  uint32_t *b1 = nullptr, *b2 = nullptr, *jcross = nullptr;
  uint32_t* counts = nullptr;  // group counts (cshift), or 16-bit counts two per word (CNT16)
  uint32_t cshift = CNT16;
  uint64_t cbytes = 0;         // bytes of counts to clear before a second pack
  uint64_t M = 0;
};

template <int NW, bool FUSE, bool MULTI, int KC = 0, int LC = 0>
static int pack_occupancy() {
  static int o = 0;  // resident CTAs per SM (per template instance)
  if (!o) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_pack<NW, FUSE, MULTI, KC, LC>, 256, 0);
    if (o < 1) o = 1;
  }
  return o;
}

// The single-job fused pack with k and l fixed at compile time: k = 31 or
// 63 with l in [8, 16] (the bucket count raises l to at least 13 for large
// jobs).  Returns false for other shapes.
template <int NW, int KC, int LC>
static bool launch_pack_fixed_l(Env& e, const JobTab* jobs, const JobTab& J, uint64_t nblocks, uint64_t* keys,
                                const FuseArgs* fz) {
  const int o = pack_occupancy<NW, true, false, KC, LC>();
  const int grid = int(std::max<uint64_t>(1, std::min<uint64_t>(nblocks, uint64_t(e.sm_count) * o)));
  ++e.launches;
  k_pack<NW, true, false, KC, LC><<<grid, 256, 0, e.stream>>>(jobs, J, 1, nblocks, nullptr, KC, keys, &e.ctr->err,
                                                               LC, fz->seed, fz->jb, fz->b1, fz->b2, fz->counts,
                                                               fz->cshift, fz->jcross);
  return true;
}

template <int NW, int KC>
static bool launch_pack_fixed(Env& e, const JobTab* jobs, const JobTab& J, uint64_t nblocks, uint64_t* keys,
                              const FuseArgs* fz) {
  switch (fz->l) {
    case 8: return launch_pack_fixed_l<NW, KC, 8>(e, jobs, J, nblocks, keys, fz);
    case 9: return launch_pack_fixed_l<NW, KC, 9>(e, jobs, J, nblocks, keys, fz);
    case 10: return launch_pack_fixed_l<NW, KC, 10>(e, jobs, J, nblocks, keys, fz);
    case 11: return launch_pack_fixed_l<NW, KC, 11>(e, jobs, J, nblocks, keys, fz);
    case 12: return launch_pack_fixed_l<NW, KC, 12>(e, jobs, J, nblocks, keys, fz);
    case 13: return launch_pack_fixed_l<NW, KC, 13>(e, jobs, J, nblocks, keys, fz);
    case 14: return launch_pack_fixed_l<NW, KC, 14>(e, jobs, J, nblocks, keys, fz);
    case 15: return launch_pack_fixed_l<NW, KC, 15>(e, jobs, J, nblocks, keys, fz);
    case 16: return launch_pack_fixed_l<NW, KC, 16>(e, jobs, J, nblocks, keys, fz);
    default: return false;
  }
}

// one: the job of a single-job launch (host copy), or NULL for a batch
// whose jobs the kernel finds in the table.
template <int NW>
static void launch_pack(Env& e, const JobTab* jobs, const JobTab* one, uint32_t njobs, uint64_t nblocks,
                        const unsigned long long* starts, int k, uint64_t* keys, const FuseArgs* fz) {
  // one wave of resident CTAs: blocks stride over equal-sized line blocks,
  // so a partial second wave would double the time
  const int o = fz ? (one ? pack_occupancy<NW, true, false>() : pack_occupancy<NW, true, true>())
                   : (one ? pack_occupancy<NW, false, false>() : pack_occupancy<NW, false, true>());
  const int grid = int(std::max<uint64_t>(1, std::min<uint64_t>(nblocks, uint64_t(e.sm_count) * o)));
  const JobTab J = one ? *one : JobTab{};
  if (fz && one && !starts) {
    if (NW == 1 && k == 31 && launch_pack_fixed<NW, 31>(e, jobs, J, nblocks, keys, fz)) return;
    if (NW == 2 && k == 63 && launch_pack_fixed<NW, 63>(e, jobs, J, nblocks, keys, fz)) return;
  }
  ++e.launches;
  if (fz && one)
    k_pack<NW, true, false><<<grid, 256, 0, e.stream>>>(jobs, J, njobs, nblocks, starts, k, keys, &e.ctr->err,
                                                        fz->l, fz->seed, fz->jb, fz->b1, fz->b2, fz->counts,
                                                        fz->cshift, fz->jcross);
  else if (fz)
    k_pack<NW, true, true><<<grid, 256, 0, e.stream>>>(jobs, J, njobs, nblocks, starts, k, keys, &e.ctr->err,
                                                       fz->l, fz->seed, fz->jb, fz->b1, fz->b2, fz->counts,
                                                       fz->cshift, fz->jcross);
  else if (one)
    k_pack<NW, false, false><<<grid, 256, 0, e.stream>>>(jobs, J, njobs, nblocks, starts, k, keys, &e.ctr->err, 0,
                                                         0, 0, nullptr, nullptr, nullptr, CNT16, nullptr);
  else
    k_pack<NW, false, true><<<grid, 256, 0, e.stream>>>(jobs, J, njobs, nblocks, starts, k, keys, &e.ctr->err, 0,
                                                        0, 0, nullptr, nullptr, nullptr, CNT16, nullptr);
}

// Grow-only device buffers for the job table and the per-job counters.
static int job_buffers(Env& e, uint32_t njobs) {
  const size_t want = size_t(njobs) * (sizeof(JobTab) + 4 * 8) + 1024;
  if (want <= e.jcap) return UC_OK;
  if (e.jbuf) {
    cudaStreamSynchronize(e.stream);
    cudaFree(e.jbuf);
  }
  e.jbuf = nullptr;
  e.jcap = 0;
  if (e.dev_malloc(reinterpret_cast<void**>(&e.jbuf), want) != cudaSuccess) {
    cudaGetLastError();
    e.jbuf = nullptr;
    return e.fail(UC_ENOMEM, "job table");
  }
  e.jcap = want;
  return UC_OK;
}
struct JobDev {
  JobTab* tab;
  uint32_t* jcross;
  uint32_t* jseg;
  unsigned long long* jout;
  unsigned long long* jclosed;
};
static JobDev job_dev(Env& e, uint32_t njobs) {
  JobDev d;
  d.tab = reinterpret_cast<JobTab*>(e.jbuf);
  char* q = e.jbuf + ((size_t(njobs) * sizeof(JobTab) + 255) & ~size_t(255));
  d.jout = reinterpret_cast<unsigned long long*>(q);
  d.jclosed = d.jout + njobs;
  d.jcross = reinterpret_cast<uint32_t*>(d.jclosed + njobs);
  d.jseg = d.jcross + njobs;
  return d;
}

// Text -> keys for one job (and, with fz, buckets + counts).  Fixed-width
// lines are packed directly; any other layout indexes the line starts first
// (back arena, which must be empty).
static int pack_single(Env& e, const char* d_text, size_t bytes, int k, uint64_t* d_keys, const FuseArgs* fz,
                       JobTab& J, JobTab* jdev) {
  const uint8_t* text = reinterpret_cast<const uint8_t*>(d_text);
  const uint64_t n = J.n, body = J.body, end = J.end;
  UC_CK(cudaMemsetAsync(&e.ctr->err, 0, 4, e.stream));
  if (n == 0) {
    if (end > body) return e.fail(UC_EINPUT, "header count differs from the number of lines");
    return UC_OK;
  }
  const int nw = (k <= 31) ? 1 : 2;
  const uint64_t nblocks = (n + PACK_LINES - 1) / PACK_LINES;
  bool fixed = J.fixed != 0;
  int st;
  if (fixed) {
    if (nw == 1) launch_pack<1>(e, jdev, &J, 1, nblocks, nullptr, k, d_keys, fz);
    else launch_pack<2>(e, jdev, &J, 1, nblocks, nullptr, k, d_keys, fz);
    UC_CK(cudaGetLastError());
    st = e.read_ctr();
    if (st) return st;
    if (e.h_ctr->err & ERR_LAYOUT) {
      fixed = false;
      UC_CK(cudaMemsetAsync(&e.ctr->err, 0, 4, e.stream));
      if (fz) {
        UC_CK(cudaMemsetAsync(fz->counts, 0, fz->cbytes, e.stream));
        UC_CK(cudaMemsetAsync(fz->jcross, 0, 4, e.stream));
      }
    } else if (e.h_ctr->err) {
      return e.check_err(e.h_ctr);
    }
  }
  if (!fixed) {
    const uint32_t chunk = 1 << 16;
    const uint64_t nchunks = std::max<uint64_t>(1, (end - body + chunk - 1) / chunk);
    st = e.reserve(1, line_index_bytes(bytes, n));
    if (st) return st;
    uint32_t* cnt = static_cast<uint32_t*>(e.take(1, nchunks * 4));
    unsigned long long* off = static_cast<unsigned long long*>(e.take(1, (nchunks + 1) * 8));
    unsigned long long* tmp = static_cast<unsigned long long*>(e.take(1, scan_tmp_elems(nchunks) * 8));
    unsigned long long* starts = static_cast<unsigned long long*>(e.take(1, (n + 1) * 8));
    if (!cnt || !off || !tmp || !starts) return e.fail(UC_EBUDGET, "scratch for the line index");
    ++e.launches;
    k_count_nl<<<unsigned(nchunks), 256, 0, e.stream>>>(text, body, end, cnt, chunk);
    e.launches += 2 * 3;
    scan_excl<uint32_t, unsigned long long>(cnt, nchunks, off, tmp, e.stream);
    unsigned long long lines_m1 = 0;
    UC_CK(cudaMemcpyAsync(&lines_m1, off + nchunks, 8, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    if (lines_m1 + 1 != n) return e.fail(UC_EINPUT, "header count differs from the number of lines");
    ++e.launches;
    k_write_starts<<<unsigned(nchunks), 256, 0, e.stream>>>(text, body, end, off, chunk, starts, n);
    if (nw == 1) launch_pack<1>(e, jdev, &J, 1, nblocks, starts, k, d_keys, fz);
    else launch_pack<2>(e, jdev, &J, 1, nblocks, starts, k, d_keys, fz);
    UC_CK(cudaGetLastError());
    st = e.read_ctr();
    e.ar[1].used = 0;
    if (st) return st;
    if (e.h_ctr->err) return e.check_err(e.h_ctr);
  }
  return UC_OK;
}

// Host view of one job's text: count line, body offset, end, layout.
static int host_job(Env& e, const char* d_text, size_t bytes, int k, JobTab& J) {
  uint64_t n = 0, body = 0, end = 0;
  int st = parse_header(e, d_text, bytes, n, body);
  if (st) return st;
  st = text_end(e, d_text, bytes, body, end);
  if (st) return st;
  J = JobTab{};
  J.text = reinterpret_cast<const uint8_t*>(d_text);
  J.tbytes = bytes;
  J.n = n;
  J.body = body;
  J.end = end;
  const uint64_t stride = uint64_t(k) + 1;
  J.fixed = ((n == 0 && end == body) || (n > 0 && end - body == n * stride - 1)) ? 1u : 0u;
  return UC_OK;
}

int pack(Env& e, const char* d_text, size_t bytes, int k, uint64_t* d_keys, uint64_t& n_out) {
  if (k < 2 || k > 63) return e.fail(UC_EINPUT, "k must be in [2, 63]");
  e.reset();
  JobTab J;
  int r = host_job(e, d_text, bytes, k, J);
  if (r) return r;
  n_out = J.n;
  r = job_buffers(e, 1);
  if (r) return r;
  JobDev jd = job_dev(e, 1);
  UC_CK(cudaMemcpyAsync(jd.tab, &J, sizeof(JobTab), cudaMemcpyHostToDevice, e.stream));
  r = pack_single(e, d_text, bytes, k, d_keys, nullptr, J, jd.tab);
  e.reset();
  return r;
}

int minimizers(Env& e, const uint64_t* d_keys, uint64_t n, int k, int l, uint64_t seed,
               const uint32_t* d_table, uint32_t* l1, uint32_t* l2) {
  if (k < 2 || k > 63) return e.fail(UC_EINPUT, "k must be in [2, 63]");
  if (l < 1 || l > 16 || l > k - 1) return e.fail(UC_EINPUT, "l must be in [1, min(16, k-1)]");
  if (n == 0) return UC_OK;
  const int grid = grid_for(e, n, 256);
  ++e.launches;
  if (k <= 31) k_lmin<1><<<grid, 256, 0, e.stream>>>(d_keys, n, k, l, seed, d_table, l1, l2);
  else k_lmin<2><<<grid, 256, 0, e.stream>>>(d_keys, n, k, l, seed, d_table, l1, l2);
  UC_CK(cudaGetLastError());
  return UC_OK;
}

// Bucket plan.  A job's buckets are (job << jb) | local: the largest job
// sizes jb, and njobs << jb buckets in all (rounded up to a power of two,
// bits = log2 of that).
struct Plan {
  uint32_t bits, jb, cap, pack, tslots, wcap, wts, wbytes, lf;
  uint32_t cg;  // the pack's count groups: 2^cg buckets each
  int l_used;
  uint64_t M;
};

// Count groups of 2^bits buckets: at most 2^COUNT_GROUPS_BITS of them,
// from 2^24 buckets on (below that one 32-bit count per bucket, at most
// 32 MiB, stays in L2 and level 3 needs no counting pass).
static uint32_t count_group_bits(uint32_t bits) {
  return bits >= 24 ? bits - COUNT_GROUPS_BITS : 0u;
}
static uint64_t count_groups(uint64_t M) { return std::min<uint64_t>(M, 1ull << COUNT_GROUPS_BITS); }

static uint32_t ceil_log2(uint64_t x) {
  uint32_t b = 0;
  while ((1ull << b) < x) ++b;
  return b;
}

static Plan plan_buckets(const Env& e, uint64_t nmax, uint32_t njobs, int k, int l) {
  Plan P{};
  const int nw = (k <= 31) ? 1 : 2;
  uint32_t cap = e.tune.tile_capacity ? e.tune.tile_capacity : 4096;
  while (cap > 256 && tile_bytes(nw, cap, pow2_at_least(2ull * cap)) > size_t(e.smem_optin)) cap -= 256;
  // warp tiles: <= wcap copies, one warp each (1 disables the tier)
  uint32_t wcap = e.tune.warp_capacity ? e.tune.warp_capacity : 256;
  if (wcap > cap) wcap = cap;
  const bool warp_tier = wcap >= 32;
  const uint32_t pack_cap = warp_tier ? wcap : cap;  // tiles are packed for this capacity
  const uint32_t jbits_max = 25 - std::min<uint32_t>(25, ceil_log2(njobs));
  const uint64_t copies = nmax + nmax / 8 + 1;
  uint32_t jb = 0;
  if (e.tune.bucket_bits) {
    jb = e.tune.bucket_bits;
  } else {
    // about bucket_fill buckets per tile: small enough that tiles pack well,
    // large enough that each bucket gathers several l-mers
    const uint32_t fill = e.tune.bucket_fill ? e.tune.bucket_fill : 8;
    while ((copies >> jb) > std::max<uint32_t>(1, pack_cap / fill) && jb < 25) ++jb;
  }
  jb = std::min(jb, jbits_max);
  // enough l-mers that each bucket gathers several of them
  const int lmin = int((jb + 2 + 1) / 2);
  int lu = std::max(l, lmin);
  lu = std::min(lu, std::min(16, k - 1));
  const uint32_t lf = e.tune.load_factor_pct ? e.tune.load_factor_pct : 200;
  uint32_t ts = big_slots(cap, lf);
  while (ts > pow2_at_least(2ull * cap) && tile_bytes(nw, cap, ts) > size_t(e.smem_optin)) ts >>= 1;
  P.jb = jb;
  P.bits = ceil_log2(uint64_t(njobs) << jb);
  P.cap = cap;
  P.pack = pack_cap;
  P.tslots = ts;
  P.wcap = warp_tier ? wcap : 0;
  uint32_t wts = warp_tier ? big_slots(wcap, lf) : 0;
  // eight warp tiles share a CTA's shared memory
  while (warp_tier && wts > pow2_at_least(2ull * wcap) && 8 * tile_bytes(nw, wcap, wts) > size_t(e.smem_optin))
    wts >>= 1;
  P.wts = wts;
  P.lf = lf;
  P.wbytes = warp_tier ? uint32_t((tile_bytes(nw, wcap, P.wts) + 15) & ~size_t(15)) : 0;
  P.l_used = lu;
  P.M = 1ull << P.bits;
  P.cg = count_group_bits(P.bits);
  return P;
}

struct Front {
  uint64_t* keys;
  uint32_t *b1, *b2, *counts, *c16, *gcount;
  unsigned long long *boff, *cursor, *fcur, *tile_begin, *scan_tmp, *goff;
  uint32_t *flag, *fidx, *big_list, *wlist, *blist, *tile_job;
  unsigned long long* big_size;
};

static size_t front_bytes(uint64_t n, int nw, uint64_t M, bool own_keys) {
  size_t need = 0;
  auto add = [&](size_t b) { need += (b + 255) & ~size_t(255); };
  if (own_keys) add(n * 8 * nw);
  add(n * 4); add(n * 4); add(M * 4); add((M + 1) * 8); add(M * 8); add(M * 8); add((M + 2) * 8);
  add(scan_tmp_elems(M) * 8); add(M * 4); add((M + 1) * 4); add(M * 4); add(M * 8);
  add(M * 4); add(M * 4); add(M * 4);
  add((M + 1) / 2 * 4);
  add(count_groups(M) * 4); add((count_groups(M) + 1) * 8);
  return need;
}

static int take_front(Env& e, uint64_t n, int nw, uint64_t M, bool own_keys, Front& f) {
  f.keys = own_keys ? static_cast<uint64_t*>(e.take(0, n * 8 * nw)) : nullptr;
  f.b1 = static_cast<uint32_t*>(e.take(0, n * 4));
  f.b2 = static_cast<uint32_t*>(e.take(0, n * 4));
  f.counts = static_cast<uint32_t*>(e.take(0, M * 4));
  f.boff = static_cast<unsigned long long*>(e.take(0, (M + 1) * 8));
  f.cursor = static_cast<unsigned long long*>(e.take(0, M * 8));
  f.fcur = static_cast<unsigned long long*>(e.take(0, M * 8));
  f.tile_begin = static_cast<unsigned long long*>(e.take(0, (M + 2) * 8));
  f.scan_tmp = static_cast<unsigned long long*>(e.take(0, scan_tmp_elems(M) * 8));
  f.flag = static_cast<uint32_t*>(e.take(0, M * 4));
  f.fidx = static_cast<uint32_t*>(e.take(0, (M + 1) * 4));
  f.big_list = static_cast<uint32_t*>(e.take(0, M * 4));
  f.big_size = static_cast<unsigned long long*>(e.take(0, M * 8));
  f.wlist = static_cast<uint32_t*>(e.take(0, M * 4));
  f.blist = static_cast<uint32_t*>(e.take(0, M * 4));
  f.tile_job = static_cast<uint32_t*>(e.take(0, M * 4));
  f.c16 = static_cast<uint32_t*>(e.take(0, (M + 1) / 2 * 4));
  f.gcount = static_cast<uint32_t*>(e.take(0, count_groups(M) * 4));
  f.goff = static_cast<unsigned long long*>(e.take(0, (count_groups(M) + 1) * 8));
  if (!f.goff) return e.fail(UC_EBUDGET, "front arena overflow");
  return UC_OK;
}

// counts -> offsets (M entries: buckets or count groups); returns the total
// number of copies (host sync).
static int bucket_offsets(Env& e, const Front& f, const uint32_t* counts, uint64_t M, unsigned long long* offs,
                          uint64_t& copies) {
  e.launches += 6;
  scan_excl<uint32_t, unsigned long long>(counts, M, offs, f.scan_tmp, e.stream);
  unsigned long long tot = 0;
  UC_CK(cudaMemcpyAsync(&tot, offs + M, 8, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  copies = tot;
  return UC_OK;
}
static int bucket_offsets(Env& e, const Front& f, uint64_t M, uint64_t& copies) {
  return bucket_offsets(e, f, f.counts, M, f.boff, copies);
}

// Let a kernel take all the dynamic shared memory an SM offers a block.  The
// attribute is process-wide, so it is always set to the same maximum: a
// per-call size would let one host thread lower it under another thread's
// launch (concurrent contexts and server lanes).
template <class K>
static int allow_max_smem(Env& e, K kernel) {
  cudaFuncAttributes a{};
  UC_CK(cudaFuncGetAttributes(&a, kernel));
  UC_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             e.smem_optin - int(a.sharedSizeBytes)));
  return UC_OK;
}

// Level split of the scatter: 2^mcb coarse partitions of 2^fb buckets.
static void scatter_split(uint32_t bbits, uint32_t& mcb, uint32_t& fb) {
  mcb = std::min<uint32_t>(bbits, 8);
  fb = bbits - mcb;
}

static size_t scatter_stage_bytes(uint64_t copies, int nw) { return copies * (8ull * nw + 8ull); }

// tile plan + scatter of every k-mer into its bucket(s).  stage: staging
// records for level 1 (scatter_stage_bytes).
// Tiles from the bucket counts: next-fit runs of whole buckets.
static int plan_tiles(Env& e, const Front& f, const Plan& P) {
  const uint64_t M = P.M;
  const int gm = grid_for(e, M, 256);
  e.launches += 2 + 6;
  {
    // about 256 threads per SM; each run ends a tile, so runs stay long
    // where there are enough buckets
    const uint64_t want = (M + uint64_t(e.sm_count) * 256 - 1) / (uint64_t(e.sm_count) * 256);
    const uint32_t runlen = uint32_t(std::min<uint64_t>(512, std::max<uint64_t>(16, (want + 15) & ~uint64_t(15))));
    k_tile_flags<<<grid_for(e, (M + runlen - 1) / runlen, 256), 256, 0, e.stream>>>(f.counts, uint32_t(M), P.pack,
                                                                                     P.jb, runlen, f.flag);
  }
  scan_excl<uint32_t, uint32_t>(f.flag, M, f.fidx, reinterpret_cast<uint32_t*>(f.scan_tmp), e.stream);
  k_tile_write<<<gm, 256, 0, e.stream>>>(f.flag, f.fidx, f.boff, uint32_t(M), P.jb, f.tile_begin, f.tile_job, e.ctr);
  UC_CK(cudaGetLastError());
  return UC_OK;
}

// The three placement levels of the bucketed copies.  Level 1
// (k_scatter_coarse) writes region r1; then either level 2 (k_scatter_mid)
// writes r2 and level 3 (k_scatter_sub) writes back into r1, or, where a
// coarse partition is already small, level 3 writes r2 straight away.  Both
// regions hold scatter_stage_bytes(copies, nw); the final copies (pkeys,
// plink) are the key and link arrays of the region level 3 wrote.  Level 1
// may run over the k-mers in several launches (the streamed path's chunks):
// its cursors and the cross-index counter carry over.
struct Scatter {
  uint32_t mcb = 0, fb = 0, mc = 0, sb = 0, nsub = 0, cap3 = 0;
  // offsets of the pack's count groups (2^cg buckets each); level 3 writes
  // every bucket's count and offset to cout / bout (null: they are known)
  const unsigned long long* goff = nullptr;
  uint32_t cg = 0;
  uint32_t* cout = nullptr;
  unsigned long long* bout = nullptr;
  bool mid = false;
  int nw = 1;
  uint64_t copies = 0;
  uint64_t *k1 = nullptr, *k2 = nullptr;
  uint32_t *l1 = nullptr, *l2 = nullptr, *b1 = nullptr, *b2 = nullptr;
};

// cg > 0: the copies are counted per group of 2^cg buckets (offsets in
// f.goff) and level 3 writes f.counts and f.boff; cg = 0 with
// group_offsets false: f.boff holds every bucket's offset already.
static int scatter_begin(Env& e, const Front& f, const Plan& P, int nw, char* r1, char* r2, uint64_t copies,
                         Scatter& sc, uint32_t cg = 0, bool group_offsets = false) {
  const uint64_t M = P.M;
  sc.nw = nw;
  sc.copies = copies;
  sc.cg = cg;
  sc.goff = group_offsets ? f.goff : f.boff;
  sc.cout = group_offsets ? f.counts : nullptr;
  sc.bout = group_offsets ? f.boff : nullptr;
  auto region = [&](char* base, uint64_t*& key, uint32_t*& link, uint32_t*& bkt) {
    key = reinterpret_cast<uint64_t*>(base);
    link = reinterpret_cast<uint32_t*>(base + copies * 8ull * nw);
    bkt = link + copies;
  };
  region(r1, sc.k1, sc.l1, sc.b1);
  region(r2, sc.k2, sc.l2, sc.b2);
  scatter_split(P.bits, sc.mcb, sc.fb);
  sc.mc = 1u << sc.mcb;
  // level-3 staging holds cap3 records (two CTAs per SM); sub-partitions of
  // about half that many copies, at most 2^SUB_MAX_BITS buckets and at most
  // MID_MAX_BINS of them per coarse partition
  sc.cap3 = (nw == 1) ? 8192u : 4096u;
  const double avg = double(copies) / double(M);
  int sbi = avg > 0 ? int(std::lround(std::log2(0.5 * sc.cap3 / avg))) : SUB_MAX_BITS;
  sbi = std::min(sbi, SUB_MAX_BITS);
  sbi = std::min(sbi, int(sc.fb));
  sbi = std::max(sbi, int(sc.fb) - int(std::log2(double(MID_MAX_BINS))));
  sbi = std::max(sbi, int(cg));  // a sub-partition is whole count groups
  sbi = std::max(sbi, 0);
  if (sbi > SUB_MAX_BITS || sbi > int(sc.fb))
    return e.fail(UC_EINTERNAL, "bucket count beyond the three scatter levels");
  sc.sb = uint32_t(sbi);
  sc.mid = sc.sb < sc.fb;
  sc.nsub = uint32_t(M >> sc.sb);
  int r0 = allow_max_smem(e, k_scatter_coarse<1>);
  if (!r0) r0 = allow_max_smem(e, k_scatter_coarse<2>);
  if (!r0) r0 = allow_max_smem(e, k_scatter_mid<1>);
  if (!r0) r0 = allow_max_smem(e, k_scatter_mid<2>);
  if (!r0) r0 = allow_max_smem(e, k_scatter_sub<1>);
  if (!r0) r0 = allow_max_smem(e, k_scatter_sub<2>);
  if (r0) return r0;
  UC_CK(cudaMemsetAsync(&e.ctr->cross_count, 0, 4, e.stream));
  e.launches += 1;
  k_coarse_init<<<grid_for(e, sc.mc, 256), 256, 0, e.stream>>>(sc.goff, sc.fb - sc.cg, sc.mc, f.cursor);
  UC_CK(cudaGetLastError());
  return UC_OK;
}

static int scatter_l1(Env& e, const Front& f, const Scatter& sc, const uint64_t* keys, const uint32_t* b1,
                      const uint32_t* b2, uint64_t n, int ids_mode) {
  if (n == 0) return UC_OK;
  const int nw = sc.nw;
  const uint64_t chunk = (nw == 1) ? sc_chunk<1>() : sc_chunk<2>();
  const size_t sm1 = size_t(2 * chunk) * (8 * nw + 8) + size_t(sc.mc) * 16 + 16;
  // one wave of resident CTAs (the chunks are strided statically)
  int o1 = 0;
  if (nw == 1) UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k_scatter_coarse<1>, COARSE_THREADS, sm1));
  else UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k_scatter_coarse<2>, COARSE_THREADS, sm1));
  if (o1 < 1) return e.fail(UC_EINTERNAL, "scatter kernel does not fit an SM");
  const int g1 = int(std::max<uint64_t>(1, std::min<uint64_t>((n + chunk - 1) / chunk,
                                                              uint64_t(e.sm_count) * uint64_t(o1))));
  e.launches += 1;
  if (nw == 1)
    k_scatter_coarse<1><<<g1, COARSE_THREADS, sm1, e.stream>>>(keys, b1, b2, n, sc.fb, sc.mc, f.cursor, sc.k1, sc.l1,
                                                               sc.b1, ids_mode, e.ctr);
  else
    k_scatter_coarse<2><<<g1, COARSE_THREADS, sm1, e.stream>>>(keys, b1, b2, n, sc.fb, sc.mc, f.cursor, sc.k1, sc.l1,
                                                               sc.b1, ids_mode, e.ctr);
  UC_CK(cudaGetLastError());
  return UC_OK;
}

static int scatter_finish(Env& e, const Front& f, const Scatter& sc, uint64_t*& pkeys, uint32_t*& plink) {
  const int nw = sc.nw;
  pkeys = sc.k2;
  plink = sc.l2;
  if (sc.copies == 0) {
    if (sc.bout) {  // no copies: every bucket empty
      const uint64_t M = uint64_t(sc.nsub) << sc.sb;
      UC_CK(cudaMemsetAsync(sc.cout, 0, M * 4, e.stream));
      UC_CK(cudaMemsetAsync(sc.bout, 0, (M + 1) * 8, e.stream));
    }
    return UC_OK;
  }
  if (sc.mid) {
    const uint32_t nb = 1u << (sc.fb - sc.sb);
    uint32_t* item_start = reinterpret_cast<uint32_t*>(f.cursor + sc.mc);
    const size_t sm2 = size_t(MID_CHUNK) * (8 * nw + 8) + size_t(nb) * 16 + 4 + size_t(sc.mc + 1) * 4;
    int o2 = 0;
    if (nw == 1) UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k_scatter_mid<1>, MID_THREADS, sm2));
    else UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k_scatter_mid<2>, MID_THREADS, sm2));
    if (o2 < 1) return e.fail(UC_EINTERNAL, "scatter kernel does not fit an SM");
    e.launches += 3;
    k_mid_items<<<1, 256, 0, e.stream>>>(sc.goff, sc.fb - sc.cg, sc.mc, item_start);
    k_coarse_init<<<grid_for(e, sc.nsub, 256), 256, 0, e.stream>>>(sc.goff, sc.sb - sc.cg, sc.nsub, f.fcur);
    UC_CK(cudaMemsetAsync(&e.ctr->work_next, 0, 4, e.stream));
    if (nw == 1)
      k_scatter_mid<1><<<e.sm_count * o2, MID_THREADS, sm2, e.stream>>>(sc.k1, sc.l1, sc.b1, sc.goff, sc.cg,
                                                                        item_start, sc.fb, sc.sb, sc.mc, f.fcur,
                                                                        sc.k2, sc.l2, sc.b2, e.ctr);
    else
      k_scatter_mid<2><<<e.sm_count * o2, MID_THREADS, sm2, e.stream>>>(sc.k1, sc.l1, sc.b1, sc.goff, sc.cg,
                                                                        item_start, sc.fb, sc.sb, sc.mc, f.fcur,
                                                                        sc.k2, sc.l2, sc.b2, e.ctr);
    pkeys = sc.k1;
    plink = sc.l1;
  }
  const uint64_t* ik = sc.mid ? sc.k2 : sc.k1;
  const uint32_t* il = sc.mid ? sc.l2 : sc.l1;
  const uint32_t* ib = sc.mid ? sc.b2 : sc.b1;
  UC_CK(cudaMemsetAsync(&e.ctr->work_next, 0, 4, e.stream));
  e.launches += 1;
  const size_t sm3 = size_t(sc.cap3) * (8 * nw + 4);
  int o3 = 0;
  if (nw == 1) UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o3, k_scatter_sub<1>, 512, sm3));
  else UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o3, k_scatter_sub<2>, 512, sm3));
  if (o3 < 1) return e.fail(UC_EINTERNAL, "scatter kernel does not fit an SM");
  const int g3 = int(std::min<uint64_t>(sc.nsub, uint64_t(e.sm_count) * uint64_t(o3)));
  if (nw == 1)
    k_scatter_sub<1><<<g3, 512, sm3, e.stream>>>(ik, il, ib, sc.goff, sc.sb - sc.cg, sc.sb, sc.nsub, sc.cap3, pkeys,
                                                 plink, sc.cout, sc.bout, e.ctr);
  else
    k_scatter_sub<2><<<g3, 512, sm3, e.stream>>>(ik, il, ib, sc.goff, sc.sb - sc.cg, sc.sb, sc.nsub, sc.cap3, pkeys,
                                                 plink, sc.cout, sc.bout, e.ctr);
  UC_CK(cudaGetLastError());
  if (sc.bout) {
    // the total after the last bucket, for the tile plan
    UC_CK(cudaMemcpyAsync(sc.bout + (uint64_t(sc.nsub) << sc.sb), sc.goff + (uint64_t(sc.nsub) << (sc.sb - sc.cg)),
                          8, cudaMemcpyDeviceToDevice, e.stream));
  }
  return UC_OK;
}

// Sort the tiles [t0, t1) (clipped to the tile count) into their tiers.
static int classify_tiles(Env& e, const Front& f, const Plan& P, int nw, uint32_t t0 = 0,
                          uint32_t t1 = 0xFFFFFFFFu) {
  ++e.launches;
  k_classify<<<grid_for(e, P.M, 256), 256, 0, e.stream>>>(f.tile_begin, e.ctr, P.wcap, P.cap, f.wlist, f.blist,
                                                           f.big_list, f.big_size, nw, P.lf, t0, t1);
  UC_CK(cudaGetLastError());
  return UC_OK;
}

// The bucketed copies of all k-mers in one pass, then the tiles (from the
// bucket counts, which level 3 writes when the pack counted groups).
static int plan_and_scatter(Env& e, const Front& f, const Plan& P, uint64_t n, int nw, int ids_mode,
                            char* r1, char* r2, uint64_t copies, uint64_t*& pkeys, uint32_t*& plink,
                            bool group_offsets = false) {
  Scatter sc;
  int r = scatter_begin(e, f, P, nw, r1, r2, copies, sc, group_offsets ? P.cg : 0u, group_offsets);
  if (r) return r;
  r = scatter_l1(e, f, sc, f.keys, f.b1, f.b2, n, ids_mode);
  if (r) return r;
  r = scatter_finish(e, f, sc, pkeys, plink);
  if (r) return r;
  r = plan_tiles(e, f, P);
  if (r) return r;
  return classify_tiles(e, f, P, nw);
}

template <int NW, int KC>
static int run_tiles(Env& e, TileParams& tp, const Front& f, uint32_t threads) {
  tp.wlist = f.wlist;
  tp.blist = f.blist;
  const size_t wsm = size_t(tp.wbytes) * 8;
  int wocc = 0;
  if (tp.wcap) {
    const int r0 = allow_max_smem(e, k_tile_warp<NW, KC>);
    if (r0) return r0;
    UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wocc, k_tile_warp<NW, KC>, 256, wsm));
    if (wocc < 1) return e.fail(UC_EINTERNAL, "warp tile kernel does not fit an SM");
  }
  cudaEventRecord(e.ev[8], e.stream);
  if (tp.wcap) {
    ++e.launches;
    k_tile_warp<NW, KC><<<e.sm_count * wocc, 256, wsm, e.stream>>>(tp);
    UC_CK(cudaGetLastError());
  }
  cudaEventRecord(e.ev[9], e.stream);
  const size_t smem = tile_bytes(NW, tp.cap, tp.tslots);
  const int r1 = allow_max_smem(e, k_tile<NW, KC>);
  if (r1) return r1;
  int occ = 0;
  UC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile<NW, KC>, int(threads), smem));
  if (occ < 1) return e.fail(UC_EINTERNAL, "tile kernel does not fit an SM");
  ++e.launches;
  k_tile<NW, KC><<<e.sm_count * occ, threads, smem, e.stream>>>(tp);
  UC_CK(cudaGetLastError());
  cudaEventRecord(e.ev[5], e.stream);
  e.tiles_timed = true;
  // oversized tiles: one CTA each in global scratch
  int st = e.read_ctr();
  if (st) return st;
  if (e.h_ctr->err) return e.check_err(e.h_ctr);
  const uint32_t nbig = e.h_ctr->nbig;
  if (nbig) {
    std::vector<unsigned long long> sz(nbig), off(nbig);
    UC_CK(cudaMemcpyAsync(sz.data(), f.big_size, nbig * 8, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    unsigned long long tot = 0;
    for (uint32_t i = 0; i < nbig; ++i) {
      off[i] = tot;
      tot += sz[i];
    }
    const size_t want = size_t(tot) + size_t(nbig) * 8 + 4096;
    char* big = nullptr;
    if (e.pool) {
      big = static_cast<char*>(e.take(1, want));
      if (!big) return e.fail(UC_EBUDGET, "scratch for oversized buckets exceeds the pool slice");
    } else if (want > e.big_cap) {
      if (e.big_buf) {
        cudaStreamSynchronize(e.stream);
        cudaFree(e.big_buf);
      }
      e.big_buf = nullptr;
      e.big_cap = 0;
      if (want > e.budget) return e.fail(UC_EBUDGET, "scratch for oversized buckets");
      if (e.dev_malloc(reinterpret_cast<void**>(&e.big_buf), want) != cudaSuccess) {
        cudaGetLastError();
        e.big_buf = nullptr;
        return e.fail(UC_ENOMEM, "scratch for oversized buckets");
      }
      e.big_cap = want;
    }
    if (!big) big = e.big_buf;
    unsigned long long* d_off = reinterpret_cast<unsigned long long*>(big);
    char* scratch = big + ((size_t(nbig) * 8 + 255) & ~size_t(255));
    UC_CK(cudaMemcpyAsync(d_off, off.data(), nbig * 8, cudaMemcpyHostToDevice, e.stream));
    tp.big_list = f.big_list;
    tp.big_scratch = scratch;
    tp.big_off = d_off;
    ++e.launches;
    k_tile_big<NW><<<nbig, 1024, 0, e.stream>>>(tp);
    UC_CK(cudaGetLastError());
    UC_CK(cudaStreamSynchronize(e.stream));
  }
  return UC_OK;
}

// The tile kernels for tp.k: compile-time k = 31 (64-bit keys) and 63
// (128-bit keys), the generic form otherwise.
static int run_tiles_k(Env& e, TileParams& tp, const Front& f, uint32_t threads, int nw) {
  if (nw == 1) return tp.k == 31 ? run_tiles<1, 31>(e, tp, f, threads) : run_tiles<1, 0>(e, tp, f, threads);
  return tp.k == 63 ? run_tiles<2, 63>(e, tp, f, threads) : run_tiles<2, 0>(e, tp, f, threads);
}

int find_edges(Env& e, const uint64_t* d_keys, uint64_t n, int k, int l, uint64_t seed, uint32_t* succ,
               uint32_t* pred) {
  if (k < 2 || k > 63) return e.fail(UC_EINPUT, "k must be in [2, 63]");
  if (l < 1 || l > 16 || l > k - 1) return e.fail(UC_EINPUT, "l must be in [1, min(16, k-1)]");
  if (n >= 0x7FFFFFFFull) return e.fail(UC_EINPUT, "too many k-mers for 31-bit ids");
  if (n == 0) return UC_OK;
  e.reset();
  const int nw = (k <= 31) ? 1 : 2;
  const Plan P = plan_buckets(e, n, 1, k, l);
  int r = e.reserve(0, front_bytes(n, nw, P.M, false));
  if (r) return r;
  Front f{};
  r = take_front(e, n, nw, P.M, false, f);
  if (r) return r;
  f.keys = const_cast<uint64_t*>(d_keys);
  UC_CK(cudaMemsetAsync(e.ctr, 0, sizeof(Counters), e.stream));
  UC_CK(cudaMemsetAsync(f.counts, 0, P.M * 4, e.stream));
  ++e.launches;
  if (nw == 1) k_lmin_count<1><<<grid_for(e, n, 256), 256, 0, e.stream>>>(d_keys, n, k, P.l_used, seed, P.jb, f.b1, f.b2, f.counts);
  else k_lmin_count<2><<<grid_for(e, n, 256), 256, 0, e.stream>>>(d_keys, n, k, P.l_used, seed, P.jb, f.b1, f.b2, f.counts);
  uint64_t copies = 0;
  r = bucket_offsets(e, f, P.M, copies);
  if (r) return r;
  r = e.reserve(1, 2 * scatter_stage_bytes(copies, nw) + 4096);
  if (r) return r;
  char* region1 = static_cast<char*>(e.take(1, scatter_stage_bytes(copies, nw)));
  char* region2 = static_cast<char*>(e.take(1, scatter_stage_bytes(copies, nw)));
  if (!region2) return e.fail(UC_EBUDGET, "back arena overflow");
  uint64_t* pkeys = nullptr;
  uint32_t* plink = nullptr;
  r = plan_and_scatter(e, f, P, n, nw, 1, region1, region2, copies, pkeys, plink);
  if (r) return r;
  TileParams tp{};
  tp.pkeys = pkeys;
  tp.plink = plink;
  tp.tile_begin = f.tile_begin;
  tp.tile_job = f.tile_job;
  tp.ctr = e.ctr;
  tp.k = k;
  tp.cap = P.cap;
  tp.tslots = P.tslots;
  tp.lf = P.lf;
  tp.wcap = P.wcap;
  tp.wts = P.wts;
  tp.wbytes = P.wbytes;
  tp.mode = 0;
  tp.succ = succ;
  tp.pred = pred;
  r = run_tiles_k(e, tp, f, 512, nw);
  if (r) return r;
  r = e.read_ctr();
  e.reset();
  if (r) return r;
  return e.check_err(e.h_ctr);
}

// Enqueue `body` through a CUDA graph: capture it, update the cached
// executable of this slot when the shape key matches (cudaGraphExecUpdate),
// instantiate otherwise, and launch.  The body must only enqueue work.
template <class F>
static int run_graph(Env& e, int slot, uint64_t key, F&& body) {
  if (!e.use_graphs) {
    body();
    return UC_OK;
  }
  const uint32_t before = e.launches;
  // the legacy default stream cannot be captured: capture on an internal
  // stream joined to the caller's stream by events
  const cudaStream_t user = e.stream;
  const bool swap = (user == nullptr || user == cudaStreamLegacy || user == cudaStreamPerThread);
  if (swap) {
    if (!e.gstream) UC_CK(cudaStreamCreateWithFlags(&e.gstream, cudaStreamNonBlocking));
    UC_CK(cudaEventRecord(e.ev[6], user));
    UC_CK(cudaStreamWaitEvent(e.gstream, e.ev[6], 0));
    e.stream = e.gstream;
  }
  struct Restore {
    Env& e;
    cudaStream_t user;
    bool swap;
    ~Restore() {
      if (swap) {
        cudaEventRecord(e.ev[7], e.stream);
        cudaStreamWaitEvent(user, e.ev[7], 0);
        e.stream = user;
      }
    }
  } restore{e, user, swap};
  UC_CK(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
  body();
  cudaGraph_t g = nullptr;
  UC_CK(cudaStreamEndCapture(e.stream, &g));
  bool ok = false;
  if (e.gexec[slot] && e.gkey[slot] == key) {
    cudaGraphExecUpdateResultInfo info;
    ok = cudaGraphExecUpdate(e.gexec[slot], g, &info) == cudaSuccess;
    if (!ok) cudaGetLastError();
  }
  if (!ok) {
    if (e.gexec[slot]) cudaGraphExecDestroy(e.gexec[slot]);
    e.gexec[slot] = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&e.gexec[slot], g, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g);
      return e.fail(UC_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
    }
    e.gkey[slot] = key;
  }
  cudaGraphDestroy(g);
  UC_CK(cudaGraphLaunch(e.gexec[slot], e.stream));
  e.graph_nodes += e.launches - before;
  return UC_OK;
}

// prefilled: X already holds a state (written by the tiles and the line
// walk) and the first round runs over the ids [0, cnt[0]), cnt[0] set on the
// device before.
static int rank_lists(Env& e, const uint32_t* prev, const uint32_t* w, uint64_t nmax, bool count_on_device,
                      unsigned long long* X, uint32_t* act0, uint32_t* act1, uint32_t* cnt, uint32_t& rounds,
                      uint32_t*& act_final, uint32_t*& cnt_final, bool prefilled = false) {
  rounds = 2;
  for (uint64_t t = 1; t < nmax; t <<= 1) ++rounds;
  const int grid = grid_for(e, nmax ? nmax : 1, 256);
  if (prefilled) {
    UC_CK(cudaMemsetAsync(cnt + 1, 0, rounds * 4, e.stream));
  } else {
    UC_CK(cudaMemsetAsync(cnt, 0, (rounds + 1) * 4, e.stream));
    ++e.launches;
    k_rank_init<<<grid, 256, 0, e.stream>>>(prev, w, nmax, count_on_device ? e.ctr : nullptr, X, act0, cnt);
  }
  uint32_t* lists[2] = {act0, act1};
  for (uint32_t r = 0; r < rounds; ++r) {
    ++e.launches;
    const uint32_t* in = (r == 0 && prefilled) ? nullptr : lists[r & 1];
    k_rank_round<<<grid, 256, 0, e.stream>>>(X, in, cnt + r, lists[(r + 1) & 1], cnt + r + 1);
  }
  UC_CK(cudaGetLastError());
  act_final = lists[rounds & 1];
  cnt_final = cnt + rounds;
  return UC_OK;
}

static size_t hec_bytes(uint64_t nmax, uint32_t R) {
  const uint64_t cap = 2 * nmax + 64;
  return 8 * ((cap * 4 + 255) & ~uint64_t(255)) + 2 * 256 + 2 * (R + 1) * 4 + 1024;
}

static int hec_take(Env& e, uint64_t nmax, uint32_t R, HecPool& h) {
  const uint64_t cap = 2 * nmax + 64;
  uint32_t** arr[8] = {&h.prv, &h.nxt, &h.wt, &h.hn, &h.vc, &h.agg, &h.loc, &h.first0};
  for (auto a : arr) *a = static_cast<uint32_t*>(e.take(1, cap * 4));
  h.lb = static_cast<uint32_t*>(e.take(1, (R + 1) * 4));
  h.ln = static_cast<uint32_t*>(e.take(1, (R + 1) * 4));
  h.cap = uint32_t(std::min<uint64_t>(cap, 0xFFFFFFF0ull));
  h.ctr = e.ctr;
  if (!h.ln) return e.fail(UC_EBUDGET, "arena overflow (HEC pool)");
  return UC_OK;
}

static uint32_t hec_rounds(uint64_t nmax) {
  uint32_t r = 8;
  for (uint64_t t = 1; t < nmax; t <<= 1) r += 2;
  return r;
}
// The rounds a run enqueues: the bound above, or the injected cap.
static uint32_t hec_rounds(const Env& e, uint64_t nmax) {
  const uint32_t r = hec_rounds(nmax);
  return (e.faults.hec_round_cap && e.faults.hec_round_cap < r) ? e.faults.hec_round_cap : r;
}

// HEC contraction of the lists (prev, next, w) into X (pointer | HEAD_BIT,
// offset) and cycle flags, all rounds enqueued on the stream.
// With seg, level 0 comes from the fused path's segment records and the
// ranking's first state in X (built from them by k_seg_xinit; nx cross
// indices) instead of (prev, next, w).
static void hec_contract(Env& e, HecPool& h, uint32_t R, const uint32_t* prev, const uint32_t* next,
                         const uint32_t* w, uint64_t nmax, bool count_on_device, unsigned long long* X,
                         uint8_t* oncycle, const SegRec* seg = nullptr, uint32_t nx = 0, int k = 0) {
  const int grid = grid_for(e, nmax ? nmax : 1, 256);
  cudaMemsetAsync(h.ln, 0, (R + 1) * 4, e.stream);
  ++e.launches;
  if (seg) k_hec_level0_seg<<<grid, 256, 0, e.stream>>>(h, seg, X, nmax, nx, k);
  else k_hec_level0<<<grid, 256, 0, e.stream>>>(h, prev, next, w, nmax, count_on_device ? e.ctr : nullptr);
  for (uint32_t r = 0; r < R; ++r) {
    e.launches += 6;
    k_hec_prep<<<grid, 256, 0, e.stream>>>(h, int(r));
    k_hec_match<<<grid, 256, 0, e.stream>>>(h, int(r), 1);
    k_hec_match<<<grid, 256, 0, e.stream>>>(h, int(r), 2);
    k_hec_roots<<<grid, 256, 0, e.stream>>>(h, int(r));
    k_hec_assign<<<grid, 256, 0, e.stream>>>(h, int(r));
    k_hec_order<<<grid, 256, 0, e.stream>>>(h, int(r));
  }
  e.launches += 1 + R + 1;
  k_hec_check<<<1, 1, 0, e.stream>>>(h, int(R));
  for (int r = int(R) - 1; r >= 0; --r) k_hec_down<<<grid, 256, 0, e.stream>>>(h, r);
  k_hec_emit<<<grid, 256, 0, e.stream>>>(h, X, oncycle);
}

static int contract_hec(Env& e, const uint64_t* d_keys, const uint32_t* succ, const uint32_t* pred, uint64_t n,
                        int k, uint32_t* head, uint32_t* rank, uint64_t& ncyc, bool& fell_back) {
  fell_back = false;
  e.reset();
  const uint32_t R = hec_rounds(e, n);
  int r = e.reserve(1, hec_bytes(n, R) + n * (8 + 4 + 1) + 8 + 4096);
  if (r) return r;
  HecPool h{};
  r = hec_take(e, n, R, h);
  if (r) return r;
  unsigned long long* X = static_cast<unsigned long long*>(e.take(1, n * 8));
  uint32_t* act = static_cast<uint32_t*>(e.take(1, n * 4));
  uint8_t* flag = static_cast<uint8_t*>(e.take(1, n));
  uint32_t* cnt = static_cast<uint32_t*>(e.take(1, 4));
  unsigned long long* dcyc = static_cast<unsigned long long*>(e.take(1, 8));
  if (!dcyc) return e.fail(UC_EBUDGET, "arena overflow");
  UC_CK(cudaMemsetAsync(&e.ctr->err, 0, 4, e.stream));
  UC_CK(cudaMemsetAsync(flag, 0, n, e.stream));
  hec_contract(e, h, R, pred, succ, nullptr, n, false, X, flag);
  e.launches += 2;
  k_head_rank<<<grid_for(e, n, 256), 256, 0, e.stream>>>(X, n, head, rank);
  UC_CK(cudaMemsetAsync(cnt, 0, 4, e.stream));
  k_cycle_list<<<grid_for(e, n, 256), 256, 0, e.stream>>>(flag, n, nullptr, act, cnt);
  uint32_t hleft = 0;
  UC_CK(cudaMemcpyAsync(&hleft, cnt, 4, cudaMemcpyDeviceToHost, e.stream));
  r = e.read_ctr();
  if (r) return r;
  if (e.h_ctr->err) {
    if (e.faults.hec_strict) {
      r = e.check_err(e.h_ctr);
      UC_CK(cudaMemsetAsync(&e.ctr->err, 0, 4, e.stream));
      e.reset();
      return r;
    }
    fell_back = true;
    UC_CK(cudaMemsetAsync(&e.ctr->err, 0, 4, e.stream));
    e.reset();
    return UC_OK;
  }
  ncyc = 0;
  if (hleft) {
    UC_CK(cudaMemsetAsync(flag, 0, n, e.stream));
    UC_CK(cudaMemsetAsync(dcyc, 0, 8, e.stream));
    ++e.launches;
    if (k <= 31) k_vertex_cycles<1><<<1, 1, 0, e.stream>>>(act, hleft, succ, d_keys, n, head, rank, flag, dcyc);
    else k_vertex_cycles<2><<<1, 1, 0, e.stream>>>(act, hleft, succ, d_keys, n, head, rank, flag, dcyc);
    unsigned long long hc = 0;
    UC_CK(cudaMemcpyAsync(&hc, dcyc, 8, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    ncyc = hc;
  }
  e.reset();
  return UC_OK;
}

int contract(Env& e, const uint64_t* d_keys, const uint32_t* succ, const uint32_t* pred, uint64_t n, int k,
             int method, uint32_t* head, uint32_t* rank, uint64_t& ncyc) {
  if (k < 2 || k > 63) return e.fail(UC_EINPUT, "k must be in [2, 63]");
  if (n >= 0x7FFFFFFFull) return e.fail(UC_EINPUT, "too many k-mers for 31-bit ids");
  ncyc = 0;
  if (n == 0) return UC_OK;
  if (method == UC_CONTRACT_HEC) {
    bool fell_back = false;
    const int r = contract_hec(e, d_keys, succ, pred, n, k, head, rank, ncyc, fell_back);
    if (r || !fell_back) return r;
    // HEC did not finish inside its pool or rounds: pointer jumping instead
  }
  e.reset();
  int r = e.reserve(1, n * (8 + 4 + 4 + 1) + 64 * 8 + 4096);
  if (r) return r;
  unsigned long long* X = static_cast<unsigned long long*>(e.take(1, n * 8));
  uint32_t* a0 = static_cast<uint32_t*>(e.take(1, n * 4));
  uint32_t* a1 = static_cast<uint32_t*>(e.take(1, n * 4));
  uint8_t* seen = static_cast<uint8_t*>(e.take(1, n));
  uint32_t* cnt = static_cast<uint32_t*>(e.take(1, 64 * 4));
  unsigned long long* dcyc = static_cast<unsigned long long*>(e.take(1, 8));
  if (!dcyc) return e.fail(UC_EBUDGET, "arena overflow");
  uint32_t rounds = 0;
  uint32_t *act = nullptr, *left = nullptr;
  r = rank_lists(e, pred, nullptr, n, false, X, a0, a1, cnt, rounds, act, left);
  if (r) return r;
  ++e.launches;
  k_head_rank<<<grid_for(e, n, 256), 256, 0, e.stream>>>(X, n, head, rank);
  uint32_t hleft = 0;
  UC_CK(cudaMemcpyAsync(&hleft, left, 4, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  if (hleft) {
    UC_CK(cudaMemsetAsync(seen, 0, n, e.stream));
    UC_CK(cudaMemsetAsync(dcyc, 0, 8, e.stream));
    ++e.launches;
    if (k <= 31) k_vertex_cycles<1><<<1, 1, 0, e.stream>>>(act, hleft, succ, d_keys, n, head, rank, seen, dcyc);
    else k_vertex_cycles<2><<<1, 1, 0, e.stream>>>(act, hleft, succ, d_keys, n, head, rank, seen, dcyc);
    unsigned long long hc = 0;
    UC_CK(cudaMemcpyAsync(&hc, dcyc, 8, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    ncyc = hc;
  }
  e.reset();
  return UC_OK;
}

int emit(Env& e, const uint64_t* d_keys, const uint32_t* succ, const uint32_t* head, const uint32_t* rank,
         uint64_t n, int k, char* out, uint64_t cap, uint64_t& out_bytes) {
  (void)succ;
  if (k < 2 || k > 63) return e.fail(UC_EINPUT, "k must be in [2, 63]");
  out_bytes = 0;
  if (n == 0) return UC_OK;
  e.reset();
  int r = e.reserve(1, n * 16 + scan_tmp_elems(n) * 8 + 4096);
  if (r) return r;
  uint32_t* cnt = static_cast<uint32_t*>(e.take(1, n * 4));
  uint32_t* len = static_cast<uint32_t*>(e.take(1, n * 4));
  unsigned long long* loff = static_cast<unsigned long long*>(e.take(1, (n + 1) * 8));
  unsigned long long* tmp = static_cast<unsigned long long*>(e.take(1, scan_tmp_elems(n) * 8));
  if (!tmp) return e.fail(UC_EBUDGET, "arena overflow");
  UC_CK(cudaMemsetAsync(cnt, 0, n * 4, e.stream));
  const int grid = grid_for(e, n, 256);
  e.launches += 2 + 6;
  k_count_members<<<grid, 256, 0, e.stream>>>(head, n, cnt);
  k_line_len<<<grid, 256, 0, e.stream>>>(head, cnt, n, k, len);
  scan_excl<uint32_t, unsigned long long>(len, n, loff, tmp, e.stream);
  unsigned long long total = 0;
  UC_CK(cudaMemcpyAsync(&total, loff + n, 8, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  out_bytes = total;
  if (out) {
    if (total > cap) return e.fail(UC_EINPUT, "output buffer too small");
    ++e.launches;
    if (k <= 31) k_spell<1><<<grid, 256, 0, e.stream>>>(d_keys, head, rank, cnt, loff, n, k, out);
    else k_spell<2><<<grid, 256, 0, e.stream>>>(d_keys, head, rank, cnt, loff, n, k, out);
    UC_CK(cudaGetLastError());
    UC_CK(cudaStreamSynchronize(e.stream));
  }
  e.reset();
  return UC_OK;
}

uint64_t emit_scratch_bytes(uint64_t n) {
  auto al = [](uint64_t b) { return (b + 255) & ~uint64_t(255); };
  return 2 * al(n * 4) + al((n + 1) * 8) + al(scan_tmp_elems(n) * 8);
}

int emit_preload(std::string& err) {
  const void* fns[] = {
      reinterpret_cast<const void*>(k_count_members),
      reinterpret_cast<const void*>(k_line_len),
      reinterpret_cast<const void*>(k_scan_reduce<uint32_t, unsigned long long>),
      reinterpret_cast<const void*>(k_scan_down<uint32_t, unsigned long long>),
      reinterpret_cast<const void*>(k_scan_reduce<unsigned long long, unsigned long long>),
      reinterpret_cast<const void*>(k_scan_down<unsigned long long, unsigned long long>),
      reinterpret_cast<const void*>(k_spell<1>),
      reinterpret_cast<const void*>(k_spell<2>)};
  for (const void* f : fns) {
    cudaFuncAttributes a;
    const cudaError_t c = cudaFuncGetAttributes(&a, f);
    if (c != cudaSuccess) {
      cudaGetLastError();
      err = std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(c);
      return UC_ECUDA;
    }
  }
  return UC_OK;
}

int emit_in(cudaStream_t s, int sm_count, const uint64_t* d_keys, const uint32_t* head, const uint32_t* rank,
            uint64_t n, int k, char* out, uint64_t cap, uint64_t& out_bytes, void* scratch, std::string& err) {
  out_bytes = 0;
  if (k < 2 || k > 63) {
    err = "k must be in [2, 63]";
    return UC_EINPUT;
  }
  if (n == 0) return UC_OK;
  auto al = [](uint64_t b) { return (b + 255) & ~uint64_t(255); };
  char* p = static_cast<char*>(scratch);
  uint32_t* cnt = reinterpret_cast<uint32_t*>(p);
  uint32_t* len = reinterpret_cast<uint32_t*>(p + al(n * 4));
  unsigned long long* loff = reinterpret_cast<unsigned long long*>(p + 2 * al(n * 4));
  unsigned long long* tmp = reinterpret_cast<unsigned long long*>(p + 2 * al(n * 4) + al((n + 1) * 8));
  auto ck = [&](cudaError_t c, const char* what) -> int {
    if (c == cudaSuccess) return UC_OK;
    err = std::string(what) + ": " + cudaGetErrorString(c);
    return int(UC_ECUDA);
  };
  const uint64_t want = (n + 255) / 256, gcap = uint64_t(sm_count) * 16;
  const int grid = int(std::max<uint64_t>(1, std::min(want, gcap)));
  int r = ck(cudaMemsetAsync(cnt, 0, n * 4, s), "cudaMemsetAsync");
  if (r) return r;
  k_count_members<<<grid, 256, 0, s>>>(head, n, cnt);
  k_line_len<<<grid, 256, 0, s>>>(head, cnt, n, k, len);
  scan_excl<uint32_t, unsigned long long>(len, n, loff, tmp, s);
  unsigned long long total = 0;
  if ((r = ck(cudaGetLastError(), "launch"))) return r;
  if ((r = ck(cudaMemcpyAsync(&total, loff + n, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync"))) return r;
  if ((r = ck(cudaStreamSynchronize(s), "cudaStreamSynchronize"))) return r;
  out_bytes = total;
  if (out) {
    if (total > cap) {
      err = "output buffer too small";
      return UC_EINPUT;
    }
    if (k <= 31) k_spell<1><<<grid, 256, 0, s>>>(d_keys, head, rank, cnt, loff, n, k, out);
    else k_spell<2><<<grid, 256, 0, s>>>(d_keys, head, rank, cnt, loff, n, k, out);
    if ((r = ck(cudaGetLastError(), "launch"))) return r;
    if ((r = ck(cudaStreamSynchronize(s), "cudaStreamSynchronize"))) return r;
  }
  return UC_OK;
}

uint64_t output_bound(size_t text_bytes, int k) {
  (void)k;
  return uint64_t(text_bytes) + 64;
}

// Segment arrays of the fused path's stitch (in the back arena).
struct StitchBufs {
  SegRec* seg;
  unsigned long long* Xr;
  char* segc;
  uint32_t *act0, *act1;
  uint8_t* oncyc;
  uint32_t* hlen;
  unsigned long long* lbase;
  uint32_t* longl;  // heads of the lines the walk leaves (lcap entries)
  uint32_t lcap;
  uint32_t* rcnt;
  HecPool hp;
};

// Heads the walk can leave: each left line holds more than the walk's cap
// of cross ids.
static uint32_t walk_cap(const Env& e) {
  return (e.faults.walk_cap && e.faults.walk_cap < WALK_CAP) ? e.faults.walk_cap : WALK_CAP;
}
static uint64_t long_cap(const Env& e, uint64_t X) { return X / walk_cap(e) + 64; }

// The cross-tile stitch over X cross-indexed segments and Hp head-pool ids,
// into out after each job's closed lines (jd.jout: each job's byte count,
// closed lines before, all lines after): the line walk, then, for the
// lines it leaves and for cycles, ranking (pointer jumping, or HEC with
// pointer jumping when its rounds run out), line lengths at the heads, one
// reservation per line, the segment copies, and the rare segment cycles.
static int run_stitch(Env& e, const StitchBufs& b, uint64_t X, uint64_t Hp, int k, int nw, bool want_hec,
                      uint32_t RH, const JobDev& jd, char* out, uint32_t& rounds) {
  rounds = 0;
  const uint32_t S = uint32_t(X + Hp), nx = uint32_t(X), H = uint32_t(Hp);
  SegRec* seg = b.seg;
  unsigned long long* Xr = b.Xr;
  char* segc = b.segc;
  uint32_t *act0 = b.act0, *act1 = b.act1, *hlen = b.hlen, *rcnt = b.rcnt;
  uint8_t* oncyc = b.oncyc;
  unsigned long long* lbase = b.lbase;
  HecPool hp = b.hp;
  uint32_t* wst = rcnt + 48;  // the walk's counters (the rounds use at most 35 list counts)
  int r = UC_OK;
  const int gs = grid_for(e, S, 256);
  uint32_t *act = nullptr, *left = nullptr;
  uint32_t nlong = 0;
  if (!want_hec) {
    // the line walk writes every line its head reaches within WALK_CAP
    // segments; the rest is ranked from the first state, built below
    UC_CK(cudaMemsetAsync(wst, 0, 8, e.stream));
    ++e.launches;
    k_walk_emit<<<grid_for(e, H, 256), 256, 0, e.stream>>>(H, seg, nx, k, jd.tab, jd.jout, segc, out, walk_cap(e),
                                                           b.longl, b.lcap, wst, e.ctr);
    uint32_t hw[2] = {0, 0};
    UC_CK(cudaMemcpyAsync(hw, wst, 8, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    if (hw[0] == nx && hw[1] == 0) return UC_OK;
    nlong = std::min(hw[1], b.lcap);
    ++e.launches;
    k_set_u32<<<1, 1, 0, e.stream>>>(rcnt, nx);
  }
  // the first state (HEC's level 0 takes the predecessors from it)
  ++e.launches;
  k_seg_xinit<<<gs, 256, 0, e.stream>>>(S, seg, nx, k, Xr);
  bool hec = want_hec;
  if (hec) {
    // HEC matching rounds, captured as one graph
    r = run_graph(e, 1, (uint64_t(RH) << 32) | uint32_t(gs), [&] {
      cudaMemsetAsync(oncyc, 0, S, e.stream);
      hec_contract(e, hp, RH, nullptr, nullptr, nullptr, S, false, Xr, oncyc, seg, nx, k);
      cudaMemsetAsync(rcnt, 0, 4, e.stream);
      ++e.launches;
      k_cycle_list<<<gs, 256, 0, e.stream>>>(oncyc, S, nullptr, act0, rcnt);
    });
    if (r) return r;
    act = act0;
    left = rcnt;
    rounds = RH;
    r = e.read_ctr();
    if (r) return r;
    if (e.h_ctr->err) {  // did not finish in its pool/rounds: pointer jumping
      if (e.faults.hec_strict) return e.check_err(e.h_ctr);
      UC_CK(cudaMemsetAsync(&e.ctr->err, 0, 4, e.stream));
      hec = false;
    }
  }
  if (!hec) {
    // pointer-jumping rounds, captured as one graph: after the walk from the
    // state rebuilt above (over the ids [0, X)); after a HEC attempt from
    // the level-0 links the HEC pool kept
    uint32_t rr = 2;
    for (uint64_t t = 1; t < S; t <<= 1) ++rr;
    int rl = UC_OK;
    const bool prefilled = !want_hec;
    r = run_graph(e, 0, (uint64_t(rr) << 33) | (uint64_t(prefilled) << 32) | uint32_t(gs), [&] {
      rl = prefilled ? rank_lists(e, nullptr, nullptr, S, false, Xr, act0, act1, rcnt, rounds, act, left, true)
                     : rank_lists(e, hp.prv, hp.wt, S, false, Xr, act0, act1, rcnt, rounds, act, left);
      cudaMemsetAsync(oncyc, 0, S, e.stream);
      ++e.launches;
      k_mark_cycle<<<gs, 256, 0, e.stream>>>(act, left, oncyc);
    });
    if (r) return r;
    if (rl) return rl;
  }
  // line length at each head, one reservation per line not yet written,
  // then every segment's chars (the segments of written lines skip)
  UC_CK(cudaMemsetAsync(hlen, 0, size_t(H) * 4, e.stream));
  UC_CK(cudaMemsetAsync(lbase, 0xFF, size_t(H) * 8, e.stream));
  e.launches += 2;
  k_chain_len<<<gs, 256, 0, e.stream>>>(S, seg, Xr, oncyc, nx, k, hlen, e.ctr);
  if (want_hec) {
    ++e.launches;
    k_line_reserve<<<grid_for(e, H, 256), 256, 0, e.stream>>>(H, nullptr, seg + nx, jd.tab, jd.jout, hlen, lbase,
                                                              e.ctr);
  } else if (nlong) {
    ++e.launches;
    k_line_reserve<<<grid_for(e, nlong, 256), 256, 0, e.stream>>>(nlong, b.longl, seg + nx, jd.tab, jd.jout, hlen,
                                                                  lbase, e.ctr);
  }
  k_seg_copy<<<grid_for(e, S, 256), 256, 0, e.stream>>>(S, seg, Xr, oncyc, nx, lbase, segc, out, k);
  uint32_t hleft = 0;
  UC_CK(cudaMemcpyAsync(&hleft, left, 4, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  if (hleft) {
    ++e.launches;
    if (nw == 1)
      k_seg_cycles<1><<<1, 1, 0, e.stream>>>(e.ctr, S, act, hleft, oncyc, seg, jd.tab, jd.jout, segc, out, k);
    else
      k_seg_cycles<2><<<1, 1, 0, e.stream>>>(e.ctr, S, act, hleft, oncyc, seg, jd.tab, jd.jout, segc, out, k);
  }
  UC_CK(cudaGetLastError());
  return UC_OK;
}

// Back arena bytes of the fused path: the bucketed copies and their staging,
// the segment pool (Sp segments for X cross k-mers) and the stitch arrays.
static size_t back_bytes(const Env& e, uint64_t copies, uint64_t X, uint64_t Sp, int nw, int k, bool want_hec) {
  const uint64_t segchars = Sp * uint64_t(k) + copies + 64;
  const uint32_t R = 64;
  size_t back = 0;
  auto add = [&](size_t b) { back += (b + 255) & ~size_t(255); };
  const uint64_t Hp = Sp - X;                                             // head pools
  add(scatter_stage_bytes(copies, nw)); add(scatter_stage_bytes(copies, nw));  // the scatter's two regions
  add(Sp * sizeof(SegRec)); add(Sp * 8);                                  // segment records, ranking
  add(segchars);
  add(Sp * 4); add(Sp * 4); add(Sp);                                      // act0, act1, oncyc
  add(Hp * 4); add(Hp * 8); add(long_cap(e, X) * 4);                         // line lengths, bases, left lines
  add(R * 4);
  if (want_hec) add(hec_bytes(Sp, hec_rounds(Sp)));
  return back;
}

void batch_footprint(const Env& e, uint32_t njobs, const size_t* bytes, int k, int l, size_t& front,
                     size_t& back) {
  const int nw = (k <= 31) ? 1 : 2;
  uint64_t N = 0, nmax = 0, tb = 0;
  for (uint32_t j = 0; j < njobs; ++j) {
    const uint64_t n = (uint64_t(bytes[j]) + 1) / uint64_t(k + 1) + 1;
    N += n;
    nmax = std::max(nmax, n);
    tb = std::max<uint64_t>(tb, bytes[j]);
  }
  const Plan P = plan_buckets(e, nmax, njobs, k, l);
  const size_t slack = size_t(16) << 20;
  front = front_bytes(N, nw, P.M, true) + slack + 4096;
  const uint64_t X = N, copies = N + X, Sp = 2 * X + njobs;
  back = std::max(back_bytes(e, copies, X, Sp, nw, k, e.tune.contract_method == UC_CONTRACT_HEC),
                  line_index_bytes(tb, nmax)) + slack + 4096;
}

// The fused path.  Device memory: the front arena holds per-k-mer arrays
// (keys, bucket ids) and per-bucket arrays; the back arena, sized once the
// cross k-mers X are counted, holds the n+X bucketed copies and the segment
// arrays (at most 2X open segments: each holds an S-only start or a P-only
// end, one of each per cross k-mer).
// The fused path over a batch of jobs (one job is a batch of one).  Device
// memory: the front arena holds per-k-mer arrays (keys, bucket ids) and
// per-bucket arrays; the back arena, sized once the cross k-mers are counted,
// holds the bucketed copies and the segment pools (a job with X cross k-mers
// has at most 2X open segments: each holds an S-only start or a P-only end).
int compact_batch(Env& e, uint32_t njobs, const char* const* texts, const size_t* bytes, int k, int l, char* out,
                  uint64_t out_cap, uint64_t* out_off, uint64_t* out_len, uc_stats* st) {
  if (k < 2 || k > 63) return e.fail(UC_EINPUT, "k must be in [2, 63]");
  if (l < 1 || l > 16 || l > k - 1) return e.fail(UC_EINPUT, "l must be in [1, min(16, k-1)]");
  if (njobs == 0) return UC_OK;
  const int nw = (k <= 31) ? 1 : 2;
  e.reset();
  e.launches = 0;
  e.graph_nodes = 0;
  int r = job_buffers(e, njobs);
  if (r) return r;
  JobDev jd = job_dev(e, njobs);
  std::vector<JobTab> J(njobs);
  if (njobs == 1) {
    r = host_job(e, texts[0], bytes[0], k, J[0]);
    if (r) return r;
  } else {
    for (uint32_t j = 0; j < njobs; ++j) {
      J[j] = JobTab{};
      J[j].text = reinterpret_cast<const uint8_t*>(texts[j]);
      J[j].tbytes = bytes[j];
    }
    UC_CK(cudaMemcpyAsync(jd.tab, J.data(), njobs * sizeof(JobTab), cudaMemcpyHostToDevice, e.stream));
    ++e.launches;
    k_headers<<<(njobs + 127) / 128, 128, 0, e.stream>>>(jd.tab, njobs, k);
    UC_CK(cudaMemcpyAsync(J.data(), jd.tab, njobs * sizeof(JobTab), cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    for (uint32_t j = 0; j < njobs; ++j) {
      if (J[j].err) return e.fail(UC_EINPUT, "job " + std::to_string(j) + ": missing or too large k-mer count");
      if (!J[j].fixed)
        return e.fail(UC_EINPUT, "job " + std::to_string(j) +
                                     ": batched jobs need k chars + '\\n' per line and a matching count");
    }
  }
  uint64_t N = 0, lb = 0, ob = 0, nmax = 0;
  for (uint32_t j = 0; j < njobs; ++j) {
    J[j].koff = N;
    J[j].lb0 = lb;
    J[j].obase = ob;
    J[j].ocap = output_bound(bytes[j], k);
    N += J[j].n;
    lb += (J[j].n + PACK_LINES - 1) / PACK_LINES;
    ob += (J[j].ocap + 15) & ~uint64_t(15);
    nmax = std::max<uint64_t>(nmax, J[j].n);
  }
  if (N >= 0x7FFFFFFFull) return e.fail(UC_EINPUT, "too many k-mers for 31-bit ids");
  if (ob > out_cap + 15) return e.fail(UC_EINPUT, "output buffer smaller than uc_output_bound");
  const Plan P = plan_buckets(e, nmax, njobs, k, l);
  r = e.reserve(0, front_bytes(N, nw, P.M, true));
  if (r) return r;
  Front f{};
  r = take_front(e, N, nw, P.M, true, f);
  if (r) return r;
  // the pack's counts: per group of 2^cg buckets, or (cg = 0) per bucket
  const uint64_t G = P.M >> P.cg;
  uint32_t* gcount = P.cg ? f.gcount : f.counts;
  unsigned long long* goff = P.cg ? f.goff : f.boff;
  UC_CK(cudaMemsetAsync(e.ctr, 0, sizeof(Counters), e.stream));
  UC_CK(cudaMemsetAsync(gcount, 0, G * 4, e.stream));
  UC_CK(cudaMemsetAsync(jd.jcross, 0, njobs * 4, e.stream));
  UC_CK(cudaMemcpyAsync(jd.tab, J.data(), njobs * sizeof(JobTab), cudaMemcpyHostToDevice, e.stream));
  cudaEventRecord(e.ev[0], e.stream);
  FuseArgs fz;
  fz.l = P.l_used;
  fz.seed = e.seed;
  fz.jb = P.jb;
  fz.b1 = f.b1;
  fz.b2 = f.b2;
  fz.counts = gcount;
  fz.cshift = P.cg;
  fz.cbytes = G * 4;
  fz.jcross = jd.jcross;
  fz.M = P.M;
  if (njobs == 1) {
    r = pack_single(e, texts[0], bytes[0], k, f.keys, &fz, J[0], jd.tab);
    if (r) return r;
  } else if (N > 0) {
    if (nw == 1) launch_pack<1>(e, jd.tab, nullptr, njobs, lb, nullptr, k, f.keys, &fz);
    else launch_pack<2>(e, jd.tab, nullptr, njobs, lb, nullptr, k, f.keys, &fz);
    UC_CK(cudaGetLastError());
  }
  cudaEventRecord(e.ev[1], e.stream);
  if (e.after_pack) e.after_pack();
  uint64_t copies = 0;
  r = bucket_offsets(e, f, gcount, G, goff, copies);
  if (r) return r;
  std::vector<uint32_t> xc(njobs);
  UC_CK(cudaMemcpyAsync(xc.data(), jd.jcross, njobs * 4, cudaMemcpyDeviceToHost, e.stream));
  r = e.read_ctr();
  if (r) return r;
  uint64_t xsum = 0;
  for (uint32_t j = 0; j < njobs; ++j) xsum += xc[j];
  if (copies != N + xsum && !e.h_ctr->err) return e.fail(UC_EINTERNAL, "bucket counts disagree with the copies");
  if (e.h_ctr->err) {
    if (e.h_ctr->err & ERR_LAYOUT) return e.fail(UC_EINPUT, "a k-mer line is shorter than k");
    return e.check_err(e.h_ctr);
  }
  const uint64_t X = copies - N;
  // segment ids: [0, X) the segments that start at a cross k-mer's S-only
  // copy; then each job's head pool (a line's first open segment ends at a
  // P-only copy, so a job has at most one per cross k-mer)
  uint64_t Hp = 0;
  for (uint32_t j = 0; j < njobs; ++j) {
    J[j].seg_base = uint32_t(Hp);
    J[j].seg_cap = xc[j] + 1;
    Hp += J[j].seg_cap;
  }
  const uint64_t Sp = X + Hp;
  if (Sp >= 0x7FFFFFF0ull) return e.fail(UC_EINPUT, "too many cross-tile segments");
  if (njobs >= (1u << (64 - SEG_OFF_BITS))) return e.fail(UC_EINPUT, "too many jobs in one batch");
  UC_CK(cudaMemcpyAsync(jd.tab, J.data(), njobs * sizeof(JobTab), cudaMemcpyHostToDevice, e.stream));
  const uint64_t segchars = Sp * uint64_t(k) + copies + 64;
  if (segchars > SEG_OFF_MASK) return e.fail(UC_EINPUT, "segment chars beyond the 40-bit offsets");
  const uint32_t R = 64;
  const bool want_hec = e.tune.contract_method == UC_CONTRACT_HEC;
  const uint32_t RH = hec_rounds(e, Sp);
  const size_t back = back_bytes(e, copies, X, Sp, nw, k, want_hec);
  r = e.reserve(1, back);
  if (r) return r;
  auto T64 = [&](uint64_t c) { return static_cast<unsigned long long*>(e.take(1, c * 8)); };
  auto T32 = [&](uint64_t c) { return static_cast<uint32_t*>(e.take(1, c * 4)); };
  char* region1 = static_cast<char*>(e.take(1, scatter_stage_bytes(copies, nw)));
  char* region2 = static_cast<char*>(e.take(1, scatter_stage_bytes(copies, nw)));
  SegRec* seg = static_cast<SegRec*>(e.take(1, Sp * sizeof(SegRec)));
  unsigned long long* Xr = T64(Sp);
  char* segc = static_cast<char*>(e.take(1, segchars));
  uint32_t* act0 = T32(Sp);
  uint32_t* act1 = T32(Sp);
  uint8_t* oncyc = static_cast<uint8_t*>(e.take(1, Sp));
  uint32_t* hlen = T32(Hp);
  unsigned long long* lbase = T64(Hp);
  uint32_t* longl = T32(long_cap(e, X));
  uint32_t* rcnt = T32(R);
  if (!rcnt) return e.fail(UC_EBUDGET, "back arena overflow");
  HecPool hp{};
  if (want_hec) {
    r = hec_take(e, Sp, RH, hp);
    if (r) return r;
  }
  // unused head-pool ids keep length 0 (every id below X gets a record)
  UC_CK(cudaMemsetAsync(seg + X, 0, Hp * sizeof(SegRec), e.stream));
  UC_CK(cudaMemsetAsync(jd.jout, 0, njobs * 8, e.stream));
  UC_CK(cudaMemsetAsync(jd.jseg, 0, njobs * 4, e.stream));
  uint64_t* pkeys = nullptr;
  uint32_t* plink = nullptr;
  r = plan_and_scatter(e, f, P, N, nw, 0, region1, region2, copies, pkeys, plink, P.cg > 0);
  if (r) return r;
  cudaEventRecord(e.ev[2], e.stream);

  TileParams tp{};
  tp.pkeys = pkeys;
  tp.plink = plink;
  tp.tile_begin = f.tile_begin;
  tp.tile_job = f.tile_job;
  tp.ctr = e.ctr;
  tp.k = k;
  tp.cap = P.cap;
  tp.tslots = P.tslots;
  tp.lf = P.lf;
  tp.wcap = P.wcap;
  tp.wts = P.wts;
  tp.wbytes = P.wbytes;
  tp.mode = 1;
  tp.out = out;
  tp.segchars = segc;
  tp.segchars_cap = segchars - 64;  // the line walk reads up to 7 bytes past a segment's chars
  tp.seg = seg;
  tp.xcount = uint32_t(X);
  tp.jobs = jd.tab;
  tp.jout = jd.jout;
  tp.jseg = jd.jseg;
  const uint32_t threads = e.tune.tile_threads ? e.tune.tile_threads : 512;
  r = run_tiles_k(e, tp, f, threads, nw);
  if (r) return r;
  cudaEventRecord(e.ev[3], e.stream);
  r = e.read_ctr();
  if (r) return r;
  if (e.h_ctr->err) return e.check_err(e.h_ctr);
  UC_CK(cudaMemcpyAsync(jd.jclosed, jd.jout, njobs * 8, cudaMemcpyDeviceToDevice, e.stream));
  uint32_t rounds = 0;
  StitchBufs sbuf{seg, Xr, segc, act0, act1, oncyc, hlen, lbase, longl, uint32_t(long_cap(e, X)), rcnt, hp};
  r = run_stitch(e, sbuf, X, Hp, k, nw, want_hec, RH, jd, out, rounds);
  if (r) return r;
  UC_CK(cudaGetLastError());
  cudaEventRecord(e.ev[4], e.stream);
  std::vector<unsigned long long> jo(njobs), jc(st ? njobs : 0);
  UC_CK(cudaMemcpyAsync(jo.data(), jd.jout, njobs * 8, cudaMemcpyDeviceToHost, e.stream));
  if (st) UC_CK(cudaMemcpyAsync(jc.data(), jd.jclosed, njobs * 8, cudaMemcpyDeviceToHost, e.stream));
  r = e.read_ctr();
  if (r) return r;
  if (e.h_ctr->err) return e.check_err(e.h_ctr);
  uint64_t total = 0;
  for (uint32_t j = 0; j < njobs; ++j) {
    if (jo[j] > J[j].ocap) return e.fail(UC_EINTERNAL, "output bound exceeded");
    if (out_off) out_off[j] = J[j].obase;
    if (out_len) out_len[j] = jo[j];
    total += jo[j];
  }
  if (st) {
    st->n_kmers = N;
    st->n_copies = copies;
    st->n_cross = X;
    st->n_tiles = e.h_ctr->ntiles;
    st->n_big_tiles = e.h_ctr->nbig;
    st->n_segments = Sp;
    st->n_cycles = e.h_ctr->cycles;
    st->closed_bytes = 0;
    for (uint32_t j = 0; j < njobs; ++j) st->closed_bytes += jc[j];
    st->seg_chars = e.h_ctr->seg_char_cursor;
    st->out_bytes = total;
    st->stitch_rounds = rounds;
    st->l_used = uint32_t(P.l_used);
    st->bucket_bits = P.bits;
    st->tile_capacity = P.cap;
    st->launches = e.launches;
    st->graph_nodes = e.graph_nodes;
    float a = 0, b = 0, c = 0, d = 0;
    cudaEventElapsedTime(&a, e.ev[0], e.ev[1]);
    cudaEventElapsedTime(&b, e.ev[1], e.ev[2]);
    cudaEventElapsedTime(&c, e.ev[2], e.ev[3]);
    cudaEventElapsedTime(&d, e.ev[3], e.ev[4]);
    st->ms_pack = a;
    st->ms_bucket = b;
    st->ms_tiles = c;
    st->ms_stitch = d;
    st->ms_total = a + b + c + d;
    if (e.tiles_timed) {
      cudaEventElapsedTime(&st->ms_tile_warp, e.ev[8], e.ev[9]);
      cudaEventElapsedTime(&st->ms_tile_block, e.ev[9], e.ev[5]);
    }
  }
  e.reset();
  return UC_OK;
}

// The streamed form of the fused path, for a job from host memory whose text
// and lines do not fit in device memory beside the working arrays.  The text
// goes to the device in chunks of whole lines, twice: the first pass counts
// the buckets (the 16-bit counts, taken again at 32 bits in a third pass if
// one wrapped), the second builds the bucketed copies (level 1 of the
// scatter per chunk, its cursors carried over; levels 2 and 3 once).  The
// tiles then run in groups of whole tiles; each group's closed lines go back
// to host memory before the next group, while the open segments stay on the
// device for the stitch, whose lines follow.  The device holds one chunk's
// text, keys and buckets, the copies' two scatter regions, the segment
// arrays and the output of one tile group; k-mer indices are 64-bit
// throughout (the reference's LARGE/HUGE widths, defs.h:30-42), cross
// indices and segment ids 31-bit.  Lines must be k chars + '\n' (the layout
// the chunks are cut on).  Unsorted output only.
int compact_streamed(Env& e, const char* h_text, size_t bytes, int k, int l, char* h_out, uint64_t cap,
                     uint64_t& out_bytes, uc_stats* st, uint64_t chunk_lines, uint64_t group_copies) {
  out_bytes = 0;
  if (k < 2 || k > 63) return e.fail(UC_EINPUT, "k must be in [2, 63]");
  if (l < 1 || l > 16 || l > k - 1) return e.fail(UC_EINPUT, "l must be in [1, min(16, k-1)]");
  if (e.sorted) return e.fail(UC_EINPUT, "the streamed path writes unsorted output");
  const int nw = (k <= 31) ? 1 : 2;
  const uint64_t stride = uint64_t(k) + 1;
  // count line (driver.cpp:296-304) and the fixed line layout
  size_t p = 0;
  while (p < bytes && (h_text[p] == ' ' || h_text[p] == '\t' || h_text[p] == '\r')) ++p;
  if (p >= bytes || h_text[p] < '0' || h_text[p] > '9') return e.fail(UC_EINPUT, "missing k-mer count header");
  uint64_t n = 0;
  while (p < bytes && h_text[p] >= '0' && h_text[p] <= '9') {
    n = n * 10 + uint64_t(h_text[p] - '0');
    if (n > (1ull << 40)) return e.fail(UC_EINPUT, "k-mer count too large");
    ++p;
  }
  while (p < bytes && h_text[p] != '\n') ++p;
  const uint64_t body = (p < bytes) ? p + 1 : bytes;
  uint64_t end = bytes;
  while (end > body && (h_text[end - 1] == '\n' || h_text[end - 1] == '\r')) --end;
  if (!((n == 0 && end == body) || (n > 0 && end - body == n * stride - 1)))
    return e.fail(UC_EINPUT, "the streamed path needs k chars + '\\n' per line and a matching count");
  e.reset();
  e.launches = 0;
  e.graph_nodes = 0;
  if (n == 0) return UC_OK;
  if (!chunk_lines) chunk_lines = 64ull << 20;
  if (!group_copies) group_copies = 256ull << 20;
  chunk_lines = std::min(chunk_lines, n);
  const Plan P = plan_buckets(e, n, 1, k, l);
  const size_t chunk_text = size_t(chunk_lines * stride + 64);
  int r = e.reserve(0, front_bytes(chunk_lines, nw, P.M, true) + chunk_text + 4096);
  if (r) return r;
  Front f{};
  r = take_front(e, chunk_lines, nw, P.M, true, f);
  if (r) return r;
  char* d_chunk = static_cast<char*>(e.take(0, chunk_text));
  if (!d_chunk) return e.fail(UC_EBUDGET, "front arena overflow");
  r = job_buffers(e, 1);
  if (r) return r;
  JobDev jd = job_dev(e, 1);
  UC_CK(cudaMemsetAsync(e.ctr, 0, sizeof(Counters), e.stream));
  UC_CK(cudaMemsetAsync(f.c16, 0, (P.M + 1) / 2 * 4, e.stream));
  UC_CK(cudaMemsetAsync(jd.jcross, 0, 4, e.stream));
  FuseArgs fz;
  fz.l = P.l_used;
  fz.seed = e.seed;
  fz.jb = P.jb;
  fz.b1 = f.b1;
  fz.b2 = f.b2;
  fz.M = P.M;
  // one chunk of lines to the device and packed (fz.counts / fz.jcross null:
  // buckets only)
  auto pack_chunk = [&](uint64_t c0, uint64_t cl, uint32_t* counts, uint32_t* jcross) -> int {
    const uint64_t src = body + c0 * stride;
    const uint64_t len = std::min<uint64_t>(cl * stride, uint64_t(bytes) - src);
    UC_CK(cudaMemcpyAsync(d_chunk, h_text + src, len, cudaMemcpyHostToDevice, e.stream));
    JobTab J{};
    J.text = reinterpret_cast<const uint8_t*>(d_chunk);
    J.tbytes = len;
    J.body = 0;
    J.end = cl * stride - 1;
    J.n = cl;
    J.fixed = 1;
    FuseArgs z = fz;
    z.counts = counts;
    z.jcross = jcross;
    const uint64_t nblocks = (cl + PACK_LINES - 1) / PACK_LINES;
    if (nw == 1) launch_pack<1>(e, jd.tab, &J, 1, nblocks, nullptr, k, f.keys, &z);
    else launch_pack<2>(e, jd.tab, &J, 1, nblocks, nullptr, k, f.keys, &z);
    UC_CK(cudaGetLastError());
    return UC_OK;
  };
  cudaEventRecord(e.ev[0], e.stream);
  for (uint64_t c0 = 0; c0 < n; c0 += chunk_lines) {
    r = pack_chunk(c0, std::min(chunk_lines, n - c0), f.c16, jd.jcross);
    if (r) return r;
  }
  r = e.read_ctr();
  if (r) return r;
  if (e.h_ctr->err) {
    if (e.h_ctr->err & ERR_LAYOUT) return e.fail(UC_EINPUT, "a k-mer line is shorter than k");
    return e.check_err(e.h_ctr);
  }
  cudaEventRecord(e.ev[1], e.stream);
  ++e.launches;
  k_widen16<<<grid_for(e, P.M, 256), 256, 0, e.stream>>>(f.c16, P.M, f.counts);
  uint64_t copies = 0;
  r = bucket_offsets(e, f, P.M, copies);
  if (r) return r;
  uint32_t xc = 0;
  UC_CK(cudaMemcpyAsync(&xc, jd.jcross, 4, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  if (copies != n + xc) {
    // a bucket holds 65536 copies or more: count again at 32 bits
    UC_CK(cudaMemsetAsync(f.counts, 0, P.M * 4, e.stream));
    for (uint64_t c0 = 0; c0 < n; c0 += chunk_lines) {
      const uint64_t cl = std::min(chunk_lines, n - c0);
      r = pack_chunk(c0, cl, nullptr, nullptr);
      if (r) return r;
      ++e.launches;
      k_count_buckets<<<grid_for(e, cl, 256), 256, 0, e.stream>>>(f.b1, f.b2, cl, f.counts);
    }
    r = bucket_offsets(e, f, P.M, copies);
    if (r) return r;
  }
  const uint64_t X = copies - n;
  const uint64_t Hp = X + 1;
  const uint64_t Sp = X + Hp;
  if (Sp >= 0x7FFFFFF0ull) return e.fail(UC_EINPUT, "too many cross-tile segments");
  const uint64_t segchars = Sp * uint64_t(k) + copies + 64;
  if (segchars > SEG_OFF_MASK) return e.fail(UC_EINPUT, "segment chars beyond the 40-bit offsets");
  // the tiles, grouped: whole tiles up to group_copies copies (a larger tile
  // alone); a group's closed lines fit its copies' lines
  r = plan_tiles(e, f, P);
  if (r) return r;
  r = e.read_ctr();
  if (r) return r;
  const uint32_t ntiles = e.h_ctr->ntiles;
  std::vector<unsigned long long> tb(size_t(ntiles) + 1);
  UC_CK(cudaMemcpyAsync(tb.data(), f.tile_begin, (size_t(ntiles) + 1) * 8, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  std::vector<uint32_t> groups{0};
  uint64_t gmax = 0;
  for (uint32_t t = 0; t < ntiles;) {
    const uint32_t g0 = t;
    do {
      ++t;
    } while (t < ntiles && tb[t + 1] - tb[g0] <= group_copies);
    groups.push_back(t);
    gmax = std::max<uint64_t>(gmax, tb[t] - tb[g0]);
  }
  const uint64_t gout = gmax * stride + 64;
  const uint64_t sout = segchars + Sp + 64;  // stitched lines: segment chars and a break each at most
  const uint32_t R = 64;
  const bool want_hec = e.tune.contract_method == UC_CONTRACT_HEC;
  const uint32_t RH = hec_rounds(e, Sp);
  r = e.reserve(1, back_bytes(e, copies, X, Sp, nw, k, want_hec) + gout + sout + 4096);
  if (r) return r;
  auto T64 = [&](uint64_t c) { return static_cast<unsigned long long*>(e.take(1, c * 8)); };
  auto T32 = [&](uint64_t c) { return static_cast<uint32_t*>(e.take(1, c * 4)); };
  char* region1 = static_cast<char*>(e.take(1, scatter_stage_bytes(copies, nw)));
  char* region2 = static_cast<char*>(e.take(1, scatter_stage_bytes(copies, nw)));
  SegRec* seg = static_cast<SegRec*>(e.take(1, Sp * sizeof(SegRec)));
  unsigned long long* Xr = T64(Sp);
  char* segc = static_cast<char*>(e.take(1, segchars));
  uint32_t* act0 = T32(Sp);
  uint32_t* act1 = T32(Sp);
  uint8_t* oncyc = static_cast<uint8_t*>(e.take(1, Sp));
  uint32_t* hlen = T32(Hp);
  unsigned long long* lbase = T64(Hp);
  uint32_t* longl = T32(long_cap(e, X));
  uint32_t* rcnt = T32(R);
  char* d_gout = static_cast<char*>(e.take(1, gout));
  char* d_sout = static_cast<char*>(e.take(1, sout));
  if (!d_sout) return e.fail(UC_EBUDGET, "back arena overflow");
  HecPool hp{};
  if (want_hec) {
    r = hec_take(e, Sp, RH, hp);
    if (r) return r;
  }
  UC_CK(cudaMemsetAsync(seg + X, 0, Hp * sizeof(SegRec), e.stream));
  UC_CK(cudaMemsetAsync(jd.jseg, 0, 4, e.stream));
  // the bucketed copies: level 1 chunk by chunk, then levels 2 and 3
  Scatter sc;
  r = scatter_begin(e, f, P, nw, region1, region2, copies, sc);
  if (r) return r;
  for (uint64_t c0 = 0; c0 < n; c0 += chunk_lines) {
    const uint64_t cl = std::min(chunk_lines, n - c0);
    r = pack_chunk(c0, cl, nullptr, nullptr);
    if (r) return r;
    r = scatter_l1(e, f, sc, f.keys, f.b1, f.b2, cl, 0);
    if (r) return r;
  }
  uint64_t* pkeys = nullptr;
  uint32_t* plink = nullptr;
  r = scatter_finish(e, f, sc, pkeys, plink);
  if (r) return r;
  cudaEventRecord(e.ev[2], e.stream);
  // one job whose region is a tile group's output buffer
  JobTab J{};
  J.n = n;
  J.obase = 0;
  J.ocap = gout;
  J.seg_base = 0;
  J.seg_cap = uint32_t(Hp);
  UC_CK(cudaMemcpyAsync(jd.tab, &J, sizeof(JobTab), cudaMemcpyHostToDevice, e.stream));
  TileParams tp{};
  tp.pkeys = pkeys;
  tp.plink = plink;
  tp.tile_begin = f.tile_begin;
  tp.tile_job = f.tile_job;
  tp.ctr = e.ctr;
  tp.k = k;
  tp.cap = P.cap;
  tp.tslots = P.tslots;
  tp.lf = P.lf;
  tp.wcap = P.wcap;
  tp.wts = P.wts;
  tp.wbytes = P.wbytes;
  tp.mode = 1;
  tp.out = d_gout;
  tp.segchars = segc;
  tp.segchars_cap = segchars - 64;  // the line walk reads up to 7 bytes past a segment's chars
  tp.seg = seg;
  tp.xcount = uint32_t(X);
  tp.jobs = jd.tab;
  tp.jout = jd.jout;
  tp.jseg = jd.jseg;
  const uint32_t threads = e.tune.tile_threads ? e.tune.tile_threads : 512;
  uint64_t closed = 0;
  float ms_tiles = 0;
  for (size_t g = 0; g + 1 < groups.size(); ++g) {
    // per group: the tier lists and their counters, the group's line cursor
    UC_CK(cudaMemsetAsync(&e.ctr->tile_next, 0, 4, e.stream));
    UC_CK(cudaMemsetAsync(&e.ctr->nbig, 0, 4, e.stream));
    UC_CK(cudaMemsetAsync(&e.ctr->nwarp, 0, 12, e.stream));  // nwarp, nblock, wtile_next
    UC_CK(cudaMemsetAsync(jd.jout, 0, 8, e.stream));
    r = classify_tiles(e, f, P, nw, groups[g], groups[g + 1]);
    if (r) return r;
    r = run_tiles_k(e, tp, f, threads, nw);
    if (r) return r;
    float a = 0;
    cudaEventElapsedTime(&a, e.ev[8], e.ev[5]);
    ms_tiles += a;
    unsigned long long gb = 0;
    UC_CK(cudaMemcpyAsync(&gb, jd.jout, 8, cudaMemcpyDeviceToHost, e.stream));
    r = e.read_ctr();
    if (r) return r;
    if (e.h_ctr->err) return e.check_err(e.h_ctr);
    if (closed + gb > cap) return e.fail(UC_EINPUT, "output buffer smaller than uc_output_bound");
    UC_CK(cudaMemcpyAsync(h_out + closed, d_gout, gb, cudaMemcpyDeviceToHost, e.stream));
    UC_CK(cudaStreamSynchronize(e.stream));
    closed += gb;
  }
  cudaEventRecord(e.ev[3], e.stream);
  // the stitch into its own buffer (no closed lines before it there)
  J.ocap = sout;
  UC_CK(cudaMemcpyAsync(jd.tab, &J, sizeof(JobTab), cudaMemcpyHostToDevice, e.stream));
  UC_CK(cudaMemsetAsync(jd.jclosed, 0, 8, e.stream));
  UC_CK(cudaMemsetAsync(jd.jout, 0, 8, e.stream));
  uint32_t rounds = 0;
  StitchBufs sbuf{seg, Xr, segc, act0, act1, oncyc, hlen, lbase, longl, uint32_t(long_cap(e, X)), rcnt, hp};
  r = run_stitch(e, sbuf, X, Hp, k, nw, want_hec, RH, jd, d_sout, rounds);
  if (r) return r;
  cudaEventRecord(e.ev[4], e.stream);
  unsigned long long sb = 0;
  UC_CK(cudaMemcpyAsync(&sb, jd.jout, 8, cudaMemcpyDeviceToHost, e.stream));
  r = e.read_ctr();
  if (r) return r;
  if (e.h_ctr->err) return e.check_err(e.h_ctr);
  if (sb > sout) return e.fail(UC_EINTERNAL, "output bound exceeded");
  if (closed + sb > cap) return e.fail(UC_EINPUT, "output buffer smaller than uc_output_bound");
  UC_CK(cudaMemcpyAsync(h_out + closed, d_sout, sb, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  out_bytes = closed + sb;
  if (st) {
    st->n_kmers = n;
    st->n_copies = copies;
    st->n_cross = X;
    st->n_tiles = ntiles;
    st->n_segments = Sp;
    st->n_cycles = e.h_ctr->cycles;
    st->closed_bytes = closed;
    st->seg_chars = e.h_ctr->seg_char_cursor;
    st->out_bytes = out_bytes;
    st->stitch_rounds = rounds;
    st->l_used = uint32_t(P.l_used);
    st->bucket_bits = P.bits;
    st->tile_capacity = P.cap;
    st->launches = e.launches;
    st->graph_nodes = e.graph_nodes;
    float a = 0, b = 0, d = 0;
    cudaEventElapsedTime(&a, e.ev[0], e.ev[1]);
    cudaEventElapsedTime(&b, e.ev[1], e.ev[2]);
    cudaEventElapsedTime(&d, e.ev[3], e.ev[4]);
    st->ms_pack = a;
    st->ms_bucket = b;
    st->ms_tiles = ms_tiles;
    st->ms_stitch = d;
    st->ms_total = a + b + ms_tiles + d;
  }
  e.reset();
  return UC_OK;
}

int compact_device(Env& e, const char* d_text, size_t bytes, int k, int l, char* out, uint64_t cap,
                   uint64_t& out_bytes, uc_stats* st) {
  uint64_t off = 0, len = 0;
  int r = compact_batch(e, 1, &d_text, &bytes, k, l, out, cap, &off, &len, st);
  out_bytes = len;
  if (r == UC_OK && e.sorted && len) r = sort_lines(e, out, len, k);
  return r;
}

// ============================================================ sorted output

// 0x80 in every byte of w that is a line break.
__device__ __forceinline__ uint32_t nl_bytes(uint32_t w) {
  const uint32_t z = w ^ 0x0A0A0A0Au;
  return ~(((z & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | z) & 0x80808080u;
}

// Line breaks in each 64 KiB chunk of out[0, n), 16-byte loads (out is
// 16-byte aligned; the tail of a chunk that ends inside a word is read
// byte by byte).
constexpr uint32_t NL_CHUNK = 1u << 16;
__global__ void __launch_bounds__(256) k_nl_count16(const char* __restrict__ out, uint64_t n,
                                                    uint32_t* __restrict__ cnt) {
  const uint64_t c0 = uint64_t(blockIdx.x) * NL_CHUNK;
  uint32_t acc = 0;
#pragma unroll 4
  for (uint32_t j = 0; j < NL_CHUNK / (16 * 256); ++j) {
    const uint64_t off = c0 + 16ull * (threadIdx.x + 256u * j);
    if (off + 16 <= n) {
      const uint4 v = __ldcs(reinterpret_cast<const uint4*>(out + off));
      acc += __popc(nl_bytes(v.x)) + __popc(nl_bytes(v.y)) + __popc(nl_bytes(v.z)) + __popc(nl_bytes(v.w));
    } else {
      for (uint64_t i = off; i < n && i < off + 16; ++i) acc += (out[i] == '\n');
    }
  }
  acc = __reduce_add_sync(0xFFFFFFFFu, acc);
  __shared__ uint32_t sh[8];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    cnt[blockIdx.x] = t;
  }
}

// Line starts: starts[0] = 0 and starts[r + 1] = 1 + the position of the
// r-th line break in out[0, n).  Each thread owns 256 contiguous bytes of its
// block's chunk: a count pass, a block scan, then a pass that writes.
__global__ void __launch_bounds__(256) k_nl_starts16(const char* __restrict__ out, uint64_t n,
                                                     const unsigned long long* __restrict__ coff,
                                                     unsigned long long* __restrict__ starts, uint64_t nlines) {
  const uint64_t t0 = uint64_t(blockIdx.x) * NL_CHUNK + 256ull * threadIdx.x;
  if (blockIdx.x == 0 && threadIdx.x == 0) starts[0] = 0;
  uint32_t mine = 0;
  for (uint32_t j = 0; j < 16; ++j) {
    const uint64_t off = t0 + 16ull * j;
    if (off + 16 <= n) {
      const uint4 v = *reinterpret_cast<const uint4*>(out + off);
      mine += __popc(nl_bytes(v.x)) + __popc(nl_bytes(v.y)) + __popc(nl_bytes(v.z)) + __popc(nl_bytes(v.w));
    } else {
      for (uint64_t i = off; i < n && i < off + 16; ++i) mine += (out[i] == '\n');
    }
  }
  __shared__ uint32_t sc[33];
  uint32_t tot;
  uint64_t r = coff[blockIdx.x] + block_excl_scan(mine, sc, &tot);
  for (uint32_t j = 0; j < 16; ++j) {
    const uint64_t off = t0 + 16ull * j;
    if (off + 16 <= n) {
      const uint4 v = *reinterpret_cast<const uint4*>(out + off);
      const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t m = nl_bytes(wv[q]);
        while (m) {
          const int b = (__ffs(m) - 1) >> 3;
          m &= m - 1;
          ++r;
          if (r < nlines) starts[r] = off + 4u * q + b + 1;
        }
      }
    } else {
      for (uint64_t i = off; i < n && i < off + 16; ++i) {
        if (out[i] == '\n') {
          ++r;
          if (r < nlines) starts[r] = i + 1;
        }
      }
    }
  }
}

// Line keys: each line's first k chars, packed big-endian (first char in the
// top bits of hi, chars 32.. in lo), so that numeric order is byte order.
// Every k-mer begins at most one line, so these keys order the lines
// completely.  The k chars are read as 4-byte words
// (funnel-shifted to the line's byte offset) and converted 4 codes at a time;
// the little-endian codes are then reversed into big-endian keys.  Reads up
// to 12 bytes past a line's k chars (inside the output buffer's bound).
__global__ void k_line_keys4(const char* __restrict__ out, const unsigned long long* __restrict__ starts,
                             uint64_t L, int k, unsigned long long* __restrict__ khi,
                             unsigned long long* __restrict__ klo, uint32_t* __restrict__ idx) {
  const int nw = (k + 3) / 4;
  const uint64_t m0 = (k >= 32) ? ~0ull : ((1ull << (2 * k)) - 1ull);
  const uint64_t m1 = (k <= 32) ? 0ull : ((k - 32 >= 32) ? ~0ull : ((1ull << (2 * (k - 32))) - 1ull));
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < L; j += uint64_t(gridDim.x) * blockDim.x) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(out + starts[j]);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    const uint32_t sh = 8u * uint32_t(a & 3u);
    uint64_t w0 = 0, w1 = 0;
    uint32_t cur = w[0];
    for (int q = 0; q < nw; ++q) {
      const uint32_t nxt = w[q + 1];
      const uint32_t x = __funnelshift_r(cur, nxt, sh);
      cur = nxt;
      const uint64_t g = gather_codes(((x >> 1) ^ (x >> 2)) & 0x03030303u);
      if (q < 8) w0 |= g << (8 * q);
      else w1 |= g << (8 * (q - 8));
    }
    khi[j] = rev2(w0 & m0);
    klo[j] = rev2(w1 & m1);
    idx[j] = uint32_t(j);
  }
}

__global__ void k_gather_u64(const unsigned long long* __restrict__ src, const uint32_t* __restrict__ idx,
                             uint64_t L, unsigned long long* __restrict__ dst) {
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < L; j += uint64_t(gridDim.x) * blockDim.x)
    dst[j] = src[idx[j]];
}

__global__ void k_sorted_len(const unsigned long long* __restrict__ starts, const uint32_t* __restrict__ idx,
                             uint64_t L, uint32_t* __restrict__ len) {
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < L; j += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t i = idx[j];
    len[j] = uint32_t(starts[i + 1] - starts[i]);
  }
}

// Lines to their sorted places: a warp resolves 32 lines, then copies them.
__global__ void k_line_copy(const char* __restrict__ src, const unsigned long long* __restrict__ starts,
                            const uint32_t* __restrict__ idx, const unsigned long long* __restrict__ dsto,
                            uint64_t L, char* __restrict__ dst) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t base = warp * 32u; base < L; base += nwarps * 32u) {
    const uint64_t j = base + uint64_t(lane);
    uint64_t so = 0, d = 0;
    uint32_t m = 0;
    if (j < L) {
      const uint32_t i = idx[j];
      so = starts[i];
      m = uint32_t(starts[i + 1] - so);
      d = dsto[j];
    }
    uint32_t todo = __ballot_sync(0xFFFFFFFFu, j < L);
    while (todo) {
      const int q = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint64_t a = __shfl_sync(0xFFFFFFFFu, so, q);
      const uint64_t b = __shfl_sync(0xFFFFFFFFu, d, q);
      const uint32_t n = __shfl_sync(0xFFFFFFFFu, m, q);
      for (uint32_t x = lane; x < n; x += 32) dst[b + x] = src[a + x];
    }
  }
}

int sort_lines(Env& e, char* out, uint64_t bytes, int k) {
  if (bytes == 0) return UC_OK;
  e.reset();
  const uint32_t chunk = NL_CHUNK;
  const uint64_t nchunks = std::max<uint64_t>(1, (bytes - 1 + chunk - 1) / chunk);
  const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15u) == 0;  // else byte-wise line scan
  // lines end with '\n'; the last one at bytes - 1
  const uint64_t Lmax = bytes / uint64_t(k + 1) + 1;
  size_t cub_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, static_cast<const unsigned long long*>(nullptr),
                                  static_cast<unsigned long long*>(nullptr), static_cast<const uint32_t*>(nullptr),
                                  static_cast<uint32_t*>(nullptr), int(Lmax), 0, 64, e.stream);
  size_t need = 0;
  auto add = [&](size_t b) { need += (b + 255) & ~size_t(255); };
  add(bytes); add(nchunks * 4); add((nchunks + 1) * 8); add(scan_tmp_elems(nchunks) * 8);
  add((Lmax + 1) * 8);                         // starts
  add(Lmax * 8); add(Lmax * 8); add(Lmax * 8); // khi, klo, sorted keys
  add(Lmax * 4); add(Lmax * 4);                // idx, sorted idx
  add(Lmax * 4); add((Lmax + 1) * 8); add(scan_tmp_elems(Lmax) * 8);
  add(cub_bytes);
  int r = e.reserve(1, need);
  if (r) return r;
  char* tmp = static_cast<char*>(e.take(1, bytes));
  uint32_t* cnt = static_cast<uint32_t*>(e.take(1, nchunks * 4));
  auto T64 = [&](uint64_t c) { return static_cast<unsigned long long*>(e.take(1, c * 8)); };
  auto T32 = [&](uint64_t c) { return static_cast<uint32_t*>(e.take(1, c * 4)); };
  unsigned long long* coff = T64(nchunks + 1);
  unsigned long long* ctmp = T64(scan_tmp_elems(nchunks));
  unsigned long long* starts = T64(Lmax + 1);
  unsigned long long* khi = T64(Lmax);
  unsigned long long* klo = T64(Lmax);
  unsigned long long* ks = T64(Lmax);
  uint32_t* idx = T32(Lmax);
  uint32_t* idx2 = T32(Lmax);
  uint32_t* len = T32(Lmax);
  unsigned long long* dsto = T64(Lmax + 1);
  unsigned long long* stmp = T64(scan_tmp_elems(Lmax));
  void* cub_tmp = e.take(1, cub_bytes);
  if (!cub_tmp) return e.fail(UC_EBUDGET, "arena overflow (sorted output)");
  const uint8_t* ob = reinterpret_cast<const uint8_t*>(out);
  e.launches += 1 + 6 + 1;
  if (aligned) k_nl_count16<<<unsigned(nchunks), 256, 0, e.stream>>>(out, bytes - 1, cnt);
  else k_count_nl<<<unsigned(nchunks), 256, 0, e.stream>>>(ob, 0, bytes - 1, cnt, chunk);
  scan_excl<uint32_t, unsigned long long>(cnt, nchunks, coff, ctmp, e.stream);
  unsigned long long nl = 0;
  UC_CK(cudaMemcpyAsync(&nl, coff + nchunks, 8, cudaMemcpyDeviceToHost, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  const uint64_t L = nl + 1;
  if (L > Lmax || L >= 0x7FFFFFFFull) return e.fail(UC_EINTERNAL, "line count of the output out of range");
  if (aligned) k_nl_starts16<<<unsigned(nchunks), 256, 0, e.stream>>>(out, bytes - 1, coff, starts, L);
  else k_write_starts<<<unsigned(nchunks), 256, 0, e.stream>>>(ob, 0, bytes - 1, coff, chunk, starts, L);
  UC_CK(cudaMemcpyAsync(starts + L, &bytes, 8, cudaMemcpyHostToDevice, e.stream));
  const int g = grid_for(e, L, 256);
  e.launches += 1;
  k_line_keys4<<<g, 256, 0, e.stream>>>(out, starts, L, k, khi, klo, idx);
  // least significant part first; radix sort is stable
  uint32_t* order = idx;
  if (k > 32) {
    UC_CK(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_bytes, klo, ks, idx, idx2, int(L), 128 - 2 * k, 64,
                                          e.stream));
    ++e.launches;
    k_gather_u64<<<g, 256, 0, e.stream>>>(khi, idx2, L, klo);
    UC_CK(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_bytes, klo, ks, idx2, idx, int(L), 0, 64, e.stream));
    order = idx;
  } else {
    UC_CK(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_bytes, khi, ks, idx, idx2, int(L), 64 - 2 * k, 64,
                                          e.stream));
    order = idx2;
  }
  e.launches += 2 + 6;
  k_sorted_len<<<g, 256, 0, e.stream>>>(starts, order, L, len);
  scan_excl<uint32_t, unsigned long long>(len, L, dsto, stmp, e.stream);
  k_line_copy<<<g, 256, 0, e.stream>>>(out, starts, order, dsto, L, tmp);
  UC_CK(cudaGetLastError());
  UC_CK(cudaMemcpyAsync(out, tmp, bytes, cudaMemcpyDeviceToDevice, e.stream));
  UC_CK(cudaStreamSynchronize(e.stream));
  e.reset();
  return UC_OK;
}

}  // namespace uc
