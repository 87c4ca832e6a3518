// uc_common.cuh — key layout, minimizer priority and small device helpers
// shared by the unitig-compaction kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace uc {

constexpr uint32_t NONE = 0xFFFFFFFFu;
// Role bits live in the two top bits of a key's last 64-bit word; a key uses
// at most 62 bits of that word (k <= 31 in one word, k <= 63 in two).
constexpr uint64_t ROLE_P = 1ull << 63;  // copy sits in its prefix-minimizer bucket
constexpr uint64_t ROLE_S = 1ull << 62;  // copy sits in its suffix-minimizer bucket
constexpr uint64_t ROLE_MASK = ROLE_P | ROLE_S;

// device error word bits
enum : uint32_t {
  ERR_LINE = 1u,      // a k-mer line shorter than k
  ERR_COUNT = 2u,     // header count differs from the line count
  ERR_TIMEOUT = 4u,   // a bounded device wait gave up
  ERR_CAPACITY = 8u,  // an output or scratch bound was exceeded
  ERR_LAYOUT = 16u,   // fixed-width line layout did not hold (fast path)
  ERR_INTERNAL = 32u,
};

template <int NW>
struct Key {
  uint64_t w[NW];
};

template <int NW>
__device__ __forceinline__ Key<NW> ld_key(const uint64_t* p, size_t i) {
  Key<NW> k;
  if constexpr (NW == 1) {
    k.w[0] = p[i];
  } else {
    const ulonglong2 v = reinterpret_cast<const ulonglong2*>(p)[i];
    k.w[0] = v.x;
    k.w[1] = v.y;
  }
  return k;
}

template <int NW>
__device__ __forceinline__ void st_key(uint64_t* p, size_t i, const Key<NW>& k) {
  if constexpr (NW == 1) {
    p[i] = k.w[0];
  } else {
    reinterpret_cast<ulonglong2*>(p)[i] = make_ulonglong2(k.w[0], k.w[1]);
  }
}

template <int NW>
__device__ __forceinline__ uint64_t roles(const Key<NW>& k) {
  return k.w[NW - 1] & ROLE_MASK;
}

template <int NW>
__device__ __forceinline__ Key<NW> strip(Key<NW> k) {
  k.w[NW - 1] &= ~ROLE_MASK;
  return k;
}

// Mask keeping the low 2*(k-1) bits: the (k-1)-prefix.
struct PrefMask {
  uint64_t m0, m1;
};
__host__ __device__ inline PrefMask pref_mask(int k) {
  const int bits = 2 * (k - 1);
  PrefMask m;
  if (bits >= 64) {
    m.m0 = ~0ull;
    m.m1 = (bits == 64) ? 0ull : ((1ull << (bits - 64)) - 1ull);
  } else {
    m.m0 = (1ull << bits) - 1ull;
    m.m1 = 0ull;
  }
  return m;
}

template <int NW>
__device__ __forceinline__ Key<NW> prefix_of(const Key<NW>& x, const PrefMask& m) {
  Key<NW> r;
  r.w[0] = x.w[0] & m.m0;
  if constexpr (NW == 2) r.w[1] = x.w[1] & m.m1;
  return r;
}

// chars 1..k-1 moved down to position 0 (role bits fall outside the mask)
template <int NW>
__device__ __forceinline__ Key<NW> suffix_of(const Key<NW>& x, const PrefMask& m) {
  Key<NW> r;
  if constexpr (NW == 1) {
    r.w[0] = (x.w[0] >> 2) & m.m0;
  } else {
    r.w[0] = ((x.w[0] >> 2) | (x.w[1] << 62)) & m.m0;
    r.w[1] = (x.w[1] >> 2) & m.m1;
  }
  return r;
}

template <int NW>
__device__ __forceinline__ bool key_eq(const Key<NW>& a, const Key<NW>& b) {
  bool e = a.w[0] == b.w[0];
  if constexpr (NW == 2) e = e && (a.w[1] == b.w[1]);
  return e;
}

// numeric order of the packed value (last word most significant), roles ignored
template <int NW>
__device__ __forceinline__ bool key_lt(const Key<NW>& a, const Key<NW>& b) {
  if constexpr (NW == 1) {
    return (a.w[0] & ~ROLE_MASK) < (b.w[0] & ~ROLE_MASK);
  } else {
    const uint64_t ah = a.w[1] & ~ROLE_MASK, bh = b.w[1] & ~ROLE_MASK;
    return ah < bh || (ah == bh && a.w[0] < b.w[0]);
  }
}

// Slot hash of a (k-1)-mer for the tile tables (at most 2^15 slots): the
// high half of a multiplicative (Fibonacci) hash, which every key bit reaches.
template <int NW>
__device__ __forceinline__ uint32_t key_hash(const Key<NW>& p) {
  uint64_t h = p.w[0] * 0x9E3779B97F4A7C15ull;
  if constexpr (NW == 2) h += p.w[1] * 0xC2B2AE3D27D4EB4Full;
  return static_cast<uint32_t>(h >> 32);
}

// 2-bit code of char x of a packed key
template <int NW>
__device__ __forceinline__ uint32_t key_char(const Key<NW>& x, int i) {
  if constexpr (NW == 1) {
    return static_cast<uint32_t>(x.w[0] >> (2 * i)) & 3u;
  } else {
    return static_cast<uint32_t>((i < 32 ? x.w[0] >> (2 * i) : x.w[1] >> (2 * (i - 32)))) & 3u;
  }
}

__device__ __forceinline__ char acgt(uint32_t c) {
  return static_cast<char>(0x54474341u >> (8 * c));  // "ACGT"
}

// Seeded bijection of [0, 4^l): the l-mer priority.  The reference draws a
// random permutation of the 4^l l-mers (generate_permutation,
// driver.cpp:356-402); any permutation gives the same unitigs.  Multiplying
// by an odd number and adding are each invertible modulo 4^l; both come from
// the seed.
__host__ __device__ __forceinline__ uint32_t lmer_mult(uint64_t seed) {
  return (0x9E3779B1u ^ (static_cast<uint32_t>(seed) << 1)) | 1u;
}
__host__ __device__ __forceinline__ uint32_t lmer_priority(uint32_t x, int l, uint64_t seed) {
  const uint32_t b = 2u * static_cast<uint32_t>(l);
  const uint32_t mask = (b >= 32u) ? 0xFFFFFFFFu : ((1u << b) - 1u);
  return (x * lmer_mult(seed) + static_cast<uint32_t>(seed >> 32)) & mask;
}

// Bucket of a minimizer priority.  Any function of the minimizer keeps every
// (k-1)-overlap inside one bucket; this one spreads the small-valued
// minimizers (a minimum is biased low) evenly over 2^bits buckets.
__host__ __device__ __forceinline__ uint32_t bucket_of(uint32_t pr, uint32_t bits) {
  uint32_t h = pr * 0x9E3779B1u;
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return bits ? (h >> (32u - bits)) : 0u;
}

// ASCII of the 4 codes in the low 8 bits of c (first char in the low byte):
// spread the 2-bit codes into nibbles, then select bytes of "ACGT".
__device__ __forceinline__ uint32_t ascii4(uint32_t c) {
  uint32_t x = (c | (c << 4)) & 0x0F0Fu;
  x = (x | (x << 2)) & 0x3333u;
  return __byte_perm(0x54474341u, 0u, x);
}

// codes of chars ch..ch+3 of a packed key in the low 8 bits (chars past the
// key read as 0)
template <int NW>
__device__ __forceinline__ uint32_t codes4(const Key<NW>& x, int ch) {
  if constexpr (NW == 1) {
    return uint32_t(x.w[0] >> (2 * ch)) & 0xFFu;
  } else {
    const uint64_t v = (ch < 32) ? ((x.w[0] >> (2 * ch)) | (ch > 0 ? (x.w[1] << (64 - 2 * ch)) : 0ull))
                                 : (x.w[1] >> (2 * (ch - 32)));
    return uint32_t(v) & 0xFFu;
  }
}

// Write the k chars of a packed key at dst (any alignment): byte stores up
// to the first aligned word, then the key moved down by those chars (one
// shift) and aligned 32-bit stores from constant shifts, then byte stores
// for the rest.
template <int NW>
__device__ __forceinline__ void spell_key(char* dst, const Key<NW>& x, int k) {
  const int ch0 = min(k, int((4u - uint32_t(reinterpret_cast<uintptr_t>(dst) & 3u)) & 3u));
  Key<NW> y = x;
  if (ch0) {
    const uint32_t a = ascii4(codes4(x, 0));
    for (int i = 0; i < ch0; ++i) dst[i] = char(a >> (8 * i));
    if constexpr (NW == 1) {
      y.w[0] = x.w[0] >> (2 * ch0);
    } else {
      y.w[0] = (x.w[0] >> (2 * ch0)) | (x.w[1] << (64 - 2 * ch0));
      y.w[1] = x.w[1] >> (2 * ch0);
    }
  }
  const int rest = k - ch0;
  const int nw4 = rest >> 2;
  uint32_t* d = reinterpret_cast<uint32_t*>(dst + ch0);
#pragma unroll
  for (int w = 0; w < 8 * NW; ++w)
    if (w < nw4) d[w] = ascii4(codes4(y, 4 * w));
  if (rest & 3) {
    const uint32_t a = ascii4(codes4(y, 4 * nw4));
    for (int i = 0; i < (rest & 3); ++i) dst[ch0 + 4 * nw4 + i] = char(a >> (8 * i));
  }
}

// reverse the order of the 2-bit groups of a 64-bit word
__device__ __forceinline__ uint64_t rev2(uint64_t x) {
  x = __brevll(x);
  return ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
}

// Prefix (l1) and suffix (l2) minimizer priorities of one k-mer
// (get_double_lmin, lmin_buckets.h:67-94): l-mer ids are big-endian (first
// char in the top bits); l1 covers the l-mers inside chars [0, k-1), l2 the
// ones inside chars [1, k).  Requires 1 <= l <= min(16, k-1).
//
// Without a table the priority is computed in the top 2l bits of a 32-bit
// word: (id * m + a) << (32 - 2l) equals id * (m << (32 - 2l)) + (a << ...)
// modulo 2^32, and chars left of the l-mer in the id's upper bits drop out of
// that product, so each l-mer costs one shift, one multiply-add and one min.
template <int NW>
__device__ __forceinline__ void lmins(const Key<NW>& key, int k, int l, uint64_t seed,
                                      const uint32_t* __restrict__ table, uint32_t& l1,
                                      uint32_t& l2) {
  uint64_t hi, lo;
  if constexpr (NW == 1) {
    hi = rev2(key.w[0] & ~ROLE_MASK);
    lo = 0;
  } else {
    hi = rev2(key.w[0]);
    lo = rev2(key.w[1] & ~ROLE_MASK);
  }
  const int w = k - l + 1;  // l-mers in the k-mer (>= 2)
  if (table == nullptr) {
    const uint32_t ps = 32u - 2u * uint32_t(l);
    const uint32_t m = lmer_mult(seed) << ps, a = static_cast<uint32_t>(seed >> 32) << ps;
    uint32_t first, mid = 0xFFFFFFFFu, last;
    if constexpr (NW == 1) {
      // l-mer p sits in bits [64 - 2p - 2l, 64 - 2p) of hi
      int s = 64 - 2 * l;
      first = static_cast<uint32_t>(hi >> s) * m + a;
#pragma unroll
      for (int p = 1; p < w - 1; ++p) {
        s -= 2;
        mid = min(mid, static_cast<uint32_t>(hi >> s) * m + a);
      }
      last = static_cast<uint32_t>(hi >> (s - 2)) * m + a;
    } else {
      const int s = 64 - 2 * l;
      first = static_cast<uint32_t>(hi >> s) * m + a;
#pragma unroll
      for (int p = 1; p < w - 1; ++p) {
        hi = (hi << 2) | (lo >> 62);
        lo <<= 2;
        mid = min(mid, static_cast<uint32_t>(hi >> s) * m + a);
      }
      hi = (hi << 2) | (lo >> 62);
      last = static_cast<uint32_t>(hi >> s) * m + a;
    }
    l1 = min(first, mid) >> ps;
    l2 = min(mid, last) >> ps;
    return;
  }
  const int sh = 64 - 2 * l;
  auto pri = [&](uint32_t id) { return __ldg(table + id); };
  const uint32_t first = pri(static_cast<uint32_t>(hi >> sh));
  uint32_t mid = NONE;
  for (int p = 1; p < w - 1; ++p) {
    hi = (hi << 2) | (lo >> 62);
    lo <<= 2;
    mid = min(mid, pri(static_cast<uint32_t>(hi >> sh)));
  }
  hi = (hi << 2) | (lo >> 62);
  const uint32_t last = pri(static_cast<uint32_t>(hi >> sh));
  l1 = min(first, mid);
  l2 = min(mid, last);
}

// ---- warp / block helpers ---------------------------------------------

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Exclusive block scan; every thread of the block must call it.  scratch
// holds at least 33 values.  Returns the exclusive prefix, total in *total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* scratch, T* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  T inc = warp_incl_scan(v);
  if (lane == 31) scratch[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T s = (lane < nw) ? scratch[lane] : T(0);
    T si = warp_incl_scan(s);
    if (lane < nw) scratch[lane] = si - s;
    if (lane == nw - 1) scratch[32] = si;
  }
  __syncthreads();
  T r = scratch[wid] + inc - v;
  *total = scratch[32];
  __syncthreads();
  return r;
}

}  // namespace uc
