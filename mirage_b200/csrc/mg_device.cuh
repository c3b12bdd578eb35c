// Device-side data structures and group-cooperative primitives of the classification path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/mirage_b200.h"

namespace mg {

// Domain of the relative-score logarithm patched to the host libm's logf: [1, 2^20).
constexpr uint32_t kLogLoBits = 0x3F800000u;  // 1.0f
constexpr uint32_t kLogHiBits = 0x49800000u;  // 2^20
constexpr uint32_t kLogDomain = kLogHiBits - kLogLoBits;

// Hash slots: one 64-byte slot per 28-bit hash, 64-byte aligned. Word 0 holds the bucket's
// posting count, word 1 its first posting in post, words 2-15 its first kSlotPosts postings as
// (refID, position) pairs: a seed whose bucket holds at most kSlotPosts postings gets all of them
// from one 64-byte block instead of a directory sector and then a dependent posting sector.
constexpr int kSlotPosts = 7;
constexpr int kSlotVecs = 4;  // uint4 per slot

// HBM-resident index (all pointers device memory).
struct DevIndex {
  const uint32_t* dir;      // 2^28 + 1 bucket offsets into post (CSR over the 28-bit hash)
  const uint2* post;        // (refID, position) per posting, bucket order
  const uint4* slots;       // 2^28 hash slots (kSlotVecs uint4 each), or nullptr: probes read dir
                            // and post
  const uint8_t* bases;     // reference sequence block
  const uint64_t* ref_off;  // offset of each reference in bases
  const uint32_t* ref_len;
  uint32_t n_refs;
  uint32_t empty_hash;      // hash present with no postings (0xFFFFFFFF: none)
  int k, step, hlen;
  const uint32_t* logx_bitmap;  // kLogDomain bits: 1 where host logf differs from the device log
  const uint32_t* logx_keys;    // sorted float bits of those inputs
  const float* logx_vals;       // host logf at those inputs
  uint32_t n_logx;
  const float* log_den;         // [lm] logf(scoreMax(lm)) for lm in [0, 65536): the relative
                                // score's denominator, which depends only on min(qlen, rlen)
};

// Error word bits set by kernels (first error kept by the host).
enum : int {
  kErrBadInput = 1,   // read byte without a reverse complement
  kErrLimit = 2,      // read beyond every tier's capacity
  kErrOutput = 4,     // candidate buffer too small
  kErrLogRange = 8,   // relative-score log outside the patched domain
  kErrArena = 16,     // staging arena too small for the reads with more than kSlots candidates
  kErrInternal = 32,  // a bounded device loop reached its bound (an invariant failed)
  kErrHuge = 64,      // a read needs a larger oversize-tier workspace (the host grows it and reruns)
};

struct BatchDev {
  uint64_t n;
  const uint64_t* offs;
  const uint8_t* bases;
  mg_read_result* reads;
  mg_candidate* cands;
  uint64_t cand_cap;
  unsigned long long* n_cands;   // output cursor
  int* err;                      // OR of kErr* bits
  unsigned int* work;            // work-stealing cursor for the dual-strand warp tier
  uint32_t* ovf0;                // reads handed to the second dual-strand tier
  unsigned int* n_ovf0;
  unsigned int* work0b;          // cursor over ovf0
  uint32_t* ovf0b;               // reads handed to the general warp tier
  unsigned int* n_ovf0b;
  unsigned int* work1;           // cursor over ovf0b
  uint32_t* ovf1;                // reads handed to the block tier
  unsigned int* n_ovf1;
  unsigned int* work2;           // cursor over ovf1
  uint32_t* ovf2;                // reads handed to the global-memory tier
  unsigned int* n_ovf2;
  unsigned int* work3;           // cursor over ovf2
};

// ------------------------------------------------------------------------------ helpers

__device__ __forceinline__ uint32_t hash28_dev(const uint8_t* p, int len) {
  uint32_t h = 2166136261u;
  if (len == 17) {  // the window of the default k (31), unrolled
#pragma unroll
    for (int i = 0; i < 17; i++) h = (h * 16777619u) ^ p[i];
    return ((h >> 28) ^ h) & 0x0FFFFFFFu;
  }
  for (int i = 0; i < len; i++) h = (h * 16777619u) ^ p[i];
  return ((h >> 28) ^ h) & 0x0FFFFFFFu;
}

// Sequences::SequenceToUpperCase (Sequences.cpp:43-55): signed char above 96 loses 32.
__device__ __forceinline__ uint8_t upper_dev(uint8_t c) {
  return ((int8_t)c > 96) ? (uint8_t)(c - 32) : c;
}

__device__ __forceinline__ uint8_t complement_dev(uint8_t c) {
  switch (c) {
    case 'A': return 'T'; case 'T': return 'A'; case 'U': return 'A';
    case 'G': return 'C'; case 'C': return 'G'; case 'Y': return 'R'; case 'R': return 'Y';
    case 'S': return 'S'; case 'W': return 'W'; case 'K': return 'M'; case 'M': return 'K';
    case 'B': return 'V'; case 'D': return 'H'; case 'H': return 'D'; case 'V': return 'B';
    case 'N': return 'N'; case '-': return '-'; case '~': return '~';
    default: return 0;
  }
}

// The device logarithm: CUDA's double-precision log rounded once to float.
__device__ __forceinline__ float log_dev_raw(float x) { return __double2float_rn(log((double)x)); }

// logf exactly as the host libm computes it, for x in [1, 2^20): the device value, replaced
// by the host's where the two were found to differ when the index was opened. Out of line: called
// once per scored candidate, and keeping its double-precision log out of the warp tier's hot
// code measurably reduces instruction-fetch stalls there.
static __device__ __noinline__ float ref_logf(const DevIndex& ix, float x, int* err) {
  const uint32_t b = __float_as_uint(x);
  const bool in = b >= kLogLoBits && b < kLogHiBits;
  const uint32_t r = in ? b - kLogLoBits : 0u;
  const uint32_t word = __ldg(ix.logx_bitmap + (r >> 5));  // in flight while the logarithm runs
  const float v = log_dev_raw(x);
  if (!in) {
    *err |= kErrLogRange;
    return v;
  }
  if (word & (1u << (r & 31))) {
    uint32_t lo = 0, hi = ix.n_logx;
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (ix.logx_keys[mid] < b) lo = mid + 1; else hi = mid;
    }
    return ix.logx_vals[lo];
  }
  return v;
}

// MatrixResult::GetRelativeScore (MatrixResult.cpp:21-29) with explicit IEEE roundings:
// lenMax float; scoreMax in double then float; score + 1 in float; logf / logf in float.
static __device__ __noinline__ float relative_score(const DevIndex& ix, float qlen, float rlen, float score, int* err) {
  const float len_max = qlen < rlen ? qlen : rlen;
  const double lm = (double)len_max;
  const float score_max = __double2float_rn(__dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(lm, __dadd_rn(lm, 1.0)), 2.0), lm), 1.0));
  const float s1 = __fadd_rn(score, 1.0f);
  return __fdiv_rn(ref_logf(ix, s1, err), ref_logf(ix, score_max, err));
}

// relative_score for integer lengths, the denominator read from ix.log_den (filled at open with
// the same arithmetic as relative_score, so the result is the same float). min(qlen, rlen) equals
// the float min of relative_score: qlen < 2^16 is exact, and an rlen that float rounds is > qlen.
__device__ __forceinline__ float relative_score_tab(const DevIndex& ix, uint32_t qlen, uint32_t rlen, float score,
                                                    int* err) {
  const uint32_t lm = qlen < rlen ? qlen : rlen;
  if (lm == 0 || lm > 0xFFFFu) return relative_score(ix, __uint2float_rn(qlen), __uint2float_rn(rlen), score, err);
  const float s1 = __fadd_rn(score, 1.0f);
  return __fdiv_rn(ref_logf(ix, s1, err), __ldg(ix.log_den + lm));
}

// CalculateScore's final arithmetic (MatrixCPU.cpp:209-212).
__device__ __forceinline__ void final_score(uint64_t sum_r, uint64_t sum_c, uint32_t hits, uint32_t L,
                                            float* score_out, float* pct_out) {
  const float score = __fdiv_rn(__ull2float_rn(sum_r), __ull2float_rn(sum_c));
  const double pctd = __dmul_rn(__ddiv_rn(100.0, (double)__uint2float_rn(L)), (double)__uint2float_rn(hits));
  const float pct = __double2float_rn(pctd);
  *pct_out = pct;
  *score_out = __double2float_rn(__dmul_rn(__ddiv_rn((double)score, 100.0), (double)pct));
}

// ------------------------------------------------------------------------------ groups
// A "group" is either one warp (G == 32, several groups per block) or a whole block (G > 32).

template <int G>
struct Grp {
  static __device__ __forceinline__ int tid() { return G == 32 ? (threadIdx.x & 31) : threadIdx.x; }
  static __device__ __forceinline__ void sync() {
    if (G == 32) __syncwarp(); else __syncthreads();
  }
};

// Scratch for group reductions: G/32 words (+1) per group, in shared memory.
template <int G>
struct RedTmp {
  uint64_t v[G / 32 + 1];
  uint32_t f[G / 32 + 1];
};

template <int G>
__device__ __forceinline__ uint64_t grp_max_u64(uint64_t v, RedTmp<G>* t) {
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  if (G == 32) return v;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) t->v[wid] = v;
  __syncthreads();
  uint64_t r = 0;
  for (int i = 0; i < G / 32; i++) r = t->v[i] > r ? t->v[i] : r;
  __syncthreads();
  return r;
}

template <int G>
__device__ __forceinline__ uint64_t grp_sum_u64(uint64_t v, RedTmp<G>* t) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (G == 32) return v;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) t->v[wid] = v;
  __syncthreads();
  uint64_t r = 0;
  for (int i = 0; i < G / 32; i++) r += t->v[i];
  __syncthreads();
  return r;
}

// Exclusive prefix sum over the group's threads; *total receives the sum.
template <int G>
__device__ __forceinline__ uint32_t grp_excl_sum(uint32_t v, RedTmp<G>* t, uint32_t* total) {
  const int lane = threadIdx.x & 31;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (G == 32) {
    *total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
  }
  const int wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 31) t->f[wid] = x;
  __syncthreads();
  uint32_t base = 0, tot = 0;
  for (int i = 0; i < G / 32; i++) {
    if (i < wid) base += t->f[i];
    tot += t->f[i];
  }
  __syncthreads();
  *total = tot;
  return base + x - v;
}

// Exclusive segmented scan across the group's threads (thread order) of (value, head)
// pairs: the result for a thread combines the values of all earlier threads back to the last
// head among them. op must have identity 0 on the values used (add, max of unsigned).
template <int G, class Op>
__device__ __forceinline__ uint32_t grp_seg_scan_excl(uint32_t r, uint32_t f, RedTmp<G>* t, Op op) {
  const int lane = threadIdx.x & 31;
  uint32_t x = r, g = f;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    uint32_t h = __shfl_up_sync(0xffffffffu, g, o);
    if (lane >= o) {
      if (!g) x = op(y, x);
      g |= h;
    }
  }
  uint32_t cx = 0;
  if (G > 32) {
    const int wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 31) {
      t->v[wid] = x;
      t->f[wid] = g;
    }
    __syncthreads();
    for (int i = 0; i < wid; i++) cx = t->f[i] ? (uint32_t)t->v[i] : op(cx, (uint32_t)t->v[i]);
    __syncthreads();
    if (!g) x = op(cx, x);
  }
  uint32_t ex = __shfl_up_sync(0xffffffffu, x, 1);
  if (lane == 0) ex = cx;
  return ex;
}

struct OpAdd {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a + b; }
};
struct OpMax {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

// Blocked segmented inclusive scan over an array of n elements: out[i] = op-fold of val(j)
// for j from the last head <= i up to i. Each thread owns a contiguous chunk. With Rev the
// scan runs from the end (head() then marks segment tails). out may alias val's source as
// long as val(i) only reads index i of it.
template <int G, bool Rev, class Op, class V, class H>
__device__ __forceinline__ void arr_seg_scan(uint32_t* out, int n, V val, H head, Op op, RedTmp<G>* t) {
  const int tid = Grp<G>::tid();
  const int C = (n + G - 1) / G;
  const int lo = tid * C < n ? tid * C : n;
  const int hi = lo + C < n ? lo + C : n;
  uint32_t r = 0, f = 0;
  for (int u = lo; u < hi; u++) {
    const int i = Rev ? n - 1 - u : u;
    uint32_t v = val(i);
    bool h = head(i);
    r = h ? v : op(r, v);
    f |= h ? 1u : 0u;
  }
  uint32_t run = grp_seg_scan_excl<G>(r, f, t, op);
  for (int u = lo; u < hi; u++) {
    const int i = Rev ? n - 1 - u : u;
    uint32_t v = val(i);
    bool h = head(i);
    run = h ? v : op(run, v);
    out[i] = run;
  }
  Grp<G>::sync();
}

}  // namespace mg
