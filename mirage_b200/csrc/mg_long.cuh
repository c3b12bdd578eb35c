// Long-read tier: reads longer than the warp tiers take, one block of kLgThreads threads per
// read, both strands in turn, over reads taken from a list by work stealing. Two sizes: reads up
// to kLsQ bases with up to kLsE postings and kLsK kept postings per strand in a block of about
// 51 KB of shared memory (four blocks per SM), then what they hand on, up to kLgQ bases, kLgE
// postings and kLgK kept postings, in blocks of about 105 KB (two per SM).
//
// The general path (process_strand, mg_kernels.cuh) sorts every posting of a strand twice:
// by (refID, found index) for the occurrence filter and again, with the postings it dropped
// padded in, by (refID, position, query position) for the diagonal runs. A 5 kb read has about
// 750 postings per strand, a 20 kb read 3,000, while only the postings of the one or two
// references with the longest occurrence runs survive the filter. Here the filter needs no sort:
//   occurrence filter  every (refID, found index) pair of the strand goes into a hash set in
//                      shared memory; a pair whose (refID, found index - 1) is absent starts an
//                      occurrence run, whose length is the number of (refID, found index + t)
//                      present after it; occMax of a reference is its longest run
//                      (Analyser.cpp:2057-2115: consecutive found indices of one reference, a
//                      reference counted once per found index), hs the longest of all
//   keep rule          the references with a run of at least max(1, hs - 1) go to a small table
//                      and only their postings are compacted (Analyser.cpp:2115-2196)
//   sort               the kept postings only, by (refID, position, query position)
// and the diagonal runs, the walks, the coverage and the scores follow as in process_strand
// (Analyser.cpp:2337-2490, MatrixCPU.cpp:18-214), the coverage through a bitmap in shared memory.
#pragma once
#include "mg_kernels.cuh"

namespace mg {

constexpr int kLgThreads = 256;
constexpr int kLgQ = 20480;     // longest read (the config's 20 kb reads)
constexpr int kLgSeeds = 2047;  // seeds per strand (found index and seed index take 11 bits each)
constexpr int kLgE = 4096;      // postings per strand
constexpr int kLsQ = 8192;      // the smaller size: longest read
constexpr int kLsE = 2048;      // the smaller size: postings per strand
constexpr int kLgK = 2048;      // kept postings per strand (the larger size)
constexpr int kLsK = 1024;      // the smaller size: kept postings per strand
constexpr int kLgC = 64;        // scored candidates per strand
constexpr int kLgRT = 128;      // table of kept references (at most half of it used)
constexpr uint32_t kLgEmpty = 0xFFFFFFFFu;

// Dynamic shared memory of one block. From the compaction on, the hash set holds the sort keys
// (kA: K uint64, kB: K uint32), p_ref and p_pos the per-entry scratch X and Y, and p_fj
// the coverage bitmap.
template <int Q, int E, int K>
struct alignas(16) LongSmemT {
  static constexpr int kQ = Q, kE = E, kK = K;
  uint32_t hs[2 * E];         // (refID << 11 | found index) set, open addressing
  uint32_t p_ref[E];          // the strand's postings in seed order
  uint32_t p_pos[E];
  uint32_t p_fj[E];           // found index | seed index << 11 | 1 << 31 for the pair's first posting
  uint32_t rt[kLgRT];         // kept references
  mg_candidate cb[2][kLgC];   // scored candidates of the two strands
  RedTmp<kLgThreads> red;
  uint32_t n_kept, n_rt;
  uint32_t scored[kLgC / 32];  // candidates with a score (bit per candidate)
  uint32_t rrank[kLgRT];       // kept reference of a table slot: its rank by refID
  uint32_t bcnt[kLgRT / 2], bfill[kLgRT / 2], boff[kLgRT / 2 + 1], bmax;  // the kept references' ranges
  uint32_t n_sc;
  float hi;
  uint8_t q[Q];               // strand bases
  static_assert(K * 12 <= 2 * E * 4 && K <= E && Q / 32 + 1 <= E && 4 * kLgThreads <= 2 * E, "aliased regions");
};
using LongSmem = LongSmemT<kLgQ, kLgE, kLgK>;   // two blocks per SM
using LongSmemS = LongSmemT<kLsQ, kLsE, kLsK>;  // four blocks per SM
static_assert(2 * (sizeof(LongSmem) + 1024) <= 233472, "two blocks per SM");
static_assert(4 * (sizeof(LongSmemS) + 1024) <= 233472, "four blocks per SM");

__device__ __forceinline__ uint32_t lg_mix(uint32_t x) { return (x * 2654435761u) ^ (x >> 15); }

// The probes visit each slot at most once: every caller keeps its table at most half full, so an
// empty slot ends them first; reaching the bound sets kErrInternal in *err.
__device__ __forceinline__ bool lg_contains(const uint32_t* set, uint32_t mask, uint32_t key, int* err) {
  uint32_t s = lg_mix(key) & mask;
  for (uint32_t n = 0; n <= mask; n++, s = (s + 1) & mask) {
    const uint32_t v = set[s];
    if (v == key) return true;
    if (v == kLgEmpty) return false;
  }
  *err |= kErrInternal;
  return false;
}

// The slot holding key, or -1 (bounded like lg_contains).
__device__ __forceinline__ int lg_find(const uint32_t* set, uint32_t mask, uint32_t key, int* err) {
  uint32_t s = lg_mix(key) & mask;
  for (uint32_t n = 0; n <= mask; n++, s = (s + 1) & mask) {
    const uint32_t v = set[s];
    if (v == key) return (int)s;
    if (v == kLgEmpty) return -1;
  }
  *err |= kErrInternal;
  return -1;
}

// Inserts key; true when this call inserted it (false: it was there already).
__device__ __forceinline__ bool lg_insert(uint32_t* set, uint32_t mask, uint32_t key, int* err) {
  uint32_t s = lg_mix(key) & mask;
  for (uint32_t n = 0; n <= mask; n++, s = (s + 1) & mask) {
    const uint32_t old = atomicCAS(&set[s], kLgEmpty, key);
    if (old == kLgEmpty) return true;
    if (old == key) return false;
  }
  *err |= kErrInternal;
  return false;
}

// One strand of a read (raw bytes, L <= SM::kQ) on the whole block. Same contract as
// process_strand: kStrandOverflow hands the read to the block tier.
template <class SM>
__device__ int long_strand(const DevIndex& ix, const uint8_t* raw, uint32_t L, int strand, SM& S, int* err,
                           uint32_t* n_out, float* highest) {
  constexpr int kE = SM::kE;
  constexpr int G = kLgThreads;
  const int tid = threadIdx.x;
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  RedTmp<G>* red = &S.red;
  *n_out = 0;
  *highest = -1.0f;
  // strand bases (A0)
  uint32_t bad = 0;
  for (uint32_t i = tid; i < L; i += G) {
    uint8_t c;
    if (strand == 0) {
      c = upper_dev(raw[i]);
    } else {
      c = complement_dev(upper_dev(raw[L - 1 - i]));
      if (!c) bad = 1;
    }
    S.q[i] = c;
  }
  if (grp_max_u64<G>(bad, red)) return kStrandBad;
  if (L <= k) return kStrandOk;
  const uint32_t ns = (L - k + step - 1) / step;
  if (ns > (uint32_t)kLgSeeds) return kStrandOverflow;
  // 1. seeds, probe, found indices, postings in seed order
  uint32_t nf = 0, ne = 0;
  for (uint32_t j0 = 0; j0 < ns; j0 += G) {
    const uint32_t j = j0 + tid;
    uint32_t found = 0, cnt = 0, o0 = 0;
    uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0, v2 = v0, v3 = v0;
    if (j < ns) {
      const uint32_t h = hash28_dev(S.q + j * step, ix.hlen);
      if (ix.slots) {
        const uint4* sl = ix.slots + (size_t)h * kSlotVecs;
        v0 = __ldg(sl);
        v1 = __ldg(sl + 1);
        cnt = v0.x;
        o0 = v0.y;
        if (cnt > 3) {
          v2 = __ldg(sl + 2);
          v3 = __ldg(sl + 3);
        }
      } else {
        o0 = __ldg(ix.dir + h);
        cnt = __ldg(ix.dir + h + 1) - o0;
      }
      found = (cnt > 0 || h == ix.empty_hash) ? 1u : 0u;
    }
    const uint32_t x = cnt > (uint32_t)kE ? (uint32_t)kE + 1 : cnt;
    uint32_t fr, er;
    const uint32_t fi = grp_excl_sum<G>(found, red, &fr);
    const uint32_t ei = grp_excl_sum<G>(x, red, &er);
    if (ne + er > (uint32_t)kE) return kStrandOverflow;  // group-uniform
    const uint32_t e = ne + ei, fj = (nf + fi) | (j << 11);
    uint32_t t0 = 0;
    if (ix.slots) {
      auto put = [&](uint32_t t, uint32_t ref, uint32_t pos) {
        if (t < cnt) {
          S.p_ref[e + t] = ref;
          S.p_pos[e + t] = pos;
          S.p_fj[e + t] = fj;
        }
      };
      put(0, v0.z, v0.w);
      put(1, v1.x, v1.y);
      put(2, v1.z, v1.w);
      put(3, v2.x, v2.y);
      put(4, v2.z, v2.w);
      put(5, v3.x, v3.y);
      put(6, v3.z, v3.w);
      t0 = kSlotPosts;
    }
    // the postings past the slot's (all of them without slots), a warp per seed with its lanes on
    // consecutive postings: each seed's (offset, count, start, fj) goes to the hash set's space,
    // unused until step 2 (the barriers of the next group's sums order its reuse)
    uint32_t* o0S = S.hs;
    uint32_t* cntS = S.hs + G;
    uint32_t* eS = S.hs + 2 * G;
    uint32_t* fjS = S.hs + 3 * G;
    o0S[tid] = o0;
    cntS[tid] = cnt;
    eS[tid] = e;
    fjS[tid] = fj;
    __syncthreads();
    {
      const uint32_t gn = min((uint32_t)G, ns - j0), lane = (uint32_t)tid & 31u;
      for (uint32_t sd = (uint32_t)tid >> 5; sd < gn; sd += G / 32) {
        const uint32_t c = cntS[sd];
        if (c <= t0) continue;  // warp-uniform
        const uint32_t o = o0S[sd], es = eS[sd], f = fjS[sd];
        for (uint32_t t = t0 + lane; t < c; t += 32) {
          const uint2 p = __ldg(ix.post + o + t);
          S.p_ref[es + t] = p.x;
          S.p_pos[es + t] = p.y;
          S.p_fj[es + t] = f;
        }
      }
    }
    nf += fr;
    ne += er;
  }
  __syncthreads();  // the postings in place before step 2 clears the hash set
  if (ne == 0) return kStrandOk;  // nothing found: the reference skips the strand
  // 2. occurrence filter: the (refID, found index) set
  uint32_t hsz = 64;
  while (hsz < 2 * ne) hsz <<= 1;
  const uint32_t mask = hsz - 1;
  for (uint32_t i = tid; i < hsz; i += G) S.hs[i] = kLgEmpty;
  for (uint32_t i = tid; i < (uint32_t)kLgRT; i += G) S.rt[i] = kLgEmpty;
  if (tid == 0) {
    S.n_kept = 0;
    S.n_rt = 0;
  }
  __syncthreads();
  for (uint32_t i = tid; i < ne; i += G)
    if (lg_insert(S.hs, mask, (S.p_ref[i] << 11) | (S.p_fj[i] & 0x7FFu), err)) S.p_fj[i] |= 0x80000000u;
  __syncthreads();
  // occurrence runs from their first found index: the longest is hs
  auto run_from = [&](uint32_t i) -> uint32_t {  // 0 unless posting i starts a run
    const uint32_t fj = S.p_fj[i];
    if (!(fj >> 31)) return 0;
    const uint32_t key = (S.p_ref[i] << 11) | (fj & 0x7FFu);
    if ((fj & 0x7FFu) && lg_contains(S.hs, mask, key - 1, err)) return 0;
    uint32_t len = 1;
    while ((fj & 0x7FFu) + len < nf && lg_contains(S.hs, mask, key + len, err)) len++;
    return len;
  };
  uint32_t mx = 0;
  for (uint32_t i = tid; i < ne; i += G) mx = max(mx, run_from(i));
  const uint32_t hs = (uint32_t)grp_max_u64<G>(mx, red);
  // hs only grows on a continued occurrence (Analyser.cpp:2087-2099): below 2 no reference can
  // reach a diagonal run of 2 either, so the strand has no candidate
  if (hs < 2) return kStrandOk;
  const uint32_t keep_min = hs - 1;  // max(1, hs - 1), Analyser.cpp:2115
  // each insertion attempt first claims a count (n_rt, an upper bound of the distinct references:
  // threads racing on one reference each claim one): at most kLgRT / 2 insertions happen, so the
  // table never fills, and a refused one leaves n_rt above kLgRT / 2, which sends the strand to the
  // block tier
  for (uint32_t i = tid; i < ne; i += G)
    if (run_from(i) >= keep_min && !lg_contains(S.rt, kLgRT - 1, S.p_ref[i], err))
      if (atomicAdd(&S.n_rt, 1u) < (uint32_t)kLgRT / 2) lg_insert(S.rt, kLgRT - 1, S.p_ref[i], err);
  __syncthreads();
  if (S.n_rt > (uint32_t)kLgRT / 2) {
    if (keep_min != 1) return kStrandOverflow;
    // hs = 2 keeps every reference with a posting (max(1, hs - 1) = 1), more than the table
    // holds. A diagonal run of 2 needs two postings of one reference on one diagonal at
    // consecutive seeds ((ref, pos, q) then (ref, pos + step, q + step), Analyser.cpp:2337-2402):
    // when the strand has no such pair its longest run M is below 2 and it has no candidate. The
    // pairs are looked for through the hash set, now free, of the postings' (ref, diagonal, seed)
    // keys folded to 32 bits; a collision can only report a pair that is not there, which sends
    // the strand on as before.
    auto dkey = [&](uint32_t i, uint32_t dj) -> uint32_t {
      const uint32_t j = (S.p_fj[i] >> 11) & 0x7FFu;
      const uint32_t d = S.p_pos[i] - j * step;  // the diagonal, modulo 2^32
      const uint64_t x = (uint64_t)S.p_ref[i] * 0x9E3779B97F4A7C15ull ^ (uint64_t)d * 0xC2B2AE3D27D4EB4Full ^
                         (uint64_t)(j + dj) * 0x165667B19E3779F9ull;
      const uint32_t v = (uint32_t)(x >> 32) ^ (uint32_t)x;
      return v == kLgEmpty ? kLgEmpty - 1u : v;
    };
    for (uint32_t i = tid; i < hsz; i += G) S.hs[i] = kLgEmpty;
    __syncthreads();
    for (uint32_t i = tid; i < ne; i += G) lg_insert(S.hs, mask, dkey(i, 0), err);
    __syncthreads();
    int pair = 0;
    for (uint32_t i = tid; i < ne && !pair; i += G) pair = lg_contains(S.hs, mask, dkey(i, 1), err) ? 1 : 0;
    if (__syncthreads_or(pair)) return kStrandOverflow;
    return kStrandOk;  // no diagonal run of 2: no candidate on this strand
  }
  // 3. the kept references' postings as (refID << 32 | position, query position) sort keys,
  //    grouped by reference: the kept references (at most kLgRT / 2) ranked by refID, each one's
  //    postings counted and given a range in that order, then scattered into it
  uint64_t* kA = reinterpret_cast<uint64_t*>(S.hs);
  constexpr int kK = SM::kK;
  constexpr int kBk = kLgRT / 2;  // ranges
  uint32_t* kB = S.hs + 2 * kK;
  if (tid < kLgRT) {
    const uint32_t r = S.rt[tid];
    uint32_t rk = 0;
    if (r != kLgEmpty)
      for (int s2 = 0; s2 < kLgRT; s2++) {
        const uint32_t r2 = S.rt[s2];
        rk += (r2 != kLgEmpty && r2 < r) ? 1u : 0u;
      }
    S.rrank[tid] = rk;
  }
  if (tid < kBk) {
    S.bcnt[tid] = 0;
    S.bfill[tid] = 0;
  }
  __syncthreads();
  for (uint32_t i = tid; i < ne; i += G) {
    const int sl = lg_find(S.rt, kLgRT - 1, S.p_ref[i], err);
    if (sl >= 0) atomicAdd(&S.bcnt[S.rrank[sl]], 1u);
  }
  __syncthreads();
  if (tid < 32) {  // the ranges' starts (two per lane), their total and the largest range
    const unsigned FULL = 0xFFFFFFFFu;
    const uint32_t c0 = S.bcnt[2 * tid], c1 = S.bcnt[2 * tid + 1];
    uint32_t x = c0 + c1;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, x, o);
      if (tid >= o) x += y;
    }
    const uint32_t ex = x - (c0 + c1);
    S.boff[2 * tid] = ex;
    S.boff[2 * tid + 1] = ex + c0;
    if (tid == 31) {
      S.boff[kBk] = x;
      S.n_kept = x;
    }
    const uint32_t mb = __reduce_max_sync(FULL, max(c0, c1));
    if (tid == 0) S.bmax = mb;
  }
  __syncthreads();
  const int T2 = (int)S.n_kept;
  if (T2 > kK) return kStrandOverflow;
  for (uint32_t i = tid; i < ne; i += G) {
    const int sl = lg_find(S.rt, kLgRT - 1, S.p_ref[i], err);
    if (sl >= 0) {
      const uint32_t b = S.rrank[sl];
      const uint32_t t = S.boff[b] + atomicAdd(&S.bfill[b], 1u);
      kA[t] = ((uint64_t)S.p_ref[i] << 32) | S.p_pos[i];
      kB[t] = ((S.p_fj[i] >> 11) & 0x7FFu) * step;
    }
  }
  __syncthreads();
  if (S.bmax <= 128u) {
    // each range sorted by (position, query position), a warp per range: an entry's place is the
    // number of its range's entries with a smaller key (the keys are distinct), written to the
    // postings' arrays, free by now, and copied back
    const uint32_t lane = (uint32_t)tid & 31u, warp = (uint32_t)tid >> 5;
    for (uint32_t b = warp; b < (uint32_t)kBk; b += G / 32) {
      const uint32_t b0 = S.boff[b], b1 = S.boff[b + 1];
      for (uint32_t e = b0 + lane; e < b1; e += 32) {
        const uint64_t ka = kA[e];
        const uint32_t kb = kB[e];
        uint32_t rk = 0;
        for (uint32_t f = b0; f < b1; f++) {
          const uint64_t fa = kA[f];
          rk += (fa < ka || (fa == ka && kB[f] < kb)) ? 1u : 0u;
        }
        S.p_ref[b0 + rk] = (uint32_t)(ka >> 32);
        S.p_pos[b0 + rk] = (uint32_t)ka;
        S.p_fj[b0 + rk] = kb;
      }
    }
    __syncthreads();
    for (int i = tid; i < T2; i += G) {
      kA[i] = ((uint64_t)S.p_ref[i] << 32) | S.p_pos[i];
      kB[i] = S.p_fj[i];
    }
    __syncthreads();
  } else {  // a large range (a read from one reference): one bitonic sort of all the keys
    const int N = next_pow2(T2);
    for (int i = T2 + tid; i < N; i += G) {
      kA[i] = ~0ull;
      kB[i] = ~0u;
    }
    __syncthreads();
    bitonic_sort<G>(kA, kB, N);
  }
  // 4. diagonal runs (Analyser.cpp:2337-2490): X = position within the run, Y = longest run of
  //    the reference
  uint32_t* X = S.p_ref;
  uint32_t* Y = S.p_pos;
  auto refA = [&](int i) { return (uint32_t)(kA[i] >> 32); };
  auto rpos = [&](int i) { return (uint32_t)(kA[i] & 0xFFFFFFFFu); };
  auto dbrk = [&](int i) {
    return i == 0 || refA(i) != refA(i - 1) ||
           !((uint64_t)rpos(i - 1) + step == rpos(i) && (uint64_t)kB[i - 1] + step == kB[i]);
  };
  auto rhead = [&](int i) { return i == 0 || refA(i) != refA(i - 1); };
  auto rtail = [&](int i) { return i == T2 - 1 || refA(i) != refA(i + 1); };
  arr_seg_scan<G, false>(X, T2, [&](int) -> uint32_t { return 1u; }, dbrk, OpAdd(), red);
  arr_seg_scan<G, false>(Y, T2, [&](int i) -> uint32_t { return X[i]; }, rhead, OpMax(), red);
  arr_seg_scan<G, true>(Y, T2, [&](int i) -> uint32_t { return Y[i]; }, rtail, OpMax(), red);
  uint32_t mr = 0;
  {
    const int C = (T2 + G - 1) / G;
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++) mr = Y[i] > mr ? Y[i] : mr;
  }
  const uint32_t M = (uint32_t)grp_max_u64<G>(mr, red);
  if (M < 2) return kStrandOk;  // Analyser.cpp:2402
  // 5. head/tail walks of every run of a reference whose longest run is M: the run's covered
  //    interval [Start.Q - head, Start.Q - head + T) and T go to X at the run's last entry
  {
    const int C = (T2 + G - 1) / G;
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++) {
      uint32_t z = 0;
      const bool rend = (i == T2 - 1) || dbrk(i + 1);
      if (rend && Y[i] == M) {
        const int s = i - (int)X[i] + 1;
        const uint32_t ref = refA(i);
        const uint32_t sr = rpos(s), sq = kB[s];
        const uint32_t lr = rpos(i) + step, lq = kB[i] + step;
        const uint8_t* rs = ix.bases + ix.ref_off[ref];
        const uint32_t rlen = ix.ref_len[ref];
        const uint32_t tail = tail_walk(S.q, rs, L, rlen, lq, lr, k);
        const uint32_t head = head_walk(S.q, rs, sq, sr, k);
        const uint32_t tot = tail + head + (lq - sq);
        if (tot >= k) z = ((sq - head) << 16) | tot;
      }
      X[i] = z;
    }
  }
  __syncthreads();
  // 6. candidates in ascending refID: the heads of the reference segments whose longest run is M
  uint32_t n_cand;
  {
    const int C = (T2 + G - 1) / G;
    uint32_t local = 0;
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++) local += (rhead(i) && Y[i] == M);
    uint32_t at = grp_excl_sum<G>(local, red, &n_cand);
    __syncthreads();
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++)
      if (rhead(i) && Y[i] == M) kB[at++] = (uint32_t)i;  // kB's query positions are walked by now
  }
  __syncthreads();
  // 7. scores, a warp per candidate (Analyser.cpp:2490-2540, MatrixCPU.cpp:18-214): the candidate's
  //    reference segment [sa, sb) of the sorted keys, its walked runs' lengths summed (sc) and summed
  //    as triangles (sr), the query bases they cover counted in the warp's own bitmap; a candidate
  //    whose runs all fell short of k keeps Score -2 and is not scored. Then the scored ones in
  //    ascending refID, and the highest relative score in that order.
  if (n_cand > (uint32_t)kLgC) return kStrandOverflow;  // group-uniform (n_rt bounds it first)
  const uint32_t nw = (L + 31) / 32;
  const uint32_t lane = (uint32_t)tid & 31u, warp = (uint32_t)tid >> 5;
  const uint32_t n_warps = min((uint32_t)(G / 32), (uint32_t)SM::kE / nw);  // bitmaps fit p_fj
  if (tid < kLgC / 32) S.scored[tid] = 0;
  __syncthreads();
  mg_candidate* out = S.cb[strand];
  if (warp < n_warps) {
    uint32_t* cov = S.p_fj + warp * nw;
    for (uint32_t c = warp; c < n_cand; c += n_warps) {
      const int sa = (int)kB[c];
      const uint32_t ref = refA(sa);
      uint32_t first = (uint32_t)T2;
      for (int i = sa + 1 + (int)lane; i < T2; i += 32)
        if (refA(i) != ref) {
          first = (uint32_t)i;
          break;
        }
      const int sb = (int)__reduce_min_sync(0xFFFFFFFFu, first);
      uint32_t sc = 0;
      uint64_t sr = 0;
      for (int i = sa + (int)lane; i < sb; i += 32) {
        const uint32_t z = X[i];
        if (z) {
          const uint64_t t = z & 0xFFFFu;
          sc += (uint32_t)t;
          sr += (t * (t + 1)) / 2;
        }
      }
      sc = __reduce_add_sync(0xFFFFFFFFu, sc);  // at most kK runs of < 2^16 bases each
      for (int o = 16; o; o >>= 1) sr += __shfl_xor_sync(0xFFFFFFFFu, sr, o);
      if (sc == 0) continue;  // warp-uniform: Score stays -2
      for (uint32_t w = lane; w < nw; w += 32) cov[w] = 0;
      __syncwarp();
      for (int i = sa + (int)lane; i < sb; i += 32) {
        const uint32_t z = X[i];
        if (!z) continue;
        const uint32_t a = z >> 16, bnd = a + (z & 0xFFFFu);
        for (uint32_t wd = a >> 5; wd <= (bnd - 1) >> 5; wd++) {
          const uint32_t w0 = wd * 32;
          const uint32_t lo = a > w0 ? a : w0, up = bnd < w0 + 32 ? bnd : w0 + 32;
          const uint32_t n = up - lo;
          atomicOr(&cov[wd], (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u)) << (lo - w0));
        }
      }
      __syncwarp();
      uint32_t hits = 0;
      for (uint32_t w = lane; w < nw; w += 32) hits += __popc(cov[w]);
      hits = __reduce_add_sync(0xFFFFFFFFu, hits);
      if (lane == 0) {
        float score, pct;
        final_score(sr, (uint64_t)sc, hits, L, &score, &pct);
        const float rel = relative_score(ix, __uint2float_rn(L), __uint2float_rn(ix.ref_len[ref]), score, err);
        out[c] = mg_candidate{ref, rel, score, pct};
        atomicOr(&S.scored[c >> 5], 1u << (c & 31u));
      }
      __syncwarp();  // the bitmap's next clear after this candidate's count
    }
  }
  __syncthreads();
  if (warp == 0) {  // in place: a scored candidate only moves down, after its chunk is read
    uint32_t n_sc = 0;
    for (uint32_t c0 = 0; c0 < n_cand; c0 += 32) {
      const uint32_t c = c0 + lane;
      const bool ok = c < n_cand && ((S.scored[c >> 5] >> (c & 31u)) & 1u);
      mg_candidate v{};
      if (ok) v = out[c];
      const uint32_t m = __ballot_sync(0xFFFFFFFFu, ok);
      __syncwarp();
      if (ok) out[n_sc + __popc(m & ((1u << lane) - 1u))] = v;
      n_sc += __popc(m);
    }
    __syncwarp();
    if (lane == 0) {
      float hi = -1.0f;
      for (uint32_t i = 0; i < n_sc; i++)
        if (out[i].rel > hi) hi = out[i].rel;
      S.n_sc = n_sc;
      S.hi = hi;
    }
  }
  __syncthreads();
  const uint32_t n_sc = S.n_sc;
  const float hi = S.hi;
  __syncthreads();  // S.n_sc and S.hi read before the next strand writes them
  *n_out = n_sc;
  *highest = hi;
  return kStrandOk;
}

// Both strands of read r, the strand merge and the staging write; false when the read must go
// to the next tier.
template <class SM>
__device__ bool process_read_long(const DevIndex& ix, const BatchDev& b, uint32_t r, SM& S, mg_candidate* stage,
                                  mg_candidate* arena, uint64_t arena_cap, unsigned long long* arena_n, int* errw) {
  const uint64_t o0 = b.offs[r];
  const uint64_t Lr = b.offs[r + 1] - o0;
  if (Lr > (uint64_t)SM::kQ || ix.n_refs > (1u << 21)) return false;  // keys hold refID << 11
  const uint32_t L = (uint32_t)Lr;
  const uint8_t* raw = b.bases + o0;
  int err = 0;
  uint32_t n[2] = {0, 0};
  float h[2] = {-1.0f, -1.0f};
  int st = long_strand(ix, raw, L, 0, S, &err, &n[0], &h[0]);
  if (st != kStrandBad && st != kStrandOverflow) st = long_strand(ix, raw, L, 1, S, &err, &n[1], &h[1]);
  if (err) atomicOr(errw, err);  // any thread's: the probes and the scoring lanes record bits per thread
  if (st == kStrandOverflow) return false;
  if (threadIdx.x == 0)
    write_read_result_s(b, r, st == kStrandBad, n[0], n[1], h[0], h[1], S.cb[0], S.cb[1], stage, arena, arena_cap,
                        arena_n, errw, err);
  __syncthreads();
  return true;
}

}  // namespace mg
