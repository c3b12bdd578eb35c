// The classification pipeline for one read, written once for a cooperating group of G
// threads (one warp, or a whole block) over a workspace that lives in shared memory (warp and
// block tiers) or in global memory (the tier for reads beyond shared-memory capacity).
//
// Per strand it restates, in data-parallel form:
//   seed hashing and lookup      Analyser.cpp:1453-1519, Hashmap.cpp:3197-3268
//   posting lists                Analyser.cpp:1602-1752 (decoded once at index load)
//   occurrence filter            Analyser.cpp:2004-2196
//   sort + group by reference    Analyser.cpp:1024-1036, 2225-2315
//   diagonal runs + keep rule    Analyser.cpp:2337-2490
//   dot-matrix score             MatrixCPU.cpp:18-214
//   relative score, best pick    MatrixCPU.cpp:323-370, MatrixResult.cpp:21-29
// and then merges the strands (Analyser.cpp:592-611).
#pragma once
#include "mg_device.cuh"

namespace mg {

// Inline candidate slots per read in the staging area; reads with more scored candidates
// place them in an overflow arena.
constexpr int kSlots = 4;

// mg_read_result::strand of a read whose candidates hold raw sums (the dual-strand tier leaves the
// scores to k_finish_dual); never left in a finished result.
constexpr uint8_t kReadUnscored = 0xFD;

struct Caps {
  int q;      // max read length
  int seeds;  // max seeds per strand
  int e;      // max postings per strand (power of two, <= 65536)
  int c;      // max scored candidates per strand
};

struct StrandWS {
  uint8_t* q;          // strand bases
  uint32_t* fpos;      // query position of each found seed
  uint64_t* kA;        // sort keys
  uint32_t* kB;        // secondary keys / scratch
  uint32_t* X;         // per-entry scratch
  uint32_t* Y;         // per-entry scratch
  mg_candidate* cb[2]; // scored candidates of the forward and reverse strands
  uint32_t* W;         // wide form only: per-entry covered-interval start
  uint32_t* cov;       // wide form only: coverage bitmap of one candidate, (q + 31) / 32 words
};

enum StrandStatus { kStrandOk = 0, kStrandOverflow = 1, kStrandBad = 2 };

__device__ __forceinline__ int next_pow2(int x) {
  int n = 1;
  while (n < x) n <<= 1;
  return n;
}

// Bitonic sort of N (power of two) (kA, kB) pairs ascending by kA, then kB (kB may be null).
template <int G>
__device__ __forceinline__ void bitonic_sort(uint64_t* kA, uint32_t* kB, int N) {
  const int tid = Grp<G>::tid();
  for (int k = 2; k <= N; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < N; i += G) {
        int p = i ^ j;
        if (p > i) {
          bool up = (i & k) == 0;
          uint64_t a = kA[i], b = kA[p];
          uint32_t a2 = kB ? kB[i] : 0, b2 = kB ? kB[p] : 0;
          bool gt = (a > b) || (a == b && a2 > b2);
          if (gt == up) {
            kA[i] = b;
            kA[p] = a;
            if (kB) {
              kB[i] = b2;
              kB[p] = a2;
            }
          }
        }
      }
      Grp<G>::sync();
    }
  }
}

// Head walk (MatrixCPU.cpp:116-171): the query byte Start.Q-1-j is compared with the reference
// byte Start.Ref-j; the walk stops at the first mismatch j, or after a match at j when
// Start.Q-1-j, Start.Ref-j or headSize-1-j reaches 0, with the count j in both cases.
__device__ __forceinline__ uint32_t head_walk(const uint8_t* q, const uint8_t* rs, uint32_t sq, uint32_t sr, uint32_t k) {
  if (sq == 0) return 0;
  uint32_t hs = sr < k ? sr : k;
  if (hs == 0) return 0;
  uint32_t jb = sq - 1 < hs - 1 ? sq - 1 : hs - 1;
  for (uint32_t j = 0;; j++) {
    if (q[sq - 1 - j] != rs[sr - j]) return j;
    if (j == jb) return j;
  }
}

// Tail walk (MatrixCPU.cpp:93-112): matches from Last onwards, bounded by the read end, the
// reference end and min(k, refSize - Last.Ref).
__device__ __forceinline__ uint32_t tail_walk(const uint8_t* q, const uint8_t* rs, uint32_t L, uint32_t rlen,
                                              uint32_t lq, uint32_t lr, uint32_t k) {
  if (lq >= L || lr >= rlen) return 0;
  uint32_t lim = rlen - lr;
  if (k < lim) lim = k;
  if (L - lq < lim) lim = L - lq;
  uint32_t i = 0;
  while (i < lim && q[lq + i] == rs[lr + i]) i++;
  return i;
}

// One strand. Returns kStrandOverflow when the read does not fit the workspace caps (the
// caller hands the read to a larger tier); on success *n_out scored candidates are in cb and
// *highest is the strand's HighestScore.
// Wide (the oversize tier): found indexes, posting indexes and query positions need not fit 16
// bits. The occurrence sort then keys (refID << 32 | found index) with the posting index as the
// secondary key, a run's covered interval keeps its start in ws.W and its length in ws.X, and a
// candidate's coverage is OR-ed into the bitmap ws.cov; the order of every sort and the values
// compared are the same as in the packed form.
template <int G, bool Wide = false>
__device__ int process_strand(const DevIndex& ix, const uint8_t* raw, uint32_t L, int strand,
                              const StrandWS& ws, const Caps& caps, RedTmp<G>* red, int* err,
                              uint32_t* n_out, float* highest) {
  const int tid = Grp<G>::tid();
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  *n_out = 0;
  *highest = -1.0f;
  if ((int)L > caps.q) return kStrandOverflow;
  // strand bases (A0): uppercase, reverse complement for strand 1
  uint32_t bad = 0;
  for (uint32_t i = tid; i < L; i += G) {
    uint8_t c;
    if (strand == 0) {
      c = upper_dev(raw[i]);
    } else {
      c = complement_dev(upper_dev(raw[L - 1 - i]));
      if (!c) bad = 1;
    }
    ws.q[i] = c;
  }
  bad = (uint32_t)grp_max_u64<G>(bad, red);
  if (bad) return kStrandBad;
  Grp<G>::sync();
  if (L <= k) return kStrandOk;  // no seed fits (the reference would hash past the read)
  const uint32_t n_seeds = (L - k + step - 1) / step;
  if ((int)n_seeds > caps.seeds) return kStrandOverflow;
  // 1. seeds, directory probe, found list, postings gather
  uint32_t nf = 0, ne = 0;
  for (uint32_t j0 = 0; j0 < n_seeds; j0 += G) {
    const uint32_t j = j0 + tid;
    uint32_t found = 0, cnt = 0, o0 = 0;
    if (j < n_seeds) {
      const uint32_t h = hash28_dev(ws.q + j * step, ix.hlen);
      o0 = __ldg(ix.dir + h);
      const uint32_t o1 = __ldg(ix.dir + h + 1);
      cnt = o1 - o0;
      found = (cnt > 0 || h == ix.empty_hash) ? 1u : 0u;
    }
    uint32_t fr, er;
    const uint32_t fi = grp_excl_sum<G>(found, red, &fr);
    const uint32_t ei = grp_excl_sum<G>(cnt, red, &er);
    if (ne + er <= (uint32_t)caps.e) {
      const uint32_t f = nf + fi, e = ne + ei;
      if (found) ws.fpos[f] = j * step;
      for (uint32_t t = 0; t < cnt; t++) {
        const uint2 p = __ldg(ix.post + o0 + t);
        ws.X[e + t] = p.y;
        if (Wide) {
          ws.kA[e + t] = ((uint64_t)p.x << 32) | (uint64_t)f;
          ws.kB[e + t] = e + t;
        } else {
          ws.kA[e + t] = ((uint64_t)p.x << 32) | ((uint64_t)f << 16) | (uint64_t)(e + t);
        }
      }
    }
    nf += fr;
    ne += er;
  }
  if (ne > (uint32_t)caps.e) return kStrandOverflow;
  if (ne == 0) return kStrandOk;  // nothing to filter: the reference skips the read
  const int T = (int)ne;
  const int N = next_pow2(T);
  for (int i = T + tid; i < N; i += G) {
    ws.kA[i] = ~0ull;
    if (Wide) ws.kB[i] = ~0u;
  }
  Grp<G>::sync();
  // 2. occurrence filter over (refID, found index)
  bitonic_sort<G>(ws.kA, Wide ? ws.kB : nullptr, N);
  uint64_t* kA = ws.kA;
  auto refA = [&](int i) { return (uint32_t)(kA[i] >> 32); };
  auto fA = [&](int i) { return Wide ? (uint32_t)kA[i] : (uint32_t)((kA[i] >> 16) & 0xFFFFu); };
  auto obrk = [&](int i) { return i == 0 || refA(i) != refA(i - 1) || fA(i) > fA(i - 1) + 1; };
  arr_seg_scan<G, false>(ws.Y, T,
                         [&](int i) -> uint32_t { return obrk(i) ? 1u : (fA(i) == fA(i - 1) + 1 ? 1u : 0u); },
                         obrk, OpAdd(), red);
  uint32_t mx = 0;
  {
    const int C = (T + G - 1) / G;
    for (int i = tid * C; i < T && i < (tid + 1) * C; i++) mx = ws.Y[i] > mx ? ws.Y[i] : mx;
  }
  uint32_t hs = (uint32_t)grp_max_u64<G>(mx, red);
  if (hs < 2) hs = 0;  // highestSuccesive only grows on a continued occurrence
  const uint32_t keep_min = hs > 1 ? hs - 1 : 1;  // Analyser.cpp:2115
  auto rhead = [&](int i) { return i == 0 || refA(i) != refA(i - 1); };
  auto rtail = [&](int i) { return i == T - 1 || refA(i) != refA(i + 1); };
  uint32_t* Y = ws.Y;
  arr_seg_scan<G, false>(ws.Y, T, [&](int i) -> uint32_t { return Y[i]; }, rhead, OpMax(), red);
  arr_seg_scan<G, true>(ws.Y, T, [&](int i) -> uint32_t { return Y[i]; }, rtail, OpMax(), red);
  // 3. kept entries become (ref << 32 | position, query position) keys
  uint32_t kept = 0;
  {
    const int C = (T + G - 1) / G;
    for (int i = tid * C; i < T && i < (tid + 1) * C; i++) {
      const uint64_t key = kA[i];
      if (ws.Y[i] >= keep_min) {
        const uint32_t idx = Wide ? ws.kB[i] : (uint32_t)(key & 0xFFFFu);
        const uint32_t f = Wide ? (uint32_t)key : (uint32_t)((key >> 16) & 0xFFFFu);
        kA[i] = ((key >> 32) << 32) | (uint64_t)ws.X[idx];
        ws.kB[i] = ws.fpos[f];
        kept++;
      } else {
        kA[i] = ~0ull;
        ws.kB[i] = ~0u;
      }
    }
    for (int i = T + tid; i < N; i += G) ws.kB[i] = ~0u;
  }
  const int T2 = (int)grp_sum_u64<G>(kept, red);
  Grp<G>::sync();
  // 4. sort by (ref, reference position, query position)
  bitonic_sort<G>(ws.kA, ws.kB, N);
  uint32_t* kB = ws.kB;
  auto rpos = [&](int i) { return (uint32_t)(kA[i] & 0xFFFFFFFFu); };
  auto dbrk = [&](int i) {
    return i == 0 || refA(i) != refA(i - 1) ||
           !((uint64_t)rpos(i - 1) + step == rpos(i) && (uint64_t)kB[i - 1] + step == kB[i]);
  };
  auto rhead2 = [&](int i) { return i == 0 || refA(i) != refA(i - 1); };
  auto rtail2 = [&](int i) { return i == T2 - 1 || refA(i) != refA(i + 1); };
  // 5. diagonal runs: X = position within the run, Y = longest run of the reference
  arr_seg_scan<G, false>(ws.X, T2, [&](int) -> uint32_t { return 1u; }, dbrk, OpAdd(), red);
  uint32_t* X = ws.X;
  arr_seg_scan<G, false>(ws.Y, T2, [&](int i) -> uint32_t { return X[i]; }, rhead2, OpMax(), red);
  arr_seg_scan<G, true>(ws.Y, T2, [&](int i) -> uint32_t { return Y[i]; }, rtail2, OpMax(), red);
  uint32_t mr = 0;
  {
    const int C = (T2 + G - 1) / G;
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++) mr = ws.Y[i] > mr ? ws.Y[i] : mr;
  }
  const uint32_t M = (uint32_t)grp_max_u64<G>(mr, red);
  if (M < 2) return kStrandOk;  // Analyser.cpp:2402
  // 6. head/tail extension of every run of a kept reference (runMax == M); the run's
  // covered interval [Start.Q - head, Start.Q - head + T) and T go to X at the run's end.
  {
    const int C = (T2 + G - 1) / G;
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++) {
      uint32_t z = 0;
      const bool rend = (i == T2 - 1) || dbrk(i + 1);
      if (rend && ws.Y[i] == M) {
        const int s = i - (int)X[i] + 1;
        const uint32_t ref = refA(i);
        const uint32_t sr = rpos(s), sq = kB[s];
        const uint32_t lr = rpos(i) + step, lq = kB[i] + step;
        const uint8_t* rs = ix.bases + ix.ref_off[ref];
        const uint32_t rlen = ix.ref_len[ref];
        const uint32_t tail = tail_walk(ws.q, rs, L, rlen, lq, lr, k);
        const uint32_t head = head_walk(ws.q, rs, sq, sr, k);
        const uint32_t tot = tail + head + (lq - sq);
        if (Wide) {
          if (tot >= k) {
            z = tot;
            ws.W[i] = sq - head;
          }
        } else if (tot >= k) {
          z = ((sq - head) << 16) | tot;
        }
      }
      X[i] = z;
    }
  }
  Grp<G>::sync();
  // 7. candidate references in ascending refID: heads of reference segments with runMax == M
  uint32_t ncand_local = 0;
  {
    const int C = (T2 + G - 1) / G;
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++) ncand_local += (rhead2(i) && ws.Y[i] == M);
    uint32_t nc_total;
    uint32_t at = grp_excl_sum<G>(ncand_local, red, &nc_total);
    Grp<G>::sync();
    for (int i = tid * C; i < T2 && i < (tid + 1) * C; i++)
      if (rhead2(i) && ws.Y[i] == M) kB[at++] = (uint32_t)i;  // kB is free after step 6
    ncand_local = nc_total;
  }
  Grp<G>::sync();
  const uint32_t n_cand = ncand_local;
  const uint32_t nw = (L + 31) / 32;
  uint32_t n_sc = 0;
  float hi = -1.0f;
  for (uint32_t c = 0; c < n_cand; c++) {
    const int sa = (int)kB[c];
    const uint32_t ref = refA(sa);
    int sb = T2;
    {
      uint32_t first = (uint32_t)T2;
      for (int i = sa + 1 + tid; i < T2; i += G)
        if (refA(i) != ref) { first = (uint32_t)i; break; }
      sb = (int)(uint32_t)(~grp_max_u64<G>(~(uint64_t)first, red));  // group min
    }
    uint64_t sc = 0, sr = 0;
    for (int i = sa + tid; i < sb; i += G) {
      const uint32_t z = X[i];
      if (z) {
        const uint64_t t = Wide ? z : z & 0xFFFFu;
        sc += t;
        sr += (t * (t + 1)) / 2;
      }
    }
    sc = grp_sum_u64<G>(sc, red);
    sr = grp_sum_u64<G>(sr, red);
    if (sc == 0) continue;  // Score stays -2
    uint32_t hits = 0;
    if (Wide) {
      // covered intervals OR-ed into the bitmap: work in proportion to the intervals' lengths,
      // not to (read words x run records)
      for (uint32_t w = tid; w < nw; w += G) ws.cov[w] = 0;
      Grp<G>::sync();
      for (int i = sa + tid; i < sb; i += G) {
        const uint32_t t = X[i];
        if (!t) continue;
        const uint32_t a = ws.W[i], b = a + t;  // b <= L: the tail walk stops at the read's end
        for (uint32_t w = a >> 5; w <= (b - 1) >> 5; w++) {
          const uint32_t w0 = w * 32, lo = a > w0 ? a : w0, up = b < w0 + 32 ? b : w0 + 32;
          const uint32_t n = up - lo;
          atomicOr(ws.cov + w, (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u)) << (lo - w0));
        }
      }
      Grp<G>::sync();
      for (uint32_t w = tid; w < nw; w += G) hits += __popc(ws.cov[w]);
    }
    for (uint32_t w = tid; !Wide && w < nw; w += G) {
      uint32_t bits = 0;
      const uint32_t w0 = w * 32, w1 = w0 + 32;
      for (int i = sa; i < sb; i++) {
        const uint32_t z = X[i];
        if (!z) continue;
        const uint32_t a = z >> 16, b = a + (z & 0xFFFFu);
        const uint32_t lo = a > w0 ? a : w0, up = b < w1 ? b : w1;
        if (lo < up) {
          const uint32_t n = up - lo;
          bits |= (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u)) << (lo - w0);
        }
      }
      hits += __popc(bits);
    }
    hits = (uint32_t)grp_sum_u64<G>(hits, red);
    float score, pct;
    final_score(sr, sc, hits, L, &score, &pct);
    const float rel = relative_score(ix, __uint2float_rn(L), __uint2float_rn(ix.ref_len[ref]), score, err);
    if ((int)n_sc >= caps.c) return kStrandOverflow;
    if (tid == 0) ws.cb[strand][n_sc] = mg_candidate{ref, rel, score, pct};
    n_sc++;
    if (rel > hi) hi = rel;
  }
  Grp<G>::sync();
  *n_out = n_sc;
  *highest = hi;
  return kStrandOk;
}

// Strand merge (Analyser.cpp:592-611), the log skip rule (:388) and the staging write of one
// read's scored candidates (forward strand first). Called by one thread; per-strand values are
// scalars (n0/h0/cb0 forward, n1/h1/cb1 reverse complement).
__device__ __forceinline__ void write_read_result_s(const BatchDev& b, uint32_t r, bool bad, uint32_t n0,
                                                    uint32_t n1, float h0, float h1, const mg_candidate* cb0,
                                                    const mg_candidate* cb1, mg_candidate* stage,
                                                    mg_candidate* arena, uint64_t arena_cap,
                                                    unsigned long long* arena_n, int* errw, int err) {
  mg_read_result rr;
  if (bad) {
    err |= kErrBadInput;
    rr = mg_read_result{-1.0f, 0, 0, 0, MG_READ_BAD_BYTE, 0, 0};
  } else {
    const int ch = h0 < h1 ? 1 : 0;  // Analyser.cpp:601
    const uint32_t nch = ch ? n1 : n0;
    const float hch = ch ? h1 : h0;
    const mg_candidate* cbc = ch ? cb1 : cb0;
    uint32_t top = 0;
    for (uint32_t c = 0; c < nch; c++) top += cbc[c].rel == hch;
    const uint32_t tot = n0 + n1;
    uint32_t where = 0;
    mg_candidate* dst = stage + (uint64_t)r * kSlots;
    if (tot > (uint32_t)kSlots) {
      unsigned long long at = atomicAdd(arena_n, (unsigned long long)tot);
      if (at + tot > arena_cap) {
        err |= kErrArena;
        dst = nullptr;
      } else {
        dst = arena + at;
        where = (uint32_t)at;
      }
    }
    if (dst) {
      for (uint32_t c = 0; c < n0; c++) dst[c] = cb0[c];
      for (uint32_t c = 0; c < n1; c++) dst[n0 + c] = cb1[c];
    }
    const uint8_t reported = (nch > 0 && hch != 0.0f) ? 1 : 0;  // Analyser.cpp:388
    rr = mg_read_result{hch, where, (uint16_t)n0, (uint16_t)n1, (uint8_t)ch, reported, (uint16_t)top};
  }
  b.reads[r] = rr;
  if (err) atomicOr(errw, err);
}

__device__ __forceinline__ void write_read_result(const BatchDev& b, uint32_t r, bool bad, const uint32_t* n,
                                                  const float* h, mg_candidate* const* cb, mg_candidate* stage,
                                                  mg_candidate* arena, uint64_t arena_cap,
                                                  unsigned long long* arena_n, int* errw, int err) {
  write_read_result_s(b, r, bad, n[0], n[1], h[0], h[1], cb[0], cb[1], stage, arena, arena_cap, arena_n, errw, err);
}

// Both strands of read r, the strand merge and the staging write. Returns false when the
// read must go to a larger tier.
template <int G, bool Wide = false>
__device__ bool process_read(const DevIndex& ix, const BatchDev& b, uint32_t r, const StrandWS& ws,
                             const Caps& caps, RedTmp<G>* red, mg_candidate* stage, mg_candidate* arena,
                             uint64_t arena_cap, unsigned long long* arena_n, int* errw) {
  const int tid = Grp<G>::tid();
  const uint64_t o0 = b.offs[r];
  const uint64_t Lr = b.offs[r + 1] - o0;
  if (Lr > (Wide ? (uint64_t)caps.q : 0xFFFFull)) return false;
  const uint32_t L = (uint32_t)Lr;
  const uint8_t* raw = b.bases + o0;
  int err = 0;
  uint32_t n[2] = {0, 0};
  float h[2] = {-1.0f, -1.0f};
  int st = process_strand<G, Wide>(ix, raw, L, 0, ws, caps, red, &err, &n[0], &h[0]);
  if (st == kStrandOverflow) return false;
  if (st != kStrandBad) st = process_strand<G, Wide>(ix, raw, L, 1, ws, caps, red, &err, &n[1], &h[1]);
  if (st == kStrandOverflow) return false;
  if (tid == 0) write_read_result(b, r, st == kStrandBad, n, h, ws.cb, stage, arena, arena_cap, arena_n, errw, err);
  Grp<G>::sync();
  return true;
}

}  // namespace mg
