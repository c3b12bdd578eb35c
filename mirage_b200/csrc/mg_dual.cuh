// Dual-strand warp path: both strands of a read at once, one half-warp per strand (lanes 0-15
// the forward strand, lanes 16-31 its reverse complement), for reads of up to kLeanQ bases with
// at most 64 postings per strand.
//
// The steps are those of process_strand (mg_kernels.cuh) on 16-lane halves. Seed j sits on lane
// j % 16, posting slot i on lane i % 16 (one to four slots per lane, as many as the strand has);
// per-half bit masks are assembled from full-warp ballots and reductions use shuffles of width 16.
//   occurrence filter  a per-half hash table keyed by reference: each posting ORs its found index
//                      into its reference's entry; the longest run of ones is occMax
//   rank sort          over the kept postings only, compacted first (usually about one per seed)
// so the serial work per strand follows the kept postings, not all of them, and the two strands
// run side by side. Nothing is indexed dynamically in registers; per-posting state lives in
// shared memory, whose regions are reused from step to step.
#pragma once
#include "mg_lean.cuh"

namespace mg {

constexpr int kDualE = 64;               // postings per strand
constexpr int kDualTab = 64;             // occurrence table entries per strand (>= distinct refs)
constexpr int kDualC = 8;                // scored candidates per strand
constexpr int kCovWords = kLeanQ / 32;   // coverage bitmap words per lane

// Per-warp shared memory of the dual path; [half] = strand.
struct DualSmem {
  uint32_t a[2][3][kDualE];     // gathered postings (ref, pos, found | seed << 8 | table entry << 16);
                                // from the rank sort on: kept postings sorted (ref, pos, seed)
  uint32_t c[2][3][kDualE];     // kept postings, compacted (ref, pos, seed); during scoring the
                                // coverage bitmaps, kCovWords words per lane
  uint32_t t[2][2][kDualTab];   // occurrence table (ref key, found mask, then occMax); from the
                                // diagonal runs on: z (run ends) and segmax (reference heads)
  mg_candidate cb[2][kDualC];   // scored candidates in ascending refID
  uint8_t q[2][kLeanQ];         // strand bases: forward, reverse complement
  uint8_t q_pad[8];             // word reads of q[1]'s last bases run up to 7 bytes past it
};
static_assert(sizeof(uint32_t) * 2 * 3 * kDualE >= sizeof(uint32_t) * 32 * kCovWords, "coverage bitmaps");

__device__ __forceinline__ unsigned long long upto64(int i) {  // bits 0..i
  return i >= 63 ? ~0ull : ((2ull << i) - 1ull);
}
__device__ __forceinline__ unsigned long long below64(int i) {  // bits 0..i-1
  return i <= 0 ? 0ull : upto64(i - 1);
}

// Four bytes from p (any alignment) as one little-endian word, read as two aligned words.
__device__ __forceinline__ uint32_t bytes4(const uint8_t* p) {
  const uintptr_t a = (uintptr_t)p;
  const uint32_t* w = (const uint32_t*)(a & ~(uintptr_t)3);
  return __funnelshift_r(w[0], w[1], (uint32_t)(a & 3) * 8u);
}

// tail_walk (mg_kernels.cuh) four bytes at a time: the length of the common prefix of the query
// from lq and the reference from lr, at most min(rlen - lr, k, L - lq). Reads up to 7 bytes past
// the last compared byte of each side (the index's base array and the strand buffers are padded).
__device__ __forceinline__ uint32_t tail_walk4(const uint8_t* q, const uint8_t* rs, uint32_t L, uint32_t rlen,
                                               uint32_t lq, uint32_t lr, uint32_t k) {
  if (lq >= L || lr >= rlen) return 0;
  const uint32_t lim = min(min(rlen - lr, k), L - lq);
  for (uint32_t i = 0; i < lim; i += 4) {
    const uint32_t x = bytes4(q + lq + i) ^ bytes4(rs + lr + i);
    if (x) return min(i + ((uint32_t)(__ffs(x) - 1) >> 3), lim);
  }
  return lim;
}

// Bits of a full-warp ballot that belong to this lane's half.
__device__ __forceinline__ uint32_t half_bits(uint32_t ballot, int sh) { return (ballot >> sh) & 0xFFFFu; }

// A candidate before scoring: the sum of T(T+1)/2 over its scored runs, the sum of T and the
// covered query bases, as the bits of the rel, score and pct fields.
__device__ __forceinline__ mg_candidate raw_candidate(uint32_t ref, uint32_t sumr, uint32_t sumc, uint32_t hits) {
  return mg_candidate{ref, __uint_as_float(sumr), __uint_as_float(sumc), __uint_as_float(hits)};
}

// Both strands of one read (bases already in S.q). Warp-uniform return: kStrandOk, or
// kStrandOverflow when either strand does not fit. Each lane receives its half's strand result:
// *n_out candidates in S.cb[half] (ascending refID), raw (raw_candidate).
__device__ int dual_strands(const DevIndex& ix, uint32_t L, DualSmem& S, uint32_t* n_out) {
  const unsigned FULL = 0xffffffffu;
  const uint32_t EMPTY = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15, sh = half * 16;
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  const uint8_t* q = S.q[half];
  uint32_t* e_ref = S.a[half][0];
  uint32_t* e_pos = S.a[half][1];
  uint32_t* e_fj = S.a[half][2];
  uint32_t* c_ref = S.c[half][0];
  uint32_t* c_pos = S.c[half][1];
  uint32_t* c_j = S.c[half][2];
  uint32_t* tkey = S.t[half][0];
  uint32_t* tval = S.t[half][1];
  *n_out = 0;
  if (L <= k) return kStrandOk;
  const uint32_t ns = (L - k + step - 1) / step;
  if (ns > 32) return kStrandOverflow;
  const int nsb = (int)(ns + 15) / 16;  // seed blocks (warp-uniform: both strands have L bases)
  // 1. seeds, probe, found list, postings, block by block in seed order (seed j = hl + 16 s)
  uint32_t fb = 0, T = 0;
  for (int s = 0; s < nsb; s++) {
    const uint32_t j = hl + 16 * s;
    uint32_t cnt = 0, o0 = 0;
    bool fnd = false;
    if (j < ns) {
      const uint32_t h = hash28_dev(q + j * step, ix.hlen);
      o0 = __ldg(ix.dir + h);
      cnt = __ldg(ix.dir + h + 1) - o0;
      fnd = cnt > 0 || h == ix.empty_hash;
    }
    fb |= half_bits(__ballot_sync(FULL, fnd), sh) << (16 * s);
    uint32_t x = cnt > (uint32_t)kDualE ? (uint32_t)kDualE + 1 : cnt;
    for (int o = 1; o < 16; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, x, o, 16);
      if (hl >= o) x += y;
    }
    const uint32_t Tn = T + __shfl_sync(FULL, x, 15, 16);
    if (__any_sync(FULL, Tn > (uint32_t)kDualE)) return kStrandOverflow;
    const uint32_t f = __popc(fb & ((1u << j) - 1u));
    const uint32_t e = T + x - cnt;
    for (uint32_t t = 0; t < cnt; t++) {
      const uint2 p = __ldg(ix.post + o0 + t);
      e_ref[e + t] = p.x;
      e_pos[e + t] = p.y;
      e_fj[e + t] = f | (j << 8);
    }
    T = Tn;
  }
  bool alive = T > 0;
  if (!__any_sync(FULL, alive)) return kStrandOk;
  // 2. occurrence filter (Analyser.cpp:2057-2115): per reference, the found indices where it
  //    occurs (a table keyed by refID); the longest run of consecutive ones is its occMax
  for (int x = hl; x < kDualTab; x += 16) {
    tkey[x] = EMPTY;
    tval[x] = 0;
  }
  __syncwarp();
  const int nslw = (int)__reduce_max_sync(FULL, (T + 15) / 16);  // posting blocks, warp-uniform
  for (int s = 0; s < nslw; s++) {
    const uint32_t i = hl + 16 * s;
    if (i < T) {
      const uint32_t ref = e_ref[i];
      uint32_t x = (ref * 2654435761u) >> 26;  // 64 entries
      for (;;) {
        const uint32_t old = atomicCAS(&tkey[x], EMPTY, ref);
        if (old == EMPTY || old == ref) break;
        x = (x + 1) & (kDualTab - 1);
      }
      const uint32_t fj = e_fj[i];
      atomicOr(&tval[x], 1u << (fj & 0xFFu));
      e_fj[i] = fj | (x << 16);
    }
  }
  __syncwarp();
  int hs = 0;
  for (int x = hl; x < kDualTab; x += 16)
    if (tkey[x] != EMPTY) {
      const int o = longest_run(tval[x]);
      tval[x] = (uint32_t)o;
      hs = max(hs, o);
    }
  for (int o = 8; o > 0; o >>= 1) hs = max(hs, __shfl_xor_sync(FULL, hs, o));
  // below 2 no reference can reach a diagonal run of 2: no candidate on this strand
  alive = alive && hs >= 2;
  if (!__any_sync(FULL, alive)) return kStrandOk;
  __syncwarp();
  const uint32_t keep_min = (uint32_t)(hs - 1);  // max(1, hs - 1), Analyser.cpp:2115
  // kept postings compacted in gather order
  uint32_t T2 = 0;
  for (int s = 0; s < nslw; s++) {
    const uint32_t i = hl + 16 * s;
    bool kp = false;
    uint32_t fj = 0;
    if (alive && i < T) {
      fj = e_fj[i];
      kp = tval[fj >> 16] >= keep_min;
    }
    const uint32_t kb = half_bits(__ballot_sync(FULL, kp), sh);
    if (kp) {
      const uint32_t c = T2 + __popc(kb & ((1u << hl) - 1u));
      c_ref[c] = e_ref[i];
      c_pos[c] = e_pos[i];
      c_j[c] = (fj >> 8) & 0xFFu;
    }
    T2 += __popc(kb);
  }
  __syncwarp();
  // 3. rank sort of the kept postings by (ref, pos, seed); the keys are distinct
  uint32_t* s_ref = S.a[half][0];
  uint32_t* s_pos = S.a[half][1];
  uint32_t* s_j = S.a[half][2];
  const int nkw = (int)__reduce_max_sync(FULL, (T2 + 15) / 16);
  for (int s = 0; s < nkw; s++) {
    const uint32_t c = hl + 16 * s;
    if (c < T2) {
      const uint32_t r = c_ref[c], p = c_pos[c], j = c_j[c];
      uint32_t rk = 0;
      for (uint32_t i = 0; i < T2; i++) {
        const uint32_t rr = c_ref[i], pp = c_pos[i], jj = c_j[i];
        rk += (rr < r || (rr == r && (pp < p || (pp == p && jj < j)))) ? 1u : 0u;
      }
      s_ref[rk] = r;
      s_pos[rk] = p;
      s_j[rk] = j;
    }
  }
  __syncwarp();
  // 4. diagonal runs over the sorted postings (Analyser.cpp:2337-2490)
  uint32_t* z = S.t[half][0];
  uint32_t* segmax = S.t[half][1];
  auto brk = [&](int i) -> bool {
    if (i == 0) return true;
    if (s_ref[i] != s_ref[i - 1]) return true;
    return !((uint64_t)s_pos[i - 1] + step == s_pos[i] && s_j[i - 1] + 1 == s_j[i]);
  };
  auto rhead = [&](int i) -> bool { return i == 0 || s_ref[i] != s_ref[i - 1]; };
  unsigned long long B = 0, R = 0;
  for (int s = 0; s < nkw; s++) {
    const int i = hl + 16 * s;
    const bool u = i < (int)T2;
    B |= (unsigned long long)half_bits(__ballot_sync(FULL, u && brk(i)), sh) << (16 * s);
    R |= (unsigned long long)half_bits(__ballot_sync(FULL, u && rhead(i)), sh) << (16 * s);
  }
  const unsigned long long V = T2 >= 64 ? ~0ull : ((1ull << T2) - 1ull);
  const unsigned long long E = T2 ? (((B >> 1) | (1ull << (T2 - 1))) & V) : 0ull;  // run ends
  auto run_start = [&](int i) { return 63 - __clzll(B & upto64(i)); };
  auto seg_end = [&](int h) {  // last slot of the reference segment starting at head h
    const unsigned long long rest = R & ~upto64(h);
    return rest ? (__ffsll(rest) - 2) : ((int)T2 - 1);
  };
  int smax = 0;
  for (int s = 0; s < nkw; s++) {
    const int i = hl + 16 * s;
    if (i < (int)T2 && ((R >> i) & 1ull)) {
      int sm = 0;
      for (unsigned long long m = E & upto64(seg_end(i)) & ~below64(i); m; m &= m - 1ull) {
        const int e = __ffsll(m) - 1;
        sm = max(sm, e - run_start(e) + 1);
      }
      segmax[i] = (uint32_t)sm;
      smax = max(smax, sm);
    }
  }
  int M = smax;
  for (int o = 8; o > 0; o >>= 1) M = max(M, __shfl_xor_sync(FULL, M, o));
  alive = alive && M >= 2;  // Analyser.cpp:2402
  if (!__any_sync(FULL, alive)) return kStrandOk;
  __syncwarp();
  // 5. head/tail extension at every run end of a kept reference (runMax == M)
  for (int s = 0; s < nkw; s++) {
    const int i = hl + 16 * s;
    uint32_t zz = 0;
    if (alive && i < (int)T2 && ((E >> i) & 1ull)) {
      const int h = 63 - __clzll(R & upto64(i));
      if (segmax[h] == (uint32_t)M) {
        const int st = run_start(i);
        const uint32_t ref = s_ref[i];
        const uint32_t sr = s_pos[st], sq = s_j[st] * step;
        const uint32_t lr = s_pos[i] + step, lq = s_j[i] * step + step;
        const uint8_t* rs = ix.bases + ix.ref_off[ref];
        const uint32_t rlen = ix.ref_len[ref];
        const uint32_t tail = tail_walk4(q, rs, L, rlen, lq, lr, k);
        const uint32_t head = head_walk(q, rs, sq, sr, k);
        const uint32_t tot = tail + head + (lq - sq);
        if (tot >= k) zz = ((sq - head) << 16) | tot;
      }
    }
    if (i < (int)T2) z[i] = zz;
  }
  __syncwarp();
  // 6. candidates: reference heads with runMax == M and a run end that scored (T >= k); their
  //    output slots follow from the mask of candidate heads, in ascending refID
  auto is_cand = [&](int h) -> bool {
    if (!alive || h >= (int)T2 || !((R >> h) & 1ull) || segmax[h] != (uint32_t)M) return false;
    const int se = seg_end(h);
    for (int i = h; i <= se; i++)
      if (z[i]) return true;
    return false;
  };
  unsigned long long Sm = 0;
  for (int s = 0; s < nkw; s++) Sm |= (unsigned long long)half_bits(__ballot_sync(FULL, is_cand(hl + 16 * s)), sh) << (16 * s);
  const int n_sc = __popcll(Sm);
  if (__any_sync(FULL, n_sc > kDualC)) return kStrandOverflow;
  //    sums and coverage, one lane per candidate (MatrixCPU.cpp:18-208); the scores from them are
  //    k_finish_dual's (MatrixCPU.cpp:209-212, MatrixResult.cpp:21-29)
  const uint32_t nw = (L + 31) / 32;
  uint32_t* cov = &S.c[0][0][0] + lane * kCovWords;
  mg_candidate* cb = S.cb[half];
  for (int s = 0; s < nkw; s++) {
    const int h = hl + 16 * s;
    if (!((Sm >> h) & 1ull)) continue;
    const int se = seg_end(h);
    for (uint32_t wd = 0; wd < nw; wd++) cov[wd] = 0;
    uint32_t sumc = 0, sumr = 0;
    for (int i = h; i <= se; i++) {
      const uint32_t zz = z[i];
      if (!zz) continue;
      const uint32_t t = zz & 0xFFFFu, a = zz >> 16, b = a + t;
      sumc += t;
      sumr += t * (t + 1) / 2;
      for (uint32_t wd = a >> 5; wd <= (b - 1) >> 5; wd++) {
        const uint32_t w0 = wd * 32;
        const uint32_t lo = a > w0 ? a : w0, up = b < w0 + 32 ? b : w0 + 32;
        const uint32_t n = up - lo;
        cov[wd] |= (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u)) << (lo - w0);
      }
    }
    uint32_t hits = 0;
    for (uint32_t wd = 0; wd < nw; wd++) hits += __popc(cov[wd]);
    cb[__popcll(Sm & below64(h))] = raw_candidate(s_ref[h], sumr, sumc, hits);
  }
  __syncwarp();
  *n_out = (uint32_t)n_sc;
  return kStrandOk;
}

// The dual tier's read result: the raw candidates go to the read's staging slots (or the arena
// when there are more than kSlots) and the read is marked kReadUnscored for k_finish_dual; a read
// without candidates is final here (what write_read_result_s gives with no candidate).
__device__ __forceinline__ void write_read_raw(const BatchDev& b, uint32_t r, uint32_t n0, uint32_t n1,
                                               const mg_candidate* cb0, const mg_candidate* cb1, mg_candidate* stage,
                                               mg_candidate* arena, uint64_t arena_cap, unsigned long long* arena_n,
                                               int* errw) {
  const uint32_t tot = n0 + n1;
  if (tot == 0) {
    b.reads[r] = mg_read_result{-1.0f, 0, 0, 0, 0, 0, 0};
    return;
  }
  uint32_t where = 0;
  uint8_t mark = kReadUnscored;
  mg_candidate* dst = stage + (uint64_t)r * kSlots;
  if (tot > (uint32_t)kSlots) {
    const unsigned long long at = atomicAdd(arena_n, (unsigned long long)tot);
    if (at + tot > arena_cap) {  // the call grows the arena and runs the batch again
      atomicOr(errw, kErrArena);
      dst = nullptr;
      mark = 0;
    } else {
      dst = arena + at;
      where = (uint32_t)at;
    }
  }
  if (dst) {
    for (uint32_t c = 0; c < n0; c++) dst[c] = cb0[c];
    for (uint32_t c = 0; c < n1; c++) dst[n0 + c] = cb1[c];
  }
  b.reads[r] = mg_read_result{-1.0f, where, (uint16_t)n0, (uint16_t)n1, mark, 0, 0};
}

// Read r on the dual path; false when it does not fit (the caller hands it on).
// comp: the block's 256-entry table of complement(upper(byte)), 0 where there is none.
__device__ bool process_read_dual(const DevIndex& ix, const BatchDev& b, uint32_t r, DualSmem& S,
                                  const uint8_t* comp, mg_candidate* stage, mg_candidate* arena, uint64_t arena_cap,
                                  unsigned long long* arena_n, int* errw) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint64_t o0 = b.offs[r];
  const uint64_t Lr = b.offs[r + 1] - o0;
  if (Lr > (uint64_t)kLeanQ) return false;
  const uint32_t L = (uint32_t)Lr;
  const uint8_t* raw = b.bases + o0;
  uint32_t badl = 0;
  for (uint32_t i = lane; i < L; i += 32) {
    S.q[0][i] = upper_dev(raw[i]);
    const uint8_t c = comp[raw[L - 1 - i]];
    badl |= c == 0;
    S.q[1][i] = c;
  }
  if (__any_sync(FULL, badl)) {
    if (lane == 0)
      write_read_result_s(b, r, true, 0, 0, -1.0f, -1.0f, S.cb[0], S.cb[1], stage, arena, arena_cap, arena_n, errw, 0);
    __syncwarp();
    return true;
  }
  __syncwarp();
  uint32_t nh;
  if (dual_strands(ix, L, S, &nh) != kStrandOk) return false;
  const uint32_t n0 = __shfl_sync(FULL, nh, 0), n1 = __shfl_sync(FULL, nh, 16);
  if (lane == 0) write_read_raw(b, r, n0, n1, S.cb[0], S.cb[1], stage, arena, arena_cap, arena_n, errw);
  __syncwarp();
  return true;
}

}  // namespace mg
