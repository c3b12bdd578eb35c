// Dual-strand warp path: both strands of a read at once, one half-warp per strand (lanes 0-15
// the forward strand, lanes 16-31 its reverse complement).
//
// The steps are those of lean_strand (mg_lean.cuh) on 16-lane halves: SPL seeds and SLOTS
// posting slots per lane (seed j = lane + 16 s, posting slot i = lane + 16 s), per-half bit masks
// assembled from full-warp ballots, shuffles of width 16. Two shapes run as two kernels:
//   <1, 2>  up to 16 seeds and 32 postings per strand: the common read (up to 271 bases at k 31)
//   <2, 4>  up to 32 seeds and 64 postings per strand: the rest of the reads up to 320 bases
// The serial per-posting loops (occurrence filter, rank sort) then cost max(T_fwd, T_rc)
// iterations instead of T_fwd + T_rc. Per-slot values live in registers (fully unrolled slot
// loops) or in shared memory indexed by the half; nothing is indexed dynamically in local memory.
#pragma once
#include <type_traits>

#include "mg_lean.cuh"

namespace mg {

constexpr int kDualC = 8;                 // scored candidates per strand
constexpr int kCovWords = kLeanQ / 32;    // coverage bitmap words per lane

// Per-warp shared arrays of the dual path ([half][slot]).
template <int SLOTS>
struct DualSmem {
  static constexpr int E = 16 * SLOTS;
  uint32_t e_ref[2][E];    // posting refID, gather order
  uint32_t e_pos[2][E];    // posting position
  uint32_t e_fj[2][E];     // found index | seed index << 8
  uint32_t s_ref[2][E];    // kept postings sorted by (ref, pos, seed)
  uint32_t s_pos[2][E];
  uint32_t s_j[2][E];
  uint32_t z[2][E];        // at a run end of a candidate: (Start.Q - head) << 16 | T, else 0
  uint32_t segmax[2][E];   // at a reference head: the reference's longest run
  mg_candidate tmp[2][E];  // scored candidate at its head slot
  mg_candidate cb[2][kDualC];  // scored candidates in ascending refID
  uint32_t cov[32][kCovWords]; // per-lane query coverage bitmap of the candidate being scored
  uint8_t q[2][kLeanQ];    // strand bases: forward, reverse complement
};

template <int SLOTS>
using DualMask = typename std::conditional<(SLOTS > 2), unsigned long long, uint32_t>::type;

template <typename Mk>
__device__ __forceinline__ Mk mk_upto(int i) {  // bits 0..i
  constexpr int W = (int)sizeof(Mk) * 8;
  return i >= W - 1 ? ~(Mk)0 : (((Mk)2 << i) - (Mk)1);
}
template <typename Mk>
__device__ __forceinline__ Mk mk_below(int i) {  // bits 0..i-1
  return i <= 0 ? (Mk)0 : mk_upto<Mk>(i - 1);
}
template <typename Mk>
__device__ __forceinline__ int mk_clz(Mk x) {
  if constexpr (sizeof(Mk) == 8) return __clzll((long long)x);
  else return __clz((int)x);
}
template <typename Mk>
__device__ __forceinline__ int mk_ffs(Mk x) {
  if constexpr (sizeof(Mk) == 8) return __ffsll((long long)x);
  else return __ffs((int)x);
}
template <typename Mk>
__device__ __forceinline__ int mk_popc(Mk x) {
  if constexpr (sizeof(Mk) == 8) return __popcll(x);
  else return __popc(x);
}

// Bits of a full-warp ballot that belong to this lane's half.
__device__ __forceinline__ uint32_t half_bits(uint32_t ballot, int sh) { return (ballot >> sh) & 0xFFFFu; }

// Per-half mask of slot flags: bit (lane + 16 s) = x[s].
template <int SLOTS>
__device__ __forceinline__ DualMask<SLOTS> slot_mask(const bool (&x)[SLOTS], int sh) {
  DualMask<SLOTS> m = 0;
#pragma unroll
  for (int s = 0; s < SLOTS; s++)
    m |= (DualMask<SLOTS>)half_bits(__ballot_sync(0xffffffffu, x[s]), sh) << (16 * s);
  return m;
}

// Both strands of one read (bases already in S.q). Warp-uniform return: kStrandOk, or
// kStrandOverflow when either strand does not fit this shape. Each lane receives its half's
// strand results: *n_out scored candidates in S.cb[half] (ascending refID) and the strand's
// HighestScore.
template <int SPL, int SLOTS>
__device__ int dual_strands(const DevIndex& ix, uint32_t L, DualSmem<SLOTS>& S, uint32_t* n_out, float* hi_out,
                            int* err) {
  using Mk = DualMask<SLOTS>;
  constexpr int E = 16 * SLOTS, NSEED = 16 * SPL, W = (int)sizeof(Mk) * 8;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15, sh = half * 16;
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  const uint8_t* q = S.q[half];
  uint32_t* e_ref = S.e_ref[half];
  uint32_t* e_pos = S.e_pos[half];
  uint32_t* e_fj = S.e_fj[half];
  uint32_t* s_ref = S.s_ref[half];
  uint32_t* s_pos = S.s_pos[half];
  uint32_t* s_j = S.s_j[half];
  uint32_t* z = S.z[half];
  uint32_t* segmax = S.segmax[half];
  mg_candidate* tmp = S.tmp[half];
  *n_out = 0;
  *hi_out = -1.0f;
  if (L <= k) return kStrandOk;
  const uint32_t ns = (L - k + step - 1) / step;
  if (ns > (uint32_t)NSEED) return kStrandOverflow;
  // 1. seeds, probe, found list, postings (seed j = hl + 16 s)
  uint32_t cnt[SPL], o0[SPL];
  bool fnd[SPL];
  bool big = false;
#pragma unroll
  for (int s = 0; s < SPL; s++) {
    const uint32_t j = hl + 16 * s;
    cnt[s] = 0;
    o0[s] = 0;
    fnd[s] = false;
    if (j < ns) {
      const uint32_t h = hash28_dev(q + j * step, ix.hlen);
      o0[s] = __ldg(ix.dir + h);
      cnt[s] = __ldg(ix.dir + h + 1) - o0[s];
      fnd[s] = cnt[s] > 0 || h == ix.empty_hash;
    }
    big |= cnt[s] > (uint32_t)E;
  }
  if (__any_sync(FULL, big)) return kStrandOverflow;
  uint32_t fb = 0;
#pragma unroll
  for (int s = 0; s < SPL; s++) fb |= half_bits(__ballot_sync(FULL, fnd[s]), sh) << (16 * s);
  uint32_t inc[SPL], T = 0;
#pragma unroll
  for (int s = 0; s < SPL; s++) {
    uint32_t x = cnt[s];
    for (int o = 1; o < 16; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, x, o, 16);
      if (hl >= o) x += y;
    }
    inc[s] = x + T;
    T += __shfl_sync(FULL, x, 15, 16);
  }
  if (__any_sync(FULL, T > (uint32_t)E)) return kStrandOverflow;
  bool alive = T > 0;
  if (!__any_sync(FULL, alive)) return kStrandOk;
#pragma unroll
  for (int s = 0; s < SPL; s++) {
    const uint32_t j = hl + 16 * s;
    const uint32_t f = __popc(fb & ((1u << j) - 1u));
    const uint32_t e = inc[s] - cnt[s];
    for (uint32_t t = 0; t < cnt[s]; t++) {
      const uint2 p = __ldg(ix.post + o0[s] + t);
      e_ref[e + t] = p.x;
      e_pos[e + t] = p.y;
      e_fj[e + t] = f | (j << 8);
    }
  }
  __syncwarp();
  // 2. occurrence filter (Analyser.cpp:2057-2115): per posting, the found indices where its
  //    reference occurs; the longest run of consecutive ones is that reference's occMax
  uint32_t r[SLOTS], m[SLOTS];
  bool v[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) {
    const uint32_t i = hl + 16 * s;
    v[s] = i < T;
    r[s] = v[s] ? e_ref[i] : 0xFFFFFFFFu;
    m[s] = 0;
  }
  for (uint32_t i = 0; i < T; i++) {
    const uint32_t rr = e_ref[i];
    const uint32_t bit = 1u << (e_fj[i] & 0xFFu);
#pragma unroll
    for (int s = 0; s < SLOTS; s++) m[s] |= (rr == r[s]) ? bit : 0u;
  }
  int occ[SLOTS];
  int hs = 0;
#pragma unroll
  for (int s = 0; s < SLOTS; s++) {
    occ[s] = v[s] ? longest_run(m[s]) : 0;
    hs = max(hs, occ[s]);
  }
  for (int o = 8; o > 0; o >>= 1) hs = max(hs, __shfl_xor_sync(FULL, hs, o));
  // below 2 no reference can reach a diagonal run of 2: no candidate on this strand
  alive = alive && hs >= 2;
  if (!__any_sync(FULL, alive)) return kStrandOk;
  const int keep_min = hs - 1;  // max(1, hs - 1), Analyser.cpp:2115
  bool kp[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) kp[s] = alive && v[s] && occ[s] >= keep_min;
  const Mk K = slot_mask<SLOTS>(kp, sh);
  const int T2 = mk_popc(K);
  // 3. rank sort of the kept postings by (ref, pos, seed); the keys are distinct
  {
    uint32_t p[SLOTS], jj[SLOTS];
    int rk[SLOTS];
#pragma unroll
    for (int s = 0; s < SLOTS; s++) {
      const uint32_t i = hl + 16 * s;
      p[s] = v[s] ? e_pos[i] : 0;
      jj[s] = v[s] ? (e_fj[i] >> 8) : 0;
      rk[s] = 0;
    }
    for (Mk mm = K; mm; mm &= mm - (Mk)1) {
      const int i = mk_ffs(mm) - 1;
      const uint32_t rr = e_ref[i], pp = e_pos[i], qj = e_fj[i] >> 8;
#pragma unroll
      for (int s = 0; s < SLOTS; s++)
        rk[s] += (rr < r[s] || (rr == r[s] && (pp < p[s] || (pp == p[s] && qj < jj[s])))) ? 1 : 0;
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < SLOTS; s++)
      if (kp[s]) {
        s_ref[rk[s]] = r[s];
        s_pos[rk[s]] = p[s];
        s_j[rk[s]] = jj[s];
      }
  }
  __syncwarp();
  // 4. diagonal runs over the sorted postings (Analyser.cpp:2337-2490)
  auto brk = [&](int i) -> bool {
    if (i == 0) return true;
    if (s_ref[i] != s_ref[i - 1]) return true;
    return !((uint64_t)s_pos[i - 1] + step == s_pos[i] && s_j[i - 1] + 1 == s_j[i]);
  };
  auto rhead = [&](int i) -> bool { return i == 0 || s_ref[i] != s_ref[i - 1]; };
  bool bb[SLOTS], rh[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) {
    const int i = hl + 16 * s;
    const bool u = i < T2;
    bb[s] = u && brk(i);
    rh[s] = u && rhead(i);
  }
  const Mk B = slot_mask<SLOTS>(bb, sh), R = slot_mask<SLOTS>(rh, sh);
  const Mk V = T2 >= W ? ~(Mk)0 : (((Mk)1 << T2) - (Mk)1);
  const Mk Ee = T2 ? (((B >> 1) | ((Mk)1 << (T2 - 1))) & V) : (Mk)0;  // run ends
  auto run_start = [&](int i) { return W - 1 - mk_clz<Mk>(B & mk_upto<Mk>(i)); };
  auto seg_end = [&](int h) {  // last slot of the reference segment starting at head h
    const Mk rest = R & ~mk_upto<Mk>(h);
    return rest ? (mk_ffs<Mk>(rest) - 2) : (T2 - 1);
  };
  int smax = 0;
#pragma unroll
  for (int s = 0; s < SLOTS; s++) {
    const int i = hl + 16 * s;
    if (i < T2 && ((R >> i) & (Mk)1)) {
      const int se = seg_end(i);
      int sm = 0;
      for (Mk mm = Ee & mk_upto<Mk>(se) & ~mk_below<Mk>(i); mm; mm &= mm - (Mk)1) {
        const int e = mk_ffs<Mk>(mm) - 1;
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
#pragma unroll 1
  for (int s = 0; s < SLOTS; s++) {
    const int i = hl + 16 * s;
    uint32_t zz = 0;
    if (alive && i < T2 && ((Ee >> i) & (Mk)1)) {
      const int h = W - 1 - mk_clz<Mk>(R & mk_upto<Mk>(i));
      if (segmax[h] == (uint32_t)M) {
        const int st = run_start(i);
        const uint32_t ref = s_ref[i];
        const uint32_t sr = s_pos[st], sq = s_j[st] * step;
        const uint32_t lr = s_pos[i] + step, lq = s_j[i] * step + step;
        const uint8_t* rs = ix.bases + ix.ref_off[ref];
        const uint32_t rlen = ix.ref_len[ref];
        const uint32_t tail = tail_walk(q, rs, L, rlen, lq, lr, k);
        const uint32_t head = head_walk(q, rs, sq, sr, k);
        const uint32_t tot = tail + head + (lq - sq);
        if (tot >= k) zz = ((sq - head) << 16) | tot;
      }
    }
    z[i] = zz;
  }
  __syncwarp();
  // 6. one lane per candidate reference (a head with runMax == M): sums, coverage, scores
  //    (MatrixCPU.cpp:18-214); coverage as a bitmap of query positions
  const uint32_t nw = (L + 31) / 32;
  uint32_t* cov = S.cov[lane];
  uint32_t scm = 0;
#pragma unroll 1
  for (int s = 0; s < SLOTS; s++) {
    const int h = hl + 16 * s;
    if (alive && h < T2 && ((R >> h) & (Mk)1) && segmax[h] == (uint32_t)M) {
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
      if (sumc) {
        uint32_t hits = 0;
        for (uint32_t wd = 0; wd < nw; wd++) hits += __popc(cov[wd]);
        float sc, pc;
        final_score(sumr, sumc, hits, L, &sc, &pc);
        const uint32_t cref = s_ref[h];
        const float rl = relative_score_tab(ix, L, ix.ref_len[cref], sc, err);
        tmp[h] = mg_candidate{cref, rl, sc, pc};
        scm |= 1u << s;
      }
    }
  }
  // 7. scored candidates in ascending refID (= ascending head slot)
  bool scd[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) scd[s] = (scm >> s) & 1u;
  const Mk Sm = slot_mask<SLOTS>(scd, sh);
  const int n_sc = mk_popc(Sm);
  if (__any_sync(FULL, n_sc > kDualC)) return kStrandOverflow;
  __syncwarp();
  mg_candidate* cb = S.cb[half];
  float hi = -1.0f;
#pragma unroll
  for (int s = 0; s < SLOTS; s++)
    if (scd[s]) {
      const int i = hl + 16 * s;
      const mg_candidate c = tmp[i];
      cb[mk_popc(Sm & mk_below<Mk>(i))] = c;
      hi = fmaxf(hi, c.rel);
    }
  for (int o = 8; o > 0; o >>= 1) hi = fmaxf(hi, __shfl_xor_sync(FULL, hi, o));
  __syncwarp();
  *n_out = (uint32_t)n_sc;
  *hi_out = hi;
  return kStrandOk;
}

// Read r on the dual path; false when it does not fit this shape (the caller hands it on).
// comp: the block's 256-entry table of complement(upper(byte)), 0 where there is none.
template <int SPL, int SLOTS>
__device__ bool process_read_dual(const DevIndex& ix, const BatchDev& b, uint32_t r, DualSmem<SLOTS>& S,
                                  const uint8_t* comp, mg_candidate* stage, mg_candidate* arena, uint64_t arena_cap,
                                  unsigned long long* arena_n, int* errw) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint64_t o0 = b.offs[r];
  const uint64_t Lr = b.offs[r + 1] - o0;
  if (Lr > (uint64_t)kLeanQ) return false;
  const uint32_t L = (uint32_t)Lr;
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  if (L > k && (L - k + step - 1) / step > (uint32_t)(16 * SPL)) return false;
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
  float hh;
  int err = 0;
  if (dual_strands<SPL, SLOTS>(ix, L, S, &nh, &hh, &err) != kStrandOk) return false;
  err = (int)__reduce_or_sync(FULL, (unsigned)err);
  const uint32_t n0 = __shfl_sync(FULL, nh, 0), n1 = __shfl_sync(FULL, nh, 16);
  const float h0 = __shfl_sync(FULL, hh, 0), h1 = __shfl_sync(FULL, hh, 16);
  if (lane == 0)
    write_read_result_s(b, r, false, n0, n1, h0, h1, S.cb[0], S.cb[1], stage, arena, arena_cap, arena_n, errw, err);
  __syncwarp();
  return true;
}

}  // namespace mg
