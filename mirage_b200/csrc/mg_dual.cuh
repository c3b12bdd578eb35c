// Dual-strand warp path: both strands of a read at once, one half-warp per strand (lanes 0-15
// the forward strand, lanes 16-31 its reverse complement), for the common read with at most 16
// seeds and 32 postings per strand (reads up to 271 bases at k 31, step 15).
//
// The steps are those of lean_strand (mg_lean.cuh) on 16-lane halves: one lane per seed, two
// posting slots per lane, 32-bit per-half masks from full-warp ballots, shuffles of width 16.
// The serial per-posting loops (occurrence filter, rank sort) then cost max(T_fwd, T_rc)
// iterations instead of T_fwd + T_rc, and every lane works on seeds instead of half of them.
// Per-strand values stay in registers or in shared memory indexed by the half (no local arrays).
// A read that does not fit goes to the lean path unchanged.
#pragma once
#include "mg_lean.cuh"

namespace mg {

constexpr int kDualSeeds = 16;  // seeds per strand: one per lane of a half-warp
constexpr int kDualE = 32;      // postings per strand: two slots per lane of a half-warp
constexpr int kDualC = 8;       // scored candidates per strand

// Per-warp shared arrays of the dual path ([half][slot]).
struct DualSmem {
  uint32_t e_ref[2][kDualE];   // posting refID, gather order
  uint32_t e_pos[2][kDualE];   // posting position
  uint32_t e_fj[2][kDualE];    // found index | seed index << 8
  uint32_t s_ref[2][kDualE];   // kept postings sorted by (ref, pos, seed)
  uint32_t s_pos[2][kDualE];
  uint32_t s_j[2][kDualE];
  uint32_t z[2][kDualE];       // at a run end of a candidate: (Start.Q - head) << 16 | T, else 0
  uint32_t segmax[2][kDualE];  // at a reference head: the reference's longest run
  mg_candidate tmp[2][kDualE]; // scored candidate at its head slot
  mg_candidate cb[2][kDualC];  // scored candidates in ascending refID
  uint8_t q[2][kLeanQ];        // strand bases: forward, reverse complement
};

__device__ __forceinline__ uint32_t upto32(int i) {  // bits 0..i
  return i >= 31 ? 0xFFFFFFFFu : ((2u << i) - 1u);
}

// Bits of a full-warp ballot that belong to this lane's half.
__device__ __forceinline__ uint32_t half_bits(uint32_t ballot, int sh) { return (ballot >> sh) & 0xFFFFu; }

// Both strands of one read (bases already in S.q). Warp-uniform return: kStrandOk, or
// kStrandOverflow when either strand does not fit. Each lane receives its half's strand results:
// *n_out scored candidates in S.cb[half] (ascending refID) and the strand's HighestScore.
__device__ int dual_strands(const DevIndex& ix, uint32_t L, DualSmem& S, uint32_t* n_out, float* hi_out,
                            int* err) {
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
  if (ns > (uint32_t)kDualSeeds) return kStrandOverflow;
  // 1. seeds, probe, found list, postings
  uint32_t found = 0, cnt = 0, o0 = 0;
  if ((uint32_t)hl < ns) {
    const uint32_t h = hash28_dev(q + hl * step, ix.hlen);
    o0 = __ldg(ix.dir + h);
    cnt = __ldg(ix.dir + h + 1) - o0;
    found = (cnt > 0 || h == ix.empty_hash) ? 1u : 0u;
  }
  if (__any_sync(FULL, cnt > (uint32_t)kDualE)) return kStrandOverflow;
  const uint32_t fb = half_bits(__ballot_sync(FULL, found), sh);
  const uint32_t f = __popc(fb & ((1u << hl) - 1u));
  uint32_t inc = cnt;
  for (int o = 1; o < 16; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, inc, o, 16);
    if (hl >= o) inc += y;
  }
  const uint32_t T = __shfl_sync(FULL, inc, 15, 16);
  if (__any_sync(FULL, T > (uint32_t)kDualE)) return kStrandOverflow;
  bool alive = T > 0;
  if (!__any_sync(FULL, alive)) return kStrandOk;
  {
    const uint32_t e = inc - cnt;
    for (uint32_t t = 0; t < cnt; t++) {
      const uint2 p = __ldg(ix.post + o0 + t);
      e_ref[e + t] = p.x;
      e_pos[e + t] = p.y;
      e_fj[e + t] = f | ((uint32_t)hl << 8);
    }
  }
  __syncwarp();
  // 2. occurrence filter (Analyser.cpp:2057-2115): per posting, the found indices where its
  //    reference occurs; the longest run of consecutive ones is that reference's occMax
  const int i0 = hl, i1 = hl + 16;
  const bool v0 = (uint32_t)i0 < T, v1 = (uint32_t)i1 < T;
  const uint32_t r0 = v0 ? e_ref[i0] : 0xFFFFFFFFu, r1 = v1 ? e_ref[i1] : 0xFFFFFFFFu;
  uint32_t m0 = 0, m1 = 0;
  for (uint32_t i = 0; i < T; i++) {
    const uint32_t rr = e_ref[i];
    const uint32_t bit = 1u << (e_fj[i] & 0xFFu);
    m0 |= (rr == r0) ? bit : 0u;
    m1 |= (rr == r1) ? bit : 0u;
  }
  const int occ0 = v0 ? longest_run(m0) : 0, occ1 = v1 ? longest_run(m1) : 0;
  int hs = max(occ0, occ1);
  for (int o = 8; o > 0; o >>= 1) hs = max(hs, __shfl_xor_sync(FULL, hs, o));
  // below 2 no reference can reach a diagonal run of 2: no candidate on this strand
  alive = alive && hs >= 2;
  if (!__any_sync(FULL, alive)) return kStrandOk;
  const int keep_min = hs - 1;  // max(1, hs - 1), Analyser.cpp:2115
  const bool k0 = alive && v0 && occ0 >= keep_min, k1 = alive && v1 && occ1 >= keep_min;
  const uint32_t K = half_bits(__ballot_sync(FULL, k0), sh) | (half_bits(__ballot_sync(FULL, k1), sh) << 16);
  const int T2 = __popc(K);
  // 3. rank sort of the kept postings by (ref, pos, seed); the keys are distinct
  {
    const uint32_t p0 = v0 ? e_pos[i0] : 0, p1 = v1 ? e_pos[i1] : 0;
    const uint32_t j0 = v0 ? (e_fj[i0] >> 8) : 0, j1 = v1 ? (e_fj[i1] >> 8) : 0;
    int rk0 = 0, rk1 = 0;
    for (uint32_t m = K; m; m &= m - 1u) {
      const int i = __ffs(m) - 1;
      const uint32_t rr = e_ref[i], pp = e_pos[i], jj = e_fj[i] >> 8;
      rk0 += (rr < r0 || (rr == r0 && (pp < p0 || (pp == p0 && jj < j0)))) ? 1 : 0;
      rk1 += (rr < r1 || (rr == r1 && (pp < p1 || (pp == p1 && jj < j1)))) ? 1 : 0;
    }
    __syncwarp();
    if (k0) {
      s_ref[rk0] = r0;
      s_pos[rk0] = p0;
      s_j[rk0] = j0;
    }
    if (k1) {
      s_ref[rk1] = r1;
      s_pos[rk1] = p1;
      s_j[rk1] = j1;
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
  const bool u0 = i0 < T2, u1 = i1 < T2;
  const uint32_t B = half_bits(__ballot_sync(FULL, u0 && brk(i0)), sh) |
                     (half_bits(__ballot_sync(FULL, u1 && brk(i1)), sh) << 16);
  const uint32_t R = half_bits(__ballot_sync(FULL, u0 && rhead(i0)), sh) |
                     (half_bits(__ballot_sync(FULL, u1 && rhead(i1)), sh) << 16);
  const uint32_t V = T2 >= 32 ? 0xFFFFFFFFu : ((1u << T2) - 1u);
  const uint32_t E = T2 ? (((B >> 1) | (1u << (T2 - 1))) & V) : 0u;  // run ends
  auto run_start = [&](int i) { return 31 - __clz(B & upto32(i)); };
  auto seg_end = [&](int h) {  // last slot of the reference segment starting at head h
    const uint32_t rest = R & ~upto32(h);
    return rest ? (__ffs(rest) - 2) : (T2 - 1);
  };
  int sm0 = 0, sm1 = 0;
  if (u0 && ((R >> i0) & 1u)) {
    const int se = seg_end(i0);
    for (int i = i0; i <= se; i++)
      if ((E >> i) & 1u) sm0 = max(sm0, i - run_start(i) + 1);
    segmax[i0] = sm0;
  }
  if (u1 && ((R >> i1) & 1u)) {
    const int se = seg_end(i1);
    for (int i = i1; i <= se; i++)
      if ((E >> i) & 1u) sm1 = max(sm1, i - run_start(i) + 1);
    segmax[i1] = sm1;
  }
  int M = max(sm0, sm1);
  for (int o = 8; o > 0; o >>= 1) M = max(M, __shfl_xor_sync(FULL, M, o));
  alive = alive && M >= 2;  // Analyser.cpp:2402
  if (!__any_sync(FULL, alive)) return kStrandOk;
  __syncwarp();
  // 5. head/tail extension at every run end of a kept reference (runMax == M)
#pragma unroll 1
  for (int s = 0; s < 2; s++) {
    const int i = hl + 16 * s;
    uint32_t zz = 0;
    if (alive && i < T2 && ((E >> i) & 1u)) {
      const int h = 31 - __clz(R & upto32(i));
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
  //    (MatrixCPU.cpp:18-214)
  const uint32_t nw = (L + 31) / 32;
  bool sc0 = false, sc1 = false;
#pragma unroll 1
  for (int s = 0; s < 2; s++) {
    const int h = hl + 16 * s;
    bool scored = false;
    if (alive && h < T2 && ((R >> h) & 1u) && segmax[h] == (uint32_t)M) {
      const int se = seg_end(h);
      uint32_t sumc = 0, sumr = 0, hits = 0;
      for (int i = h; i <= se; i++) {
        const uint32_t zz = z[i];
        if (zz) {
          const uint32_t t = zz & 0xFFFFu;
          sumc += t;
          sumr += t * (t + 1) / 2;
        }
      }
      if (sumc) {
        for (uint32_t wd = 0; wd < nw; wd++) {
          uint32_t bits = 0;
          const uint32_t w0 = wd * 32, w1 = w0 + 32;
          for (int i = h; i <= se; i++) {
            const uint32_t zz = z[i];
            if (!zz) continue;
            const uint32_t a = zz >> 16, b = a + (zz & 0xFFFFu);
            const uint32_t lo = a > w0 ? a : w0, up = b < w1 ? b : w1;
            if (lo < up) {
              const uint32_t n = up - lo;
              bits |= (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u)) << (lo - w0);
            }
          }
          hits += __popc(bits);
        }
        float sc, pc;
        final_score(sumr, sumc, hits, L, &sc, &pc);
        const uint32_t cref = s_ref[h];
        const float rl = relative_score(ix, __uint2float_rn(L), __uint2float_rn(ix.ref_len[cref]), sc, err);
        tmp[h] = mg_candidate{cref, rl, sc, pc};
        scored = true;
      }
    }
    if (s == 0) sc0 = scored;
    else sc1 = scored;
  }
  // 7. scored candidates in ascending refID (= ascending head slot)
  const uint32_t Sm = half_bits(__ballot_sync(FULL, sc0), sh) | (half_bits(__ballot_sync(FULL, sc1), sh) << 16);
  const int n_sc = __popc(Sm);
  if (__any_sync(FULL, n_sc > kDualC)) return kStrandOverflow;
  __syncwarp();
  mg_candidate* cb = S.cb[half];
  float hi = -1.0f;
  if (sc0) {
    const mg_candidate c = tmp[i0];
    cb[__popc(Sm & ((1u << i0) - 1u))] = c;
    hi = fmaxf(hi, c.rel);
  }
  if (sc1) {
    const mg_candidate c = tmp[i1];
    cb[__popc(Sm & ((1u << i1) - 1u))] = c;
    hi = fmaxf(hi, c.rel);
  }
  for (int o = 8; o > 0; o >>= 1) hi = fmaxf(hi, __shfl_xor_sync(FULL, hi, o));
  __syncwarp();
  *n_out = (uint32_t)n_sc;
  *hi_out = hi;
  return kStrandOk;
}

// Read r on the dual path; false when it does not fit (the caller hands it to the lean path).
__device__ bool process_read_dual(const DevIndex& ix, const BatchDev& b, uint32_t r, DualSmem& S,
                                  mg_candidate* stage, mg_candidate* arena, uint64_t arena_cap,
                                  unsigned long long* arena_n, int* errw) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint64_t o0 = b.offs[r];
  const uint64_t Lr = b.offs[r + 1] - o0;
  if (Lr > (uint64_t)kLeanQ) return false;
  const uint32_t L = (uint32_t)Lr;
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  if (L > k && (L - k + step - 1) / step > (uint32_t)kDualSeeds) return false;
  const uint8_t* raw = b.bases + o0;
  uint32_t badl = 0;
  for (uint32_t i = lane; i < L; i += 32) {
    S.q[0][i] = upper_dev(raw[i]);
    const uint8_t c = complement_dev(upper_dev(raw[L - 1 - i]));
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
  if (dual_strands(ix, L, S, &nh, &hh, &err) != kStrandOk) return false;
  err = (int)__reduce_or_sync(FULL, (unsigned)err);
  const uint32_t n0 = __shfl_sync(FULL, nh, 0), n1 = __shfl_sync(FULL, nh, 16);
  const float h0 = __shfl_sync(FULL, hh, 0), h1 = __shfl_sync(FULL, hh, 16);
  if (lane == 0)
    write_read_result_s(b, r, false, n0, n1, h0, h1, S.cb[0], S.cb[1], stage, arena, arena_cap, arena_n, errw, err);
  __syncwarp();
  return true;
}

}  // namespace mg
