// Lean warp path for the common read (<= 320 bases, <= 32 seeds, <= 64 postings per strand):
// the same steps as process_strand (mg_kernels.cuh) with the per-entry work held in registers
// and 64-bit ballot masks instead of sorts and scans over shared arrays.
//
//   seeds / probe          one lane per seed; found index = popc of the found ballot below it
//   occurrence filter      per posting, the bitmask of found indices where its reference occurs;
//                          the longest run of set bits is that reference's occMax
//                          (Analyser.cpp:2057-2115)
//   sort (ref, pos, q)     rank sort of the <= 64 kept postings (keys are distinct)
//   diagonal runs          run starts as a 64-bit mask; run length = i - last start + 1
//                          (Analyser.cpp:2337-2490)
//   scoring                one lane per candidate reference (MatrixCPU.cpp:18-214)
#pragma once
#include "mg_kernels.cuh"

namespace mg {

constexpr int kLeanQ = 320;
constexpr int kLeanE = 64;

// Per-warp shared arrays of the lean path (carved from the warp tier's workspace).
struct LeanWS {
  uint32_t* e_ref;   // [64] posting refID, gather order
  uint32_t* e_pos;   // [64] posting position
  uint32_t* e_fj;    // [64] found index | seed index << 8
  uint32_t* s_ref;   // [64] kept postings sorted by (ref, pos, q)
  uint32_t* s_pos;   // [64]
  uint32_t* s_j;     // [64] seed index (query position / step)
  uint32_t* z;       // [64] at a run end of a candidate: (Start.Q - head) << 16 | T, else 0
  uint32_t* segmax;  // [64] at a reference head: the reference's longest run
};

__device__ __forceinline__ uint64_t ballot64(bool lo, bool hi) {
  return (uint64_t)__ballot_sync(0xffffffffu, lo) | ((uint64_t)__ballot_sync(0xffffffffu, hi) << 32);
}
__device__ __forceinline__ uint64_t upto(int i) {  // bits 0..i
  return i >= 63 ? ~0ull : ((2ull << i) - 1ull);
}
__device__ __forceinline__ int longest_run(uint32_t m) {
  int r = 0;
  while (m) {
    m &= m >> 1;
    r++;
  }
  return r;
}

// One strand (bases already in q). Returns kStrandOk or kStrandOverflow; scored candidates in
// ascending refID go to cb[0..*n_out).
__device__ int lean_strand(const DevIndex& ix, const uint8_t* q, uint32_t L, const LeanWS& w, mg_candidate* cb,
                           int cap, uint32_t* n_out, float* highest, int* err) {
  const int lane = threadIdx.x & 31;
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  *n_out = 0;
  *highest = -1.0f;
  if (L <= k) return kStrandOk;
  const uint32_t ns = (L - k + step - 1) / step;
  if (ns > 32) return kStrandOverflow;
  // 1. seeds, probe, found list, postings
  uint32_t found = 0, cnt = 0, o0 = 0;
  if ((uint32_t)lane < ns) {
    const uint32_t h = hash28_dev(q + lane * step, ix.hlen);
    o0 = __ldg(ix.dir + h);
    cnt = __ldg(ix.dir + h + 1) - o0;
    found = (cnt > 0 || h == ix.empty_hash) ? 1u : 0u;
  }
  const uint32_t fb = __ballot_sync(0xffffffffu, found);
  const uint32_t f = __popc(fb & ((1u << lane) - 1u));
  uint32_t inc = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  const uint32_t T = __shfl_sync(0xffffffffu, inc, 31);
  if (T > (uint32_t)kLeanE) return kStrandOverflow;
  if (T == 0) return kStrandOk;
  {
    const uint32_t e = inc - cnt;
    for (uint32_t t = 0; t < cnt; t++) {
      const uint2 p = __ldg(ix.post + o0 + t);
      w.e_ref[e + t] = p.x;
      w.e_pos[e + t] = p.y;
      w.e_fj[e + t] = f | ((uint32_t)lane << 8);
    }
  }
  __syncwarp();
  // 2. occurrence filter: found-index mask per posting's reference, longest run = occMax
  const int i0 = lane, i1 = lane + 32;
  const bool v0 = (uint32_t)i0 < T, v1 = (uint32_t)i1 < T;
  const uint32_t r0 = v0 ? w.e_ref[i0] : 0xFFFFFFFFu, r1 = v1 ? w.e_ref[i1] : 0xFFFFFFFFu;
  uint32_t m0 = 0, m1 = 0;
  for (uint32_t i = 0; i < T; i++) {
    const uint32_t rr = w.e_ref[i];
    const uint32_t bit = 1u << (w.e_fj[i] & 0xFFu);
    m0 |= (rr == r0) ? bit : 0u;
    m1 |= (rr == r1) ? bit : 0u;
  }
  const int occ0 = v0 ? longest_run(m0) : 0, occ1 = v1 ? longest_run(m1) : 0;
  int hs = max(occ0, occ1);
  for (int o = 16; o > 0; o >>= 1) hs = max(hs, __shfl_xor_sync(0xffffffffu, hs, o));
  // highestSuccesive only grows on a continued occurrence; below 2 no reference can reach a
  // diagonal run of 2 (a run of m seeds needs m consecutive found indices), so no candidate
  if (hs < 2) return kStrandOk;
  const int keep_min = hs - 1;  // max(1, hs - 1), Analyser.cpp:2115
  const bool k0 = v0 && occ0 >= keep_min, k1 = v1 && occ1 >= keep_min;
  const uint64_t K = ballot64(k0, k1);
  const int T2 = __popcll(K);
  // 3. rank sort of the kept postings by (ref, pos, q)
  {
    const uint32_t p0 = v0 ? w.e_pos[i0] : 0, p1 = v1 ? w.e_pos[i1] : 0;
    const uint32_t j0 = v0 ? (w.e_fj[i0] >> 8) : 0, j1 = v1 ? (w.e_fj[i1] >> 8) : 0;
    int rk0 = 0, rk1 = 0;
    for (uint32_t i = 0; i < T; i++) {
      if (!((K >> i) & 1ull)) continue;
      const uint32_t rr = w.e_ref[i], pp = w.e_pos[i], jj = w.e_fj[i] >> 8;
      rk0 += (rr < r0 || (rr == r0 && (pp < p0 || (pp == p0 && jj < j0)))) ? 1 : 0;
      rk1 += (rr < r1 || (rr == r1 && (pp < p1 || (pp == p1 && jj < j1)))) ? 1 : 0;
    }
    __syncwarp();
    if (k0) {
      w.s_ref[rk0] = r0;
      w.s_pos[rk0] = p0;
      w.s_j[rk0] = j0;
    }
    if (k1) {
      w.s_ref[rk1] = r1;
      w.s_pos[rk1] = p1;
      w.s_j[rk1] = j1;
    }
  }
  __syncwarp();
  // 4. diagonal runs over the sorted postings
  auto brk = [&](int i) -> bool {
    if (i == 0) return true;
    if (w.s_ref[i] != w.s_ref[i - 1]) return true;
    return !((uint64_t)w.s_pos[i - 1] + step == w.s_pos[i] && w.s_j[i - 1] + 1 == w.s_j[i]);
  };
  auto rhead = [&](int i) -> bool { return i == 0 || w.s_ref[i] != w.s_ref[i - 1]; };
  const bool u0 = i0 < T2, u1 = i1 < T2;
  const uint64_t B = ballot64(u0 && brk(i0), u1 && brk(i1));
  const uint64_t R = ballot64(u0 && rhead(i0), u1 && rhead(i1));
  const uint64_t V = T2 >= 64 ? ~0ull : ((1ull << T2) - 1ull);
  const uint64_t E = ((B >> 1) | (1ull << (T2 - 1))) & V;  // run ends
  auto run_start = [&](int i) { return 63 - __clzll(B & upto(i)); };
  auto seg_end = [&](int h) {  // last position of the reference segment starting at head h
    const uint64_t rest = R & ~upto(h);
    return rest ? (__ffsll(rest) - 2) : (T2 - 1);
  };
  // longest run per reference (head lanes walk their segment's run ends)
  int sm0 = 0, sm1 = 0;
  if (u0 && ((R >> i0) & 1ull)) {
    const int se = seg_end(i0);
    for (int i = i0; i <= se; i++)
      if ((E >> i) & 1ull) sm0 = max(sm0, i - run_start(i) + 1);
    w.segmax[i0] = sm0;
  }
  if (u1 && ((R >> i1) & 1ull)) {
    const int se = seg_end(i1);
    for (int i = i1; i <= se; i++)
      if ((E >> i) & 1ull) sm1 = max(sm1, i - run_start(i) + 1);
    w.segmax[i1] = sm1;
  }
  int M = max(sm0, sm1);
  for (int o = 16; o > 0; o >>= 1) M = max(M, __shfl_xor_sync(0xffffffffu, M, o));
  if (M < 2) return kStrandOk;  // Analyser.cpp:2402
  __syncwarp();
  // 5. head/tail extension at every run end of a kept reference (runMax == M)
  for (int s = 0; s < 2; s++) {
    const int i = lane + 32 * s;
    uint32_t zz = 0;
    if (i < T2 && ((E >> i) & 1ull)) {
      const int h = 63 - __clzll(R & upto(i));
      if (w.segmax[h] == (uint32_t)M) {
        const int st = run_start(i);
        const uint32_t ref = w.s_ref[i];
        const uint32_t sr = w.s_pos[st], sq = w.s_j[st] * step;
        const uint32_t lr = w.s_pos[i] + step, lq = w.s_j[i] * step + step;
        const uint8_t* rs = ix.bases + ix.ref_off[ref];
        const uint32_t rlen = ix.ref_len[ref];
        const uint32_t tail = tail_walk(q, rs, L, rlen, lq, lr, k);
        const uint32_t head = head_walk(q, rs, sq, sr, k);
        const uint32_t tot = tail + head + (lq - sq);
        if (tot >= k) zz = ((sq - head) << 16) | tot;
      }
    }
    if (i < 64) w.z[i] = zz;
  }
  __syncwarp();
  // 6. one lane per candidate reference (a head with runMax == M): sums, coverage, scores
  const uint32_t nw = (L + 31) / 32;
  float sc[2] = {-2.0f, -2.0f}, pc[2] = {0.0f, 0.0f}, rl[2] = {-1.0f, -1.0f};
  bool scored[2] = {false, false};
  uint32_t cref[2] = {0, 0};
  for (int s = 0; s < 2; s++) {
    const int h = lane + 32 * s;
    if (h >= T2 || !((R >> h) & 1ull) || w.segmax[h] != (uint32_t)M) continue;
    const int se = seg_end(h);
    uint32_t sumc = 0, sumr = 0, hits = 0;
    for (int i = h; i <= se; i++) {
      const uint32_t zz = w.z[i];
      if (zz) {
        const uint32_t t = zz & 0xFFFFu;
        sumc += t;
        sumr += t * (t + 1) / 2;
      }
    }
    cref[s] = w.s_ref[h];
    if (sumc == 0) continue;
    for (uint32_t wd = 0; wd < nw; wd++) {
      uint32_t bits = 0;
      const uint32_t w0 = wd * 32, w1 = w0 + 32;
      for (int i = h; i <= se; i++) {
        const uint32_t zz = w.z[i];
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
    final_score(sumr, sumc, hits, L, &sc[s], &pc[s]);
    rl[s] = relative_score(ix, __uint2float_rn(L), __uint2float_rn(ix.ref_len[cref[s]]), sc[s], err);
    scored[s] = true;
  }
  // 7. scored candidates in ascending refID (= ascending head position)
  const uint64_t S = ballot64(scored[0], scored[1]);
  const int n_sc = __popcll(S);
  if (n_sc > cap) return kStrandOverflow;
  float hi = -1.0f;
  for (int s = 0; s < 2; s++) {
    if (!scored[s]) continue;
    const int h = lane + 32 * s;
    const int at = __popcll(S & (h ? upto(h - 1) : 0ull));  // scored heads before h
    cb[at] = mg_candidate{cref[s], rl[s], sc[s], pc[s]};
    hi = fmaxf(hi, rl[s]);
  }
  for (int o = 16; o > 0; o >>= 1) hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  __syncwarp();
  *n_out = (uint32_t)n_sc;
  *highest = hi;
  return kStrandOk;
}

// Both strands of read r on the lean path; false when a strand does not fit it (the caller
// then runs the general path). q: kLeanQ bytes of shared memory for the strand bases.
__device__ bool process_read_lean(const DevIndex& ix, const BatchDev& b, uint32_t r, uint8_t* q, const LeanWS& w,
                                  mg_candidate* const* cb, int cap, mg_candidate* stage, mg_candidate* arena,
                                  uint64_t arena_cap, unsigned long long* arena_n, int* errw) {
  const int lane = threadIdx.x & 31;
  const uint64_t o0 = b.offs[r];
  const uint64_t Lr = b.offs[r + 1] - o0;
  if (Lr > (uint64_t)kLeanQ) return false;
  const uint32_t L = (uint32_t)Lr;
  const uint8_t* raw = b.bases + o0;
  int err = 0;
  uint32_t n[2] = {0, 0};
  float h[2] = {-1.0f, -1.0f};
  bool bad = false;
  for (int strand = 0; strand < 2; strand++) {
    uint32_t badl = 0;
    for (uint32_t i = lane; i < L; i += 32) {
      uint8_t c;
      if (strand == 0) {
        c = upper_dev(raw[i]);
      } else {
        c = complement_dev(upper_dev(raw[L - 1 - i]));
        badl |= c == 0;
      }
      q[i] = c;
    }
    if (__any_sync(0xffffffffu, badl)) {
      bad = true;
      break;
    }
    __syncwarp();
    if (lean_strand(ix, q, L, w, cb[strand], cap, &n[strand], &h[strand], &err) != kStrandOk) return false;
    __syncwarp();
  }
  if (lane == 0) write_read_result(b, r, bad, n, h, cb, stage, arena, arena_cap, arena_n, errw, err);
  __syncwarp();
  return true;
}

}  // namespace mg
