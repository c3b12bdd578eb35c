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
// run side by side. The kernel stops at the diagonal runs: the run ends of the references that can
// become candidates leave as 16-byte records, and k_finish_dual (mg_lib.cu) walks them one record
// per lane and covers and scores them one read per lane, work whose one-lane-per-run form here
// would leave most lanes idle. Nothing is indexed dynamically in registers; per-posting state
// lives in shared memory, whose regions are reused from step to step.
#pragma once
#include "mg_lean.cuh"

namespace mg {

// Per-warp shared memory of the dual path for up to Cap postings per strand (64 or 128; the kept
// postings, at most 64, are tracked in 64-bit masks); [half] = strand. The occurrence table has
// Cap entries, at least the distinct references of Cap postings.
template <int Cap>
struct alignas(16) DualSmemT {  // 16-byte aligned: the table clear stores 16 bytes a lane
  static_assert(Cap == 64 || Cap == 128 || Cap == 256, "postings per strand");
  uint32_t a[2][3][Cap];          // gathered postings (ref, pos, found | seed << 8 | table entry << 16);
                                // from the rank sort on: kept postings sorted (ref, pos, seed)
  uint32_t c[2][3][Cap];          // kept postings, compacted (ref, pos, seed); at the end the run
                                // records' refID, first-seed position and last-seed end
  uint32_t t[2][2][Cap];          // occurrence table (ref key, found mask, then occMax); from the
                                // diagonal runs on: the records' seed indices and segmax
  uint8_t q[2][kLeanQ];         // strand bases: forward, reverse complement
};
using DualSmem = DualSmemT<64>;  // the first dual tier, over every read

__device__ __forceinline__ unsigned long long upto64(int i) {  // bits 0..i
  return i >= 63 ? ~0ull : ((2ull << i) - 1ull);
}
__device__ __forceinline__ unsigned long long below64(int i) {  // bits 0..i-1
  return i <= 0 ? 0ull : upto64(i - 1);
}

// Bits of a full-warp ballot that belong to this lane's half.
__device__ __forceinline__ uint32_t half_bits(uint32_t ballot, int sh) { return (ballot >> sh) & 0xFFFFu; }

// Both strands of one read (bases already in S.q). Warp-uniform return: kStrandOk, or
// kStrandOverflow when either strand does not fit. Each lane receives its half's strand result:
// *n_out run records (step 5) in S.c[half][0..2] and S.t[half][0], in ascending refID.
template <int Cap>
__device__ int dual_strands(const DevIndex& ix, uint32_t L, DualSmemT<Cap>& S, uint32_t* n_out) {
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
    uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0, v2 = v0, v3 = v0;  // the seed's hash slot
    bool fnd = false;
    if (j < ns) {
      const uint32_t h = hash28_dev(q + j * step, ix.hlen);
      if (ix.slots) {
        const uint4* sl = ix.slots + (size_t)h * kSlotVecs;
        v0 = __ldg(sl);
        v1 = __ldg(sl + 1);
        cnt = v0.x;
        o0 = v0.y;
        if (cnt > 3) {  // postings 3-6 lie in the slot's second 32-byte sector
          v2 = __ldg(sl + 2);
          v3 = __ldg(sl + 3);
        }
      } else {
        o0 = __ldg(ix.dir + h);
        cnt = __ldg(ix.dir + h + 1) - o0;
      }
      fnd = cnt > 0 || h == ix.empty_hash;
    }
    fb |= half_bits(__ballot_sync(FULL, fnd), sh) << (16 * s);
    uint32_t x = cnt > (uint32_t)Cap ? (uint32_t)Cap + 1 : cnt;
    for (int o = 1; o < 16; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, x, o, 16);
      if (hl >= o) x += y;
    }
    const uint32_t Tn = T + __shfl_sync(FULL, x, 15, 16);
    if (__any_sync(FULL, Tn > (uint32_t)Cap)) return kStrandOverflow;
    const uint32_t f = __popc(fb & ((1u << j) - 1u));
    const uint32_t e = T + x - cnt;
    const uint32_t fj = f | (j << 8);
    uint32_t t0 = 0;
    if (ix.slots) {
      auto put = [&](uint32_t t, uint32_t ref, uint32_t pos) {
        if (t < cnt) {
          e_ref[e + t] = ref;
          e_pos[e + t] = pos;
          e_fj[e + t] = fj;
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
    for (uint32_t t = t0; t < cnt; t++) {
      const uint2 p = __ldg(ix.post + o0 + t);
      e_ref[e + t] = p.x;
      e_pos[e + t] = p.y;
      e_fj[e + t] = fj;
    }
    T = Tn;
  }
  bool alive = T > 0;
  if (!__any_sync(FULL, alive)) return kStrandOk;
  // 2. occurrence filter (Analyser.cpp:2057-2115): per reference, the found indices where it
  //    occurs (a table keyed by refID); the longest run of consecutive ones is its occMax
#pragma unroll
  for (int u = 0; u < Cap / 64; u++) {  // 16 lanes, 4 entries each per pass
    reinterpret_cast<uint4*>(tkey)[hl + 16 * u] = make_uint4(EMPTY, EMPTY, EMPTY, EMPTY);
    reinterpret_cast<uint4*>(tval)[hl + 16 * u] = make_uint4(0u, 0u, 0u, 0u);
  }
  __syncwarp();
  const int nslw = (int)__reduce_max_sync(FULL, (T + 15) / 16);  // posting blocks, warp-uniform
  for (int s = 0; s < nslw; s++) {
    const uint32_t i = hl + 16 * s;
    if (i < T) {
      const uint32_t ref = e_ref[i];
      uint32_t x = (ref * 2654435761u) >> (Cap == 64 ? 26 : Cap == 128 ? 25 : 24);  // Cap entries
      // at most T <= Cap distinct references: a free or matching entry is found within Cap probes
      for (int n = 0; n < Cap; n++) {
        const uint32_t old = atomicCAS(&tkey[x], EMPTY, ref);
        if (old == EMPTY || old == ref) break;
        x = (x + 1) & (Cap - 1);
      }
      const uint32_t fj = e_fj[i];
      atomicOr(&tval[x], 1u << (fj & 0xFFu));
      e_fj[i] = fj | (x << 16);
    }
  }
  __syncwarp();
  int hs = 0;
  for (int x = hl; x < Cap; x += 16)
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
  // kept postings compacted in gather order: as one 64-bit key ref << 37 | pos << 5 | seed (the
  // order of (ref, pos, seed): seeds < 32, positions < 2^32, references < 2^27) in the c arrays'
  // first two rows, or, for an index of more references, as three words
  const bool k64 = ix.n_refs <= (1u << 27);  // warp-uniform
  unsigned long long* c_key = reinterpret_cast<unsigned long long*>(c_ref);  // c_ref and c_pos rows
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
      const uint32_t jj = (fj >> 8) & 0xFFu;
      if (k64) {
        c_key[c] = ((unsigned long long)e_ref[i] << 37) | ((unsigned long long)e_pos[i] << 5) | jj;
      } else {
        c_ref[c] = e_ref[i];
        c_pos[c] = e_pos[i];
        c_j[c] = jj;
      }
    }
    T2 += __popc(kb);
  }
  __syncwarp();
  if (Cap > 64 && __any_sync(FULL, T2 > 64u)) return kStrandOverflow;  // the masks below hold 64
  // 3. rank sort of the kept postings by (ref, pos, seed); the keys are distinct
  uint32_t* s_ref = S.a[half][0];
  uint32_t* s_pos = S.a[half][1];
  uint32_t* s_j = S.a[half][2];
  const int nkw = (int)__reduce_max_sync(FULL, (T2 + 15) / 16);
  for (int s = 0; s < nkw; s++) {
    const uint32_t c = hl + 16 * s;
    if (c < T2) {
      uint32_t r, p, j, rk = 0;
      if (k64) {
        const unsigned long long key = c_key[c];
        for (uint32_t i = 0; i < T2; i++) rk += c_key[i] < key ? 1u : 0u;
        r = (uint32_t)(key >> 37);
        p = (uint32_t)(key >> 5);
        j = (uint32_t)key & 31u;
      } else {
        r = c_ref[c];
        p = c_pos[c];
        j = c_j[c];
        for (uint32_t i = 0; i < T2; i++) {
          const uint32_t rr = c_ref[i], pp = c_pos[i], jj = c_j[i];
          rk += (rr < r || (rr == r && (pp < p || (pp == p && jj < j)))) ? 1u : 0u;
        }
      }
      s_ref[rk] = r;
      s_pos[rk] = p;
      s_j[rk] = j;
    }
  }
  __syncwarp();
  // 4. diagonal runs over the sorted postings (Analyser.cpp:2337-2490)
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
  // 5. one record per run end of a kept reference whose longest run is M (the references that can
  //    become candidates): refID, reference position of the run's first seed, reference end of its
  //    last seed, the two seed indices. The head/tail walks, coverage and scores of these runs are
  //    k_finish_dual's. The records go to shared memory regions free by now.
  uint32_t* r_ref = S.c[half][0];
  uint32_t* r_sr = S.c[half][1];
  uint32_t* r_lr = S.c[half][2];
  uint32_t* r_jj = S.t[half][0];
  uint32_t nrec = 0;
  for (int s = 0; s < nkw; s++) {
    const int i = hl + 16 * s;
    const bool wk = alive && i < (int)T2 && ((E >> i) & 1ull) &&
                    segmax[63 - __clzll(R & upto64(i))] == (uint32_t)M;
    const uint32_t wb = half_bits(__ballot_sync(FULL, wk), sh);
    if (wk) {
      const uint32_t at = nrec + __popc(wb & ((1u << hl) - 1u));
      const int st = run_start(i);
      r_ref[at] = s_ref[i];
      r_sr[at] = s_pos[st];
      r_lr[at] = s_pos[i] + step;
      r_jj[at] = s_j[st] | (s_j[i] << 8);
    }
    nrec += __popc(wb);
  }
  __syncwarp();
  *n_out = nrec;
  return kStrandOk;
}

// Read r on the dual path; false when it does not fit (the caller hands it on).
// comp: the block's 256-entry table of complement(upper(byte)), 0 where there is none.
// The read's run records (forward strand first) go to its staging slots, or to the arena when
// there are more than kSlots, and the read is marked kReadUnscored for k_finish_dual; a read
// without records is final here (no candidate).
template <int Cap>
__device__ bool process_read_dual(const DevIndex& ix, const BatchDev& b, uint32_t r, DualSmemT<Cap>& S,
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
      b.reads[r] = mg_read_result{-1.0f, 0, 0, 0, MG_READ_BAD_BYTE, 0, 0};
    if (lane == 0) atomicOr(errw, kErrBadInput);
    __syncwarp();
    return true;
  }
  __syncwarp();
  uint32_t nh;
  if (dual_strands(ix, L, S, &nh) != kStrandOk) return false;
  const uint32_t n0 = __shfl_sync(FULL, nh, 0), n1 = __shfl_sync(FULL, nh, 16), tot = n0 + n1;
  if (tot == 0) {
    if (lane == 0) b.reads[r] = mg_read_result{-1.0f, 0, 0, 0, 0, 0, 0};
    __syncwarp();
    return true;
  }
  unsigned long long at = 0;
  if (lane == 0 && tot > (uint32_t)kSlots) at = atomicAdd(arena_n, (unsigned long long)tot);
  at = __shfl_sync(FULL, at, 0);
  const bool big = tot > (uint32_t)kSlots;
  const bool fits = !big || at + tot <= arena_cap;  // else the call grows the arena and runs again
  if (fits) {
    mg_candidate* dst = big ? arena + at : stage + (uint64_t)r * kSlots;
    for (uint32_t x = lane; x < tot; x += 32) {
      const int h = x >= n0 ? 1 : 0;
      const uint32_t i = x - (h ? n0 : 0);
      dst[x] = mg_candidate{S.c[h][0][i], __uint_as_float(S.c[h][1][i]), __uint_as_float(S.c[h][2][i]),
                            __uint_as_float(S.t[h][0][i])};
    }
  }
  if (lane == 0) {
    if (!fits) atomicOr(errw, kErrArena);
    b.reads[r] = mg_read_result{-1.0f, big ? (uint32_t)at : 0u, (uint16_t)n0, (uint16_t)n1,
                                fits ? kReadUnscored : (uint8_t)0, 0, 0};
  }
  __syncwarp();
  return true;
}

}  // namespace mg
