// mirage_b200 C ABI: index upload, the relative-score logf table, the classification kernels
// (warp tier, block tier, global-memory tier), output compaction and the host entry points.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <dlfcn.h>
#include <sched.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mirage_b200.h"
#include "mg_device.cuh"
#include "mg_kernels.cuh"
#include "mg_lean.cuh"
#include "mg_dual.cuh"
#include "mg_long.cuh"
#include "mhm.h"

namespace mg {

// ------------------------------------------------------------------------------ errors

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define CU(call)                                                                                \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return set_error(MG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

// ------------------------------------------------------------------------------ tiers

// Warp tiers: one warp per read, workspace in shared memory (8 warps per block). The dual-strand
// tier takes reads up to kLeanQ bases with at most 64 postings and 8 scored candidates per strand;
// the general warp tier takes its leftovers within the limits below.
constexpr int kW1Warps = 8;
constexpr int kW1Q = 320, kW1Seeds = 20, kW1E = 128, kW1C = 8;
constexpr int kW1Chunk = 4;  // reads taken per work-stealing step (default)

struct WarpSmem {
  uint64_t kA[kW1E];
  uint32_t kB[kW1E];
  uint32_t X[kW1E];
  uint32_t Y[kW1E];
  uint32_t fpos[32];
  mg_candidate cb[2][kW1C];
  uint8_t q[kW1Q];
  RedTmp<32> red;
};

// Block tier: one block of 256 threads per read, workspace in dynamic shared memory.
constexpr int kB2Threads = 256;
constexpr int kB2Q = 20480, kB2Seeds = 1408, kB2E = 4096, kB2C = 128;
// Global tier: one block per read, workspace in global scratch.
constexpr int kB3Threads = 256;
constexpr int kB3Q = 65535, kB3Seeds = 4400, kB3E = 65536, kB3C = 4096;
constexpr int kB3Blocks = 32;
// Oversize tier: what the global tier cannot hold (reads over 65,535 bases, or over 4,400 seeds
// or 65,536 postings per strand), one block per read over a workspace sized on demand for the
// largest such read, 32-bit fields throughout. Hard limits: a read of at most 2,000,000 bases
// (the relative score's logarithm stays inside its patched domain up to there) and 2^24
// postings per strand; at most 4 workspaces and 1 GiB.
constexpr int kHugeThreads = 512;
constexpr uint32_t kHugeMaxQ = 2000000, kHugeMaxE = 1u << 24;
constexpr int kHugeMaxSlabs = 4;
constexpr size_t kHugeMaxBytes = size_t(1) << 30;

struct WsLayout {
  size_t kA, kB, X, Y, fpos, cb, q, red, W, cov, total;
};

static WsLayout ws_layout(int Q, int seeds, int E, int C, bool wide = false) {
  WsLayout l;
  size_t o = 0;
  auto take = [&](size_t n, size_t al) {
    o = (o + al - 1) / al * al;
    size_t at = o;
    o += n;
    return at;
  };
  l.kA = take((size_t)E * 8, 16);
  l.kB = take((size_t)E * 4, 16);
  l.X = take((size_t)E * 4, 16);
  l.Y = take((size_t)E * 4, 16);
  l.fpos = take((size_t)seeds * 4, 16);
  l.cb = take((size_t)2 * C * sizeof(mg_candidate), 16);
  l.q = take((size_t)Q, 16);
  l.red = take(sizeof(RedTmp<256>), 16);
  l.W = wide ? take((size_t)E * 4, 16) : 0;
  l.cov = wide ? take(((size_t)Q + 31) / 32 * 4, 16) : 0;
  l.total = (o + 127) / 128 * 128;
  return l;
}

__device__ __forceinline__ StrandWS ws_from(uint8_t* base, const WsLayout& l, int C) {
  StrandWS ws;
  ws.kA = (uint64_t*)(base + l.kA);
  ws.kB = (uint32_t*)(base + l.kB);
  ws.X = (uint32_t*)(base + l.X);
  ws.Y = (uint32_t*)(base + l.Y);
  ws.fpos = (uint32_t*)(base + l.fpos);
  ws.cb[0] = (mg_candidate*)(base + l.cb);
  ws.cb[1] = ws.cb[0] + C;
  ws.q = base + l.q;
  ws.W = l.W ? (uint32_t*)(base + l.W) : nullptr;
  ws.cov = l.cov ? (uint32_t*)(base + l.cov) : nullptr;
  return ws;
}

struct StageDev {
  mg_candidate* stage;   // kSlots per read
  mg_candidate* arena;
  uint64_t arena_cap;
  unsigned long long* arena_n;
};

// Dual-strand warp tier: every read of the batch, one warp per read (a half-warp per strand),
// work stealing in chunks of kW1Chunk reads; reads that do not fit go to the general warp tier.
__global__ void __launch_bounds__(kW1Warps * 32, 5) k_classify_dual(DevIndex ix, BatchDev b, StageDev sd, uint32_t chunk) {
  __shared__ DualSmem sm[kW1Warps];
  __shared__ uint8_t comp[256];
  for (int c = threadIdx.x; c < 256; c += blockDim.x) comp[c] = complement_dev(upper_dev((uint8_t)c));
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  DualSmem& S = sm[w];
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(b.work, chunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if ((uint64_t)base >= b.n) break;
    const uint64_t end64 = (uint64_t)base + chunk;
    const uint32_t end = (uint32_t)(end64 < b.n ? end64 : b.n);
    for (uint32_t r = base; r < end; r++) {
      if (!process_read_dual(ix, b, r, S, comp, sd.stage, sd.arena, sd.arena_cap, sd.arena_n, b.err)) {
        if (lane == 0) {
          unsigned at = atomicAdd(b.n_ovf0, 1u);
          b.ovf0[at] = r;
          b.reads[r] = mg_read_result{};  // not kReadUnscored: a later tier writes this read
        }
      }
      __syncwarp();
    }
  }
}

// Four bytes p..p+3, all readable, as one little-endian word: the aligned word holding p and,
// only when p is not 4-aligned, the next aligned word (which holds p+3), so nothing outside
// p..p+3's words is read.
__device__ __forceinline__ uint32_t load4(const uint8_t* p) {
  const uintptr_t a = (uintptr_t)p;
  const uint32_t* w = (const uint32_t*)(a & ~(uintptr_t)3);
  const uint32_t sh = (uint32_t)(a & 3u);
  const uint32_t lo = w[0];
  return sh ? __funnelshift_r(lo, w[1], sh * 8u) : lo;
}
// upper_dev on each byte of w: bytes 0x61..0x7F lose 0x20.
__device__ __forceinline__ uint32_t upper4(uint32_t w) {
  const uint32_t m = (((w & 0x7F7F7F7Fu) + 0x1F1F1F1Fu) & ~w) & 0x80808080u;
  return w - (m >> 2);
}

constexpr int kFinThreads = 256;
constexpr int kCovStride = kLeanQ / 32 + 1;  // coverage words per thread; odd, so no bank conflicts
constexpr int kFinRecCap = 128;              // run records a warp walks together per 32 reads

// The head and tail walks of one run record x (head_walk, tail_walk) on the strand's bases, read
// from the batch (raw, L bytes): forward in upper case, the reverse complement backwards through
// the complement table; the tail four bytes at a time while the window has four left. Returns the
// run's query start << 16 | its extended length T, or 0 when T < k.
__device__ __forceinline__ uint32_t walk_record(const DevIndex& ix, const uint8_t* comp, const uint8_t* raw, uint32_t L,
                                                int strand, const mg_candidate& x, uint32_t k, uint32_t step) {
  auto qb = [&](uint32_t p) -> uint8_t { return strand ? comp[raw[L - 1 - p]] : upper_dev(raw[p]); };
  const uint8_t* rs = ix.bases + ix.ref_off[x.ref];
  const uint32_t rlen = ix.ref_len[x.ref];
  const uint32_t sr = __float_as_uint(x.rel), lr = __float_as_uint(x.score), jj = __float_as_uint(x.pct);
  const uint32_t sq = (jj & 0xFFu) * step, lq = (jj >> 8) * step + step;
  uint32_t tail = 0;
  if (lq < L && lr < rlen) {
    const uint32_t lim = min(min(rlen - lr, k), L - lq);
    while (tail + 4 <= lim) {
      uint32_t wq;
      if (strand) {
        const uint32_t w = load4(raw + (L - 4 - (lq + tail)));
        wq = (uint32_t)comp[w >> 24] | ((uint32_t)comp[(w >> 16) & 0xFFu] << 8) |
             ((uint32_t)comp[(w >> 8) & 0xFFu] << 16) | ((uint32_t)comp[w & 0xFFu] << 24);
      } else {
        wq = upper4(load4(raw + lq + tail));
      }
      if (wq ^ load4(rs + lr + tail)) break;
      tail += 4;
    }
    while (tail < lim && qb(lq + tail) == rs[lr + tail]) tail++;
  }
  uint32_t head = 0;
  const uint32_t hsz = min(sr, k);
  if (sq != 0 && hsz != 0) {
    const uint32_t jb = min(sq - 1, hsz - 1);
    while (head < jb && qb(sq - 1 - head) == rs[sr - head]) head++;
  }
  const uint32_t tot = tail + head + (lq - sq);
  return tot >= k ? ((sq - head) << 16) | tot : 0u;
}

// Finishing pass of the dual-strand tiers over the reads they left kReadUnscored, a warp per 32
// consecutive reads. A read's run records (forward strand first, each strand in ascending refID;
// see process_read_dual) name the run ends of the references whose longest run is M. The warp
// walks its reads' records one per lane (walk_record), so that reads with many records or long
// walks do not hold the other lanes; then each read's lane groups its records by reference: the
// runs that scored (T >= k) give the sums and the query coverage, and a reference with such a run
// is a candidate whose Score, percentage and relative score (MatrixCPU.cpp:18-214,
// MatrixResult.cpp:21-29) replace its records, compacted in place; then the strand merge and top
// group as write_read_result_s (Analyser.cpp:592-611, 388).
__global__ void __launch_bounds__(kFinThreads) k_finish_dual(DevIndex ix, BatchDev b, StageDev sd) {
  const unsigned FULL = 0xffffffffu;
  __shared__ uint8_t comp[256];
  __shared__ uint32_t covs[kFinThreads * kCovStride];
  __shared__ uint32_t walks[kFinThreads / 32][kFinRecCap];
  for (int c = threadIdx.x; c < 256; c += blockDim.x) comp[c] = complement_dev(upper_dev((uint8_t)c));
  __syncthreads();
  const int lane = threadIdx.x & 31;
  uint32_t* cov = covs + threadIdx.x * kCovStride;
  uint32_t* zw = walks[threadIdx.x >> 5];
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step;
  // a warp takes 32 consecutive reads, one per lane
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < b.n;
       base += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = base + lane;
    mg_read_result rr{};
    bool mine = false;
    if (r < b.n) {
      rr = b.reads[r];
      mine = rr.strand == kReadUnscored;
    }
    const uint32_t n0 = mine ? rr.n_fwd : 0u, nrec = mine ? n0 + rr.n_rc : 0u;
    uint64_t o0 = 0;
    uint32_t L = 0;
    mg_candidate* rec = nullptr;
    if (mine) {
      o0 = b.offs[r];
      L = (uint32_t)(b.offs[r + 1] - o0);
      rec = nrec > (uint32_t)kSlots ? sd.arena + rr.cand_off : sd.stage + r * kSlots;
    }
    uint32_t incl = nrec;  // the warp's records, read by read
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t excl = incl - nrec, total = __shfl_sync(FULL, incl, 31);
    if (total == 0) continue;
    // the walks, one record per lane across the warp's reads (up to kFinRecCap records; beyond
    // that each lane walks its own read's records below)
    const bool together = total <= (uint32_t)kFinRecCap;
    if (together) {
      for (uint32_t gb = 0; gb < total; gb += 32) {
        const uint32_t g = gb + lane;
        uint32_t o = 0;  // the lane whose read holds record g: the lanes before it end at or below g
        for (int bit = 16; bit > 0; bit >>= 1)
          if (__shfl_sync(FULL, incl, o + bit - 1) <= g) o += bit;
        const uint32_t oe = __shfl_sync(FULL, excl, o), on0 = __shfl_sync(FULL, n0, o);
        const uint32_t oL = __shfl_sync(FULL, L, o);
        const uint64_t oo = __shfl_sync(FULL, (unsigned long long)o0, o);
        const mg_candidate* orec = (const mg_candidate*)__shfl_sync(FULL, (unsigned long long)rec, o);
        if (g < total) {
          const uint32_t i = g - oe;
          zw[g] = walk_record(ix, comp, b.bases + oo, oL, i >= on0 ? 1 : 0, orec[i], k, step);
        }
      }
      __syncwarp();
    }
    if (mine) {
      const uint8_t* raw = b.bases + o0;
      const bool big = nrec > (uint32_t)kSlots;
      const uint32_t nw = (L + 31) / 32;
      int err = 0;
      float hi[2] = {-1.0f, -1.0f};
      uint32_t nc[2] = {0, 0}, out = 0;
      for (int strand = 0; strand < 2; strand++) {
        const uint32_t end = strand ? nrec : n0;
        for (uint32_t g = strand ? n0 : 0; g < end;) {
          const uint32_t ref = rec[g].ref;
          uint32_t sumc = 0, sumr = 0, nsc = 0, e = g;
          for (; e < end && rec[e].ref == ref; e++) {
            const uint32_t z = together ? zw[excl + e] : walk_record(ix, comp, raw, L, strand, rec[e], k, step);
            if (!z) continue;
            const uint32_t tot = z & 0xFFFFu, a = z >> 16, bnd = a + tot;
            if (nsc++ == 0)
              for (uint32_t wd = 0; wd < nw; wd++) cov[wd] = 0;
            sumc += tot;
            sumr += tot * (tot + 1) / 2;
            for (uint32_t wd = a >> 5; wd <= (bnd - 1) >> 5; wd++) {
              const uint32_t w0 = wd * 32;
              const uint32_t lo = a > w0 ? a : w0, up = bnd < w0 + 32 ? bnd : w0 + 32;
              const uint32_t n = up - lo;
              cov[wd] |= (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u)) << (lo - w0);
            }
          }
          if (nsc) {
            uint32_t hits = 0;
            for (uint32_t wd = 0; wd < nw; wd++) hits += __popc(cov[wd]);
            float sc, pc;
            final_score(sumr, sumc, hits, L, &sc, &pc);
            const float rl = relative_score_tab(ix, L, ix.ref_len[ref], sc, &err);
            rec[out++] = mg_candidate{ref, rl, sc, pc};  // out <= g: this group's records are read
            nc[strand]++;
            hi[strand] = fmaxf(hi[strand], rl);
          }
          g = e;
        }
      }
      const uint32_t tot = nc[0] + nc[1];
      mg_candidate* fin = rec;
      if (big && tot <= (uint32_t)kSlots) {  // k_scatter takes up to kSlots candidates from the slots
        fin = sd.stage + r * kSlots;
        for (uint32_t c = 0; c < tot; c++) fin[c] = rec[c];
      }
      const int ch = hi[0] < hi[1] ? 1 : 0;  // Analyser.cpp:601
      const uint32_t nch = nc[ch];
      const float hch = hi[ch];
      const mg_candidate* cc = fin + (ch ? nc[0] : 0);
      uint32_t top = 0;
      for (uint32_t i = 0; i < nch; i++) top += cc[i].rel == hch;
      rr = mg_read_result{hch, tot > (uint32_t)kSlots ? rr.cand_off : 0u, (uint16_t)nc[0], (uint16_t)nc[1],
                          (uint8_t)ch, (uint8_t)((nch > 0 && hch != 0.0f) ? 1 : 0), (uint16_t)top};  // Analyser.cpp:388
      b.reads[r] = rr;
      if (err) atomicOr(b.err, err);
    }
    __syncwarp();  // zw is the next reads' before any lane leaves these
  }
}

// Further dual-strand tiers over the leftovers of the one before: room for Cap postings per
// strand (128 or 256, at most 64 of them kept); the reads they take leave run records for
// k_finish_dual like the first tier's, their own leftovers go to the next tier. With all_reads a
// tier takes every read of the batch (the tiers before it are not run).
constexpr int kW2Warps = 4;  // warps per block at 128 postings (35 KB of shared memory)
constexpr int kW3Warps = 2;  // at 256 postings (34 KB)
template <int Cap, int Warps>
__global__ void __launch_bounds__(Warps * 32) k_classify_dual_list(DevIndex ix, BatchDev b, StageDev sd,
                                                                     const uint32_t* list, const unsigned* list_n,
                                                                     unsigned* cursor, uint32_t* next,
                                                                     unsigned* next_n, int all_reads) {
  __shared__ DualSmemT<Cap> sm[Warps];
  __shared__ uint8_t comp[256];
  for (int c = threadIdx.x; c < 256; c += blockDim.x) comp[c] = complement_dev(upper_dev((uint8_t)c));
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  DualSmemT<Cap>& S = sm[w];
  const uint32_t n = all_reads ? (uint32_t)b.n : *list_n;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(cursor, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= n) break;
    const uint32_t r = all_reads ? item : list[item];
    if (!process_read_dual(ix, b, r, S, comp, sd.stage, sd.arena, sd.arena_cap, sd.arena_n, b.err)) {
      if (lane == 0) {
        unsigned at = atomicAdd(next_n, 1u);
        next[at] = r;
        b.reads[r] = mg_read_result{};  // not kReadUnscored: a later tier writes this read
      }
    }
    __syncwarp();
  }
}

// General warp tier over the dual tiers' leftovers; its own leftovers go to the block tier.
__global__ void __launch_bounds__(kW1Warps * 32) k_classify_warp_list(DevIndex ix, BatchDev b, StageDev sd) {
  __shared__ WarpSmem sm[kW1Warps];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& S = sm[w];
  StrandWS ws;
  ws.q = S.q;
  ws.fpos = S.fpos;
  ws.kA = S.kA;
  ws.kB = S.kB;
  ws.X = S.X;
  ws.Y = S.Y;
  ws.cb[0] = S.cb[0];
  ws.cb[1] = S.cb[1];
  const Caps caps{kW1Q, kW1Seeds, kW1E, kW1C};
  const uint32_t n = *b.n_ovf0b;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(b.work1, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= n) break;
    const uint32_t r = b.ovf0b[item];
    if (!process_read<32>(ix, b, r, ws, caps, &S.red, sd.stage, sd.arena, sd.arena_cap, sd.arena_n, b.err)) {
      if (lane == 0) {
        unsigned at = atomicAdd(b.n_ovf1, 1u);
        b.ovf1[at] = r;
      }
    }
    __syncwarp();
  }
}

// Long-read tier over the general warp tier's leftovers (reads beyond its limits), a block per
// read with work stealing: the smaller size first, then the larger over what it hands on, whose
// own leftovers go to the block tier.
template <class SM, int MinBlocks>
__global__ void __launch_bounds__(kLgThreads, MinBlocks) k_classify_long(DevIndex ix, BatchDev b, StageDev sd,
                                                                      const uint32_t* list, const unsigned* list_n,
                                                                      unsigned* cursor, uint32_t* next,
                                                                      unsigned* next_n) {
  extern __shared__ __align__(16) uint8_t dsm[];
  SM& S = *reinterpret_cast<SM*>(dsm);
  __shared__ uint32_t s_item;
  const uint32_t n = *list_n;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(cursor, 1u);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();
    if (item >= n) break;
    const uint32_t r = list[item];
    if (!process_read_long(ix, b, r, S, sd.stage, sd.arena, sd.arena_cap, sd.arena_n, b.err)) {
      if (threadIdx.x == 0) next[atomicAdd(next_n, 1u)] = r;
    }
    __syncthreads();
  }
}

// Block tier over a list of reads (list == nullptr: every read, the plain form); the reads that
// do not fit go to the next list, or, from the last tier, are marked for the oversize tier
// (kErrHuge: the host then runs the batch again with it).
template <int G>
__global__ void __launch_bounds__(G) k_classify_block(DevIndex ix, BatchDev b, StageDev sd, const uint32_t* list,
                                                       const unsigned* list_n, unsigned* cursor, uint32_t* next,
                                                       unsigned* next_n, uint8_t* gws, WsLayout lay, Caps caps,
                                                       int last_tier) {
  extern __shared__ __align__(16) uint8_t dsm[];
  __shared__ uint32_t s_item;
  uint8_t* base = gws ? gws + (size_t)blockIdx.x * lay.total : dsm;
  const StrandWS ws = ws_from(base, lay, caps.c);
  RedTmp<G>* red = (RedTmp<G>*)(base + lay.red);
  const uint64_t n = list ? (uint64_t)*list_n : b.n;
  for (;;) {
    if (threadIdx.x == 0) s_item = cursor ? atomicAdd(cursor, 1u) : 0xFFFFFFFFu;
    __syncthreads();
    uint64_t item = cursor ? (uint64_t)s_item : (uint64_t)blockIdx.x;
    __syncthreads();
    if (!cursor && item >= n) break;
    if (item >= n) break;
    const uint32_t r = list ? list[item] : (uint32_t)item;
    if (!process_read<G>(ix, b, r, ws, caps, red, sd.stage, sd.arena, sd.arena_cap, sd.arena_n, b.err)) {
      if (threadIdx.x == 0) {
        if (last_tier) {
          atomicOr(b.err, kErrHuge);
          b.reads[r] = mg_read_result{-1.0f, 0, 0, 0, MG_READ_TOO_LARGE, 0, 0};
        } else {
          next[atomicAdd(next_n, 1u)] = r;
        }
      }
    }
    __syncthreads();
    if (!cursor) break;
  }
}

// What one read asks of the oversize tier: over both strands the most seeds and the most postings
// (the bucket sizes of its seeds, each seed hashed as process_strand hashes it: the hash of
// hash28_dev over the upper-case window, on the reverse strand complemented).
template <int G>
__device__ void read_need(const DevIndex& ix, const uint8_t* raw, uint32_t L, RedTmp<G>* red, uint32_t* seeds_out,
                          uint64_t* post_out) {
  const uint32_t k = (uint32_t)ix.k, step = (uint32_t)ix.step, hl = (uint32_t)ix.hlen;
  const uint32_t n_seeds = L > k ? (L - k + step - 1) / step : 0;
  uint64_t most = 0;
  for (int strand = 0; strand < 2; strand++) {
    uint64_t e = 0;
    for (uint32_t j = threadIdx.x; j < n_seeds; j += G) {
      const uint32_t p = j * step;  // p + hl <= L: the last seed starts before L - k
      uint32_t h = 2166136261u;
      for (uint32_t t = 0; t < hl; t++) {
        const uint8_t c = strand == 0 ? upper_dev(raw[p + t]) : complement_dev(upper_dev(raw[L - 1 - p - t]));
        h = (h * 16777619u) ^ c;
      }
      h = ((h >> 28) ^ h) & 0x0FFFFFFFu;
      e += __ldg(ix.dir + h + 1) - __ldg(ix.dir + h);
    }
    e = grp_sum_u64<G>(e, red);
    most = e > most ? e : most;
  }
  *seeds_out = n_seeds;
  *post_out = most;
}

// Oversize tier over the global tier's leftovers: a block per read (work stealing), each block
// with its own workspace slab (hws; null before the first oversize read). A read that does not
// fit records what it needs in need[0..3] (most bases, seeds, postings; reads waiting) and sets
// kErrHuge, so that the host grows the slabs and runs the batch again; a read beyond the hard
// limits, or with more than 65,535 candidates on a strand, is refused (kErrLimit).
template <int G>
__global__ void __launch_bounds__(G) k_classify_huge(DevIndex ix, BatchDev b, StageDev sd, const uint32_t* list,
                                                      const unsigned* list_n, unsigned* cursor, uint8_t* hws,
                                                      WsLayout lay, Caps caps, unsigned* need) {
  __shared__ uint32_t s_item;
  __shared__ RedTmp<G> red;
  uint8_t* base = hws ? hws + (size_t)blockIdx.x * lay.total : nullptr;
  StrandWS ws{};
  if (base) ws = ws_from(base, lay, caps.c);
  const unsigned n = *list_n;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(cursor, 1u);
    __syncthreads();
    const unsigned item = s_item;
    __syncthreads();
    if (item >= n) break;
    const uint32_t r = list[item];
    if (base && process_read<G, true>(ix, b, r, ws, caps, &red, sd.stage, sd.arena, sd.arena_cap, sd.arena_n, b.err))
      continue;
    const uint64_t o0 = b.offs[r], Lr = b.offs[r + 1] - o0;
    uint32_t seeds = 0;
    uint64_t post = 0;
    if (Lr <= kHugeMaxQ) read_need<G>(ix, b.bases + o0, (uint32_t)Lr, &red, &seeds, &post);
    if (threadIdx.x == 0) {
      const bool hard = Lr > kHugeMaxQ || post > kHugeMaxE;
      const bool grow = !hard && (Lr > (uint64_t)caps.q || seeds > (uint32_t)caps.seeds || post > (uint64_t)caps.e);
      if (grow) {
        atomicMax(need + 0, (unsigned)Lr);
        atomicMax(need + 1, seeds);
        atomicMax(need + 2, (unsigned)post);
        atomicAdd(need + 3, 1u);
        atomicOr(b.err, kErrHuge);
      } else {
        atomicOr(b.err, kErrLimit);
      }
      b.reads[r] = mg_read_result{-1.0f, 0, 0, 0, MG_READ_TOO_LARGE, 0, 0};
    }
    __syncthreads();
  }
}

// 2-bit packed bases (mg_pack.cpp) back to ASCII: byte i of packed holds bases 4i..4i+3, the first
// in the low bits, codes 0-3 for A, C, G, T; then the listed exception bytes at their offsets.
__global__ void k_unpack_bases(const uint8_t* packed, uint64_t n, uint8_t* out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n + 3) / 4; i += stride) {
    const uint32_t v = packed[i];
#pragma unroll
    for (int t = 0; t < 4; t++)
      if (4 * i + t < n) out[4 * i + t] = (uint8_t)(0x54474341u >> (8 * ((v >> (2 * t)) & 3u)));  // "ACGT"
  }
}

__global__ void k_unpack_exceptions(const uint64_t* exc, uint64_t n_exc, uint64_t n, uint8_t* out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_exc; j += stride) {
    const uint64_t e = exc[j];
    if ((e >> 8) < n) out[e >> 8] = (uint8_t)(e & 0xFFu);
  }
}

// Output compaction: exclusive scan of per-read candidate counts, then a scatter into one
// contiguous array in read order.
constexpr int kScanBlock = 1024;

__global__ void k_count_sums(const mg_read_result* reads, uint64_t n, unsigned long long* block_sums) {
  __shared__ unsigned long long s[kScanBlock / 32];
  uint64_t i = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
  unsigned long long v = i < n ? (unsigned long long)(reads[i].n_fwd + reads[i].n_rc) : 0ull;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < kScanBlock / 32; w++) t += s[w];
    block_sums[blockIdx.x] = t;
  }
}

// Exclusive scan of the per-block candidate counts, one block of kScanBlock threads in tiles.
// chain (optional): candidates of earlier chunks of the same batch; the scan starts there and
// leaves the new running total behind, so chunk offsets are offsets into the batch's output.
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(unsigned long long* block_sums, uint64_t nb,
                                                          unsigned long long* total, unsigned long long* chain) {
  __shared__ unsigned long long s[kScanBlock / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned long long base = chain ? *chain : 0ull;
  unsigned long long carry = base;
  for (uint64_t t0 = 0; t0 < nb; t0 += kScanBlock) {
    const uint64_t i = t0 + threadIdx.x;
    const unsigned long long v = i < nb ? block_sums[i] : 0ull;
    unsigned long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s[wid] = x;
    __syncthreads();
    unsigned long long wb = 0, tile = 0;
    for (int w = 0; w < kScanBlock / 32; w++) {
      wb += w < wid ? s[w] : 0ull;
      tile += s[w];
    }
    if (i < nb) block_sums[i] = carry + wb + x - v;
    carry += tile;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *total = carry - base;
    if (chain) *chain = carry;
  }
}

__global__ void k_scatter(mg_read_result* reads, uint64_t n, const unsigned long long* block_sums, StageDev sd,
                          mg_candidate* out, uint64_t cap, int* err) {
  __shared__ unsigned long long s[kScanBlock / 32];
  const uint64_t i = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long v = i < n ? (unsigned long long)(reads[i].n_fwd + reads[i].n_rc) : 0ull;
  unsigned long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s[wid] = x;
  __syncthreads();
  unsigned long long wb = 0;
  for (int w = 0; w < wid; w++) wb += s[w];
  if (i >= n) return;
  const unsigned long long off = block_sums[blockIdx.x] + wb + x - v;
  mg_read_result rr = reads[i];
  const uint32_t tot = rr.n_fwd + rr.n_rc;
  const mg_candidate* src = tot > (uint32_t)kSlots ? sd.arena + rr.cand_off : sd.stage + i * kSlots;
  if (off + tot > cap) {
    atomicOr(err, kErrOutput);
  } else {
    for (uint32_t c = 0; c < tot; c++) out[off + c] = src[c];
  }
  rr.cand_off = (uint32_t)off;
  reads[i] = rr;
}

// Index construction: directory from the ascending TOC (dir[h] = first posting of the first
// TOC hash >= h), and the logf probe.
__global__ void k_fill_dir(const uint32_t* toc_hash, const uint32_t* toc_start, uint64_t n, uint32_t total,
                           uint32_t* dir) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  const uint64_t lo = i == 0 ? 0 : (uint64_t)toc_hash[i - 1] + 1;
  const uint64_t hi = i == n ? (1ull << 28) : (uint64_t)toc_hash[i];
  const uint32_t v = i == n ? total : toc_start[i];
  for (uint64_t h = lo; h <= hi; h++) dir[h] = v;
}

// The posting records of a .mhm image decoded on the device, with the host reader's checks
// (mhm_parse; the reference's reader Hashmap.cpp:402-580 and decode Analyser.cpp:1602-1752).
enum : int { kDecHash = 1, kDecOrder = 2, kDecRecord = 4 };

__device__ __forceinline__ uint64_t rd_img(const uint8_t* p, int w) {
  uint64_t v = 0;
  for (int i = 0; i < w; i++) v |= (uint64_t)p[i] << (8 * i);
  return v;
}

// Bucket TOC: hash and record stream position of every bucket.
__global__ void k_mhm_toc(const uint8_t* img, uint64_t toc_at, uint64_t n, int W, uint32_t* hash, uint64_t* sp,
                          int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint8_t* p = img + toc_at + i * 2 * (uint64_t)W;
    uint64_t h = rd_img(p, W);
    if (h > 0x0FFFFFFFull) {
      atomicOr(err, kDecHash);
      h = 0;
    }
    hash[i] = (uint32_t)h;
    sp[i] = rd_img(p + W, W);
  }
}

// Postings per bucket (numIDs of its record). The last bucket gets none: the reader stores its
// BufferSize one past the array (Hashmap.cpp:552-553), so it is present with no postings.
__global__ void k_mhm_count(const uint8_t* img, uint64_t L, const uint32_t* hash, const uint64_t* sp, uint64_t n,
                            uint64_t* cnt, int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (i > 0 && hash[i] <= hash[i - 1]) atomicOr(err, kDecOrder);
    uint64_t c = 0;
    if (i + 1 < n) {
      if (sp[i] >= L || sp[i + 1] <= sp[i]) {
        atomicOr(err, kDecRecord);
      } else {
        const uint8_t* p = img + sp[i];
        const uint64_t rem = L - sp[i];
        const uint32_t wo = rem >= 4 ? p[0] : 0, wnum = rem >= 4 ? p[3] : 0;
        if (rem < 4 || wnum > 8 || wnum < 1 || 4ull + 2ull * wo + wnum > rem) {
          atomicOr(err, kDecRecord);
        } else {
          c = rd_img(p + 4 + 2 * wo, (int)wnum);
          // widths are at least one byte: no more postings than bytes left (bounds the sum)
          if (c > rem || c > 0xFFFFFFFFull) {
            atomicOr(err, kDecRecord);
            c = 0;
          }
        }
      }
    }
    cnt[i] = c;
  }
}

__global__ void k_mhm_decode(const uint8_t* img, uint64_t L, const uint64_t* sp, const uint64_t* cnt,
                             const uint64_t* start, uint64_t n, int word, uint32_t n_refs, uint2* post, int* err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t M = word >= 8 ? ~0ull : ((1ull << (8 * word)) - 1ull);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t num = cnt[i];
    if (!num) continue;
    const uint8_t* p = img + sp[i];
    uint64_t rem = L - sp[i];
    const int wo = p[0], wid = p[1], wpos = p[2], wnum = p[3];
    bool bad = wo > word || wid > word || wpos > word || wo < 1 || wid < 1 || wpos < 1;
    uint2* out = post + start[i];
    if (!bad) {
      const uint64_t id_min = rd_img(p + 4, wo), pos_min = rd_img(p + 4 + wo, wo);
      const uint64_t hdr = 4ull + 2ull * wo + wnum;
      p += hdr;
      rem -= hdr;
      bad = (wid && num > (rem - 1 - wpos) / wid) || rem < 1ull + wpos + (uint64_t)wid * num;
      if (!bad) {
        for (uint64_t j = 0; j < num && !bad; j++) {
          const uint64_t id = (rd_img(p + j * wid, wid) + id_min) & M;  // "raise" of Analyser.cpp:1666-1686
          bad = id >= n_refs;
          out[j].x = (uint32_t)id;
        }
        p += (uint64_t)wid * num;
        rem -= (uint64_t)wid * num;
        const int wrep = p[0];
        const uint64_t nrep = rd_img(p + 1, wpos);
        p += 1 + wpos;
        rem -= 1 + wpos;
        bad = bad || wrep > word || wrep < 1 || nrep > num || nrep > rem / (uint64_t)(wrep + wpos);
        uint64_t filled = 0;
        for (uint64_t r = 0; r < nrep && !bad; r++) {
          const uint64_t c = rd_img(p, wrep);
          const uint64_t v = (rd_img(p + wrep, wpos) + pos_min) & M;
          p += wrep + wpos;
          if (filled + c > num || c > num || v > 0xFFFFFFFFull) {
            bad = true;
            break;
          }
          for (uint64_t t = 0; t < c; t++) out[filled + t].y = (uint32_t)v;
          filled += c;
        }
        bad = bad || filled != num;  // the reference pairs vSeqIDs[k] with vPos[k]
      }
    }
    if (bad) atomicOr(err, kDecRecord);
  }
}

// Directory from the ascending TOC and 64-bit bucket starts (values below 2^32).
__global__ void k_fill_dir64(const uint32_t* toc_hash, const uint64_t* toc_start, uint64_t n, uint32_t total,
                             uint32_t* dir) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  const uint64_t lo = i == 0 ? 0 : (uint64_t)toc_hash[i - 1] + 1;
  const uint64_t hi = i == n ? (1ull << 28) : (uint64_t)toc_hash[i];
  const uint32_t v = i == n ? total : (uint32_t)toc_start[i];
  for (uint64_t h = lo; h <= hi; h++) dir[h] = v;
}

// Hash slots from the directory and the postings: count, first posting and the first kSlotPosts
// postings of every 28-bit hash (zeros beyond the bucket).
__global__ void k_fill_slots(const uint32_t* dir, const uint2* post, uint4* slots) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t h = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; h < (1ull << 28); h += stride) {
    const uint32_t o = dir[h], cnt = dir[h + 1] - o;
    uint2 p[kSlotPosts];
#pragma unroll
    for (int t = 0; t < kSlotPosts; t++) p[t] = (uint32_t)t < cnt ? post[o + t] : make_uint2(0u, 0u);
    uint4* sl = slots + h * kSlotVecs;
    sl[0] = make_uint4(cnt, o, p[0].x, p[0].y);
    sl[1] = make_uint4(p[1].x, p[1].y, p[2].x, p[2].y);
    sl[2] = make_uint4(p[3].x, p[3].y, p[4].x, p[4].y);
    sl[3] = make_uint4(p[5].x, p[5].y, p[6].x, p[6].y);
  }
}

__global__ void k_log_probe(uint32_t lo_bits, uint32_t n, float* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = log_dev_raw(__uint_as_float(lo_bits + i));
}

__global__ void k_eval_logf(DevIndex ix, const float* x, float* out, uint64_t n, int* errw) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int err = 0;
  out[i] = ref_logf(ix, x[i], &err);
  if (err) atomicOr(errw, err);
}

// Scoring-only drop-in (MatrixCPU::CPUGetHighestScore): one thread per candidate, like the
// reference's CUDA kernel, with the semantics of CalculateScore.
__global__ void k_score_candidates(DevIndex ix, uint64_t n_strands, const uint64_t* q_off, const uint8_t* bases,
                                   const uint64_t* c_off, const uint32_t* cand_ref, const uint64_t* r_off,
                                   const uint32_t* runs, uint64_t n_cands, const uint64_t* cand_strand,
                                   float* score_out, float* pct_out, float* rel_out, uint32_t* hit_ws,
                                   uint64_t hit_words_per_thread, int* errw) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cands) return;
  const uint64_t s = cand_strand[c];
  const uint8_t* q = bases + q_off[s];
  const uint32_t L = (uint32_t)(q_off[s + 1] - q_off[s]);
  const uint32_t ref = cand_ref[c];
  const uint8_t* rs = ix.bases + ix.ref_off[ref];
  const uint32_t rlen = ix.ref_len[ref];
  const uint32_t k = (uint32_t)ix.k;
  uint32_t* hit = hit_ws + (uint64_t)c * hit_words_per_thread;
  const uint32_t nw = (L + 31) / 32;
  for (uint32_t w = 0; w < nw; w++) hit[w] = 0;
  uint64_t sc = 0, sr = 0;
  for (uint64_t r = r_off[c]; r < r_off[c + 1]; r++) {
    const uint32_t sref = runs[4 * r], sq = runs[4 * r + 1], lref = runs[4 * r + 2], lq = runs[4 * r + 3];
    if (sq > lq) continue;
    const uint32_t tail = tail_walk(q, rs, L, rlen, lq, lref, k);
    const uint32_t head = head_walk(q, rs, sq, sref, k);
    const uint64_t tot = (uint64_t)tail + head + (lq - sq);
    if (tot >= k) {
      sc += tot;
      sr += tot * (tot + 1) / 2;
      for (uint64_t p = sq - head; p < sq - head + tot; p++) hit[p >> 5] |= 1u << (p & 31);
    }
  }
  float score = -2.0f, pct = 0.0f, rel = -1.0f;
  int err = 0;
  if (sc > 0) {
    uint32_t hits = 0;
    for (uint32_t w = 0; w < nw; w++) hits += __popc(hit[w]);
    final_score(sr, sc, hits, L, &score, &pct);
    rel = relative_score(ix, __uint2float_rn(L), __uint2float_rn(rlen), score, &err);
  }
  score_out[c] = score;
  pct_out[c] = pct;
  rel_out[c] = rel;
  if (err) atomicOr(errw, err);
}

// ------------------------------------------------------------------------------ host side

}  // namespace mg

#include "mg_internal.h"

namespace mg {

// Compare the device log with the host libm logf over the whole domain and record where
// they differ, so that the device reproduces the reference's logf bit for bit.
// log_den[lm] = the denominator of relative_score at len_max = lm (its own code, so the values are
// the ones relative_score computes).
__global__ void k_fill_log_den(DevIndex ix, float* out) {
  const uint32_t lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm > 0xFFFFu) return;
  const double l = (double)__uint2float_rn(lm);
  const float score_max = __double2float_rn(__dadd_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(l, __dadd_rn(l, 1.0)), 2.0), l), 1.0));
  int err = 0;
  out[lm] = ref_logf(ix, score_max, &err);
}

static int build_log_table(mg_index* ix) {
  const uint32_t chunk = 1u << 23;
  DevBuf dprobe;
  if (dprobe.alloc((size_t)chunk * 4)) return set_error(MG_ERR_OOM, "log table probe");
  std::vector<float> dev(chunk);
  std::vector<uint32_t> keys;
  std::vector<float> vals;
  std::vector<uint32_t> bitmap(kLogDomain / 32, 0);
  int nt = std::max(1u, std::thread::hardware_concurrency());
  for (uint32_t lo = kLogLoBits; lo < kLogHiBits; lo += chunk) {
    uint32_t n = std::min<uint32_t>(chunk, kLogHiBits - lo);
    k_log_probe<<<(n + 255) / 256, 256, 0, ix->stream>>>(lo, n, dprobe.as<float>());
    CU(cudaMemcpyAsync(dev.data(), dprobe.p, (size_t)n * 4, cudaMemcpyDeviceToHost, ix->stream));
    CU(cudaStreamSynchronize(ix->stream));
    std::vector<std::vector<uint32_t>> lk(nt);
    std::vector<std::vector<float>> lv(nt);
    std::vector<std::thread> th;
    uint32_t per = (n + nt - 1) / nt;
    for (int t = 0; t < nt; t++)
      th.emplace_back([&, t] {
        uint32_t a = std::min(n, per * t), b = std::min(n, a + per);
        for (uint32_t i = a; i < b; i++) {
          uint32_t bits = lo + i;
          float x;
          std::memcpy(&x, &bits, 4);
          float h = logf(x);
          uint32_t hb, db;
          std::memcpy(&hb, &h, 4);
          std::memcpy(&db, &dev[i], 4);
          if (hb != db) {
            lk[t].push_back(bits);
            lv[t].push_back(h);
          }
        }
      });
    for (auto& x : th) x.join();
    for (int t = 0; t < nt; t++) {
      for (size_t j = 0; j < lk[t].size(); j++) {
        uint32_t r = lk[t][j] - kLogLoBits;
        bitmap[r >> 5] |= 1u << (r & 31);
        keys.push_back(lk[t][j]);
        vals.push_back(lv[t][j]);
      }
    }
  }
  dprobe.release();
  if (ix->logx_bitmap.alloc(bitmap.size() * 4) || ix->logx_keys.alloc(keys.size() * 4 + 4) ||
      ix->logx_vals.alloc(vals.size() * 4 + 4))
    return set_error(MG_ERR_OOM, "log table");
  CU(cudaMemcpy(ix->logx_bitmap.p, bitmap.data(), bitmap.size() * 4, cudaMemcpyHostToDevice));
  if (!keys.empty()) {
    CU(cudaMemcpy(ix->logx_keys.p, keys.data(), keys.size() * 4, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(ix->logx_vals.p, vals.data(), vals.size() * 4, cudaMemcpyHostToDevice));
  }
  ix->dix.logx_bitmap = ix->logx_bitmap.as<uint32_t>();
  ix->dix.logx_keys = ix->logx_keys.as<uint32_t>();
  ix->dix.logx_vals = ix->logx_vals.as<float>();
  ix->dix.n_logx = (uint32_t)keys.size();
  ix->device_bytes += bitmap.size() * 4 + keys.size() * 8;
  if (ix->log_den.alloc(65536 * 4)) return set_error(MG_ERR_OOM, "log table");
  k_fill_log_den<<<256, 256, 0, ix->stream>>>(ix->dix, ix->log_den.as<float>());
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(ix->stream));
  ix->dix.log_den = ix->log_den.as<float>();
  ix->device_bytes += 65536 * 4;
  return MG_OK;
}

// Hash slots (DevIndex::slots) are built at open for indexes of at least this many postings; the
// table takes 2^28 x 64 bytes (17.2 GB) whatever the index size, which small indexes do not repay.
constexpr uint64_t kSlotsFromPostings = 1ull << 25;

static int set_probe_slots(mg_index* ix, bool on) {
  if (!on) {
    ix->slots.release();
    ix->dix.slots = nullptr;
    return MG_OK;
  }
  if (ix->dix.slots) return MG_OK;
  if (ix->slots.alloc((1ull << 28) * kSlotVecs * sizeof(uint4)))
    return set_error(MG_ERR_OOM, "device memory for the hash slots");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
  k_fill_slots<<<(unsigned)sms * 8, 256, 0, ix->stream>>>(ix->dix.dir, ix->dix.post, ix->slots.as<uint4>());
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(ix->stream));
  ix->dix.slots = ix->slots.as<uint4>();
  return MG_OK;
}

// The HBM index from a .mhm image: the host parses the header and reference tables; the image
// is copied to the device once and the bucket TOC and posting records are decoded there.
static int upload_index_image(mg_index* ix, const uint8_t* image, uint64_t L, const MhmMeta& meta, int k) {
  MhmIndex& h = ix->host;
  const uint64_t n = h.n_hash;
  CU(cudaStreamCreateWithFlags(&ix->stream, cudaStreamNonBlocking));
  cudaStream_t st = ix->stream;
  DevBuf img, dhash, dsp, dcnt, dstart, derr, tmp;
  if (img.alloc(L + 16) || dhash.alloc(n * 4 + 4) || dsp.alloc(n * 8 + 8) || dcnt.alloc(n * 8 + 8) ||
      dstart.alloc(n * 8 + 8) || derr.alloc(4))
    return set_error(MG_ERR_OOM, "device memory for the index image");
  CU(cudaMemcpy(img.p, image, L, cudaMemcpyHostToDevice));
  CU(cudaMemsetAsync(derr.p, 0, 4, st));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
  const unsigned grid = (unsigned)sms * 8;
  uint64_t total = 0;
  int err = 0;
  if (n) {
    k_mhm_toc<<<grid, 256, 0, st>>>(img.as<uint8_t>(), meta.toc_at, n, h.word, dhash.as<uint32_t>(),
                                     dsp.as<uint64_t>(), derr.as<int>());
    k_mhm_count<<<grid, 256, 0, st>>>(img.as<uint8_t>(), L, dhash.as<uint32_t>(), dsp.as<uint64_t>(), n,
                                       dcnt.as<uint64_t>(), derr.as<int>());
    CU(cudaGetLastError());
    size_t tb = 0;
    CU(cub::DeviceScan::ExclusiveSum(nullptr, tb, dcnt.as<uint64_t>(), dstart.as<uint64_t>(), (int64_t)n, st));
    if (tmp.alloc(tb + 16)) return set_error(MG_ERR_OOM, "device memory for the index scan");
    CU(cub::DeviceScan::ExclusiveSum(tmp.p, tb, dcnt.as<uint64_t>(), dstart.as<uint64_t>(), (int64_t)n, st));
    uint64_t ls = 0, lc = 0;
    CU(cudaMemcpyAsync(&ls, dstart.as<uint64_t>() + n - 1, 8, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(&lc, dcnt.as<uint64_t>() + n - 1, 8, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(&err, derr.p, 4, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    total = ls + lc;
    if (err & kDecHash) return set_error(MG_ERR_BADFMT, "hash wider than 28 bits");
    if (err & kDecRecord) return set_error(MG_ERR_BADFMT, "malformed posting record");
    if (err & kDecOrder) return set_error(MG_ERR_BADFMT, "TOC hashes not strictly ascending");
  }
  if (total >= 0xFFFFFFFFull) return set_error(MG_ERR_LIMIT, "more than 2^32-1 postings");
  if (ix->dir.alloc(((1ull << 28) + 1) * 4) || ix->post.alloc(total * 8 + 8) || ix->bases.alloc(meta.bases_len + 64) ||
      ix->ref_off.alloc(h.ref_off.size() * 8 + 8) || ix->ref_len.alloc(h.ref_len.size() * 4 + 4))
    return set_error(MG_ERR_OOM, "device allocation for the index");
  ix->device_bytes += ix->dir.n + ix->post.n + ix->bases.n + ix->ref_off.n + ix->ref_len.n;
  if (n) {
    k_mhm_decode<<<grid, 256, 0, st>>>(img.as<uint8_t>(), L, dsp.as<uint64_t>(), dcnt.as<uint64_t>(),
                                        dstart.as<uint64_t>(), n, h.word, h.n_refs, ix->post.as<uint2>(),
                                        derr.as<int>());
    CU(cudaGetLastError());
  }
  if (meta.bases_len)
    CU(cudaMemcpyAsync(ix->bases.p, img.as<uint8_t>() + meta.bases_at, meta.bases_len, cudaMemcpyDeviceToDevice, st));
  CU(cudaMemcpyAsync(ix->ref_off.p, h.ref_off.data(), h.ref_off.size() * 8, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(ix->ref_len.p, h.ref_len.data(), h.ref_len.size() * 4, cudaMemcpyHostToDevice, st));
  k_fill_dir64<<<(unsigned)((n + 1 + 255) / 256), 256, 0, st>>>(dhash.as<uint32_t>(), dstart.as<uint64_t>(), n,
                                                                 (uint32_t)total, ix->dir.as<uint32_t>());
  CU(cudaGetLastError());
  uint32_t last_hash = 0;
  if (n) CU(cudaMemcpyAsync(&last_hash, dhash.as<uint32_t>() + n - 1, 4, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(&err, derr.p, 4, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if (err & kDecRecord) return set_error(MG_ERR_BADFMT, "malformed posting record");
  h.has_empty_last = n > 0;
  h.empty_last_hash = last_hash;
  ix->info.n_postings = total;
  DevIndex& d = ix->dix;
  d.dir = ix->dir.as<uint32_t>();
  d.post = ix->post.as<uint2>();
  d.bases = ix->bases.as<uint8_t>();
  d.ref_off = ix->ref_off.as<uint64_t>();
  d.ref_len = ix->ref_len.as<uint32_t>();
  d.n_refs = h.n_refs;
  d.empty_hash = h.has_empty_last ? h.empty_last_hash : 0xFFFFFFFFu;
  d.k = k;
  d.step = k / 2;
  d.hlen = k - k / 2 + 1;
  if (total >= kSlotsFromPostings) {
    const int rc = set_probe_slots(ix, true);
    if (rc) return rc;
  }
  return build_log_table(ix);
}

static void load_tuning(mg_index* ix);

static int open_image(mg_index* ix, const uint8_t* image, uint64_t L, int k, int device) {
  ix->device = device;
  CU(cudaSetDevice(device));
  std::string err;
  MhmMeta meta;
  auto t0 = std::chrono::steady_clock::now();
  int rc = mhm_parse_meta(image, L, k, &ix->host, &meta, false, &err);
  if (rc != MHM_OK)
    return set_error(rc == MHM_ERR_IO ? MG_ERR_IO : rc == MHM_ERR_OOM ? MG_ERR_OOM : rc == MHM_ERR_LIMIT ? MG_ERR_LIMIT : MG_ERR_BADFMT, err);
  auto t1 = std::chrono::steady_clock::now();
  ix->info.load_seconds += std::chrono::duration<double>(t1 - t0).count();
  rc = upload_index_image(ix, image, L, meta, k);
  ix->info.upload_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  ix->info.k = k;
  ix->info.word = ix->host.word;
  ix->info.n_hashes = ix->host.n_hash;
  ix->info.n_refs = ix->host.n_refs;
  ix->info.ref_bases = meta.bases_len;
  ix->info.device_bytes = ix->device_bytes;
  if (rc == MG_OK) load_tuning(ix);
  return rc;
}

// ---------------------------------------------------------------------- classification

// ---------------------------------------------------------------------- launch shapes

// The launch shapes in effect: mg_tuning's fields with the defaults filled in and clamped to what
// the kernels can be launched with.
struct Shapes {
  unsigned dual_blocks_per_sm, steal_chunk, first_tier, second_blocks_per_sm, finish_blocks_per_sm,
      long_blocks_per_sm, chunks, weighted_chunks, third_blocks_per_sm, pack_bases;
  unsigned long_small_blocks_per_sm;  // the smaller long-read size: its occupancy (not tuned)
};

static int occupancy(const void* fn, int threads, size_t smem) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem);
  return std::max(1, n);
}

static Shapes shapes(const mg_index* ix) {
  static int occ_dual = 0, occ_second = 0, occ_third = 0, occ_long = 0, occ_long_s = 0;
  if (!occ_dual) {
    cudaFuncSetAttribute(k_classify_long<LongSmem, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(LongSmem));
    cudaFuncSetAttribute(k_classify_long<LongSmemS, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(LongSmemS));
    occ_second = occupancy((const void*)k_classify_dual_list<128, kW2Warps>, kW2Warps * 32, 0);
    occ_third = occupancy((const void*)k_classify_dual_list<256, kW3Warps>, kW3Warps * 32, 0);
    occ_long = occupancy((const void*)k_classify_long<LongSmem, 2>, kLgThreads, sizeof(LongSmem));
    occ_long_s = occupancy((const void*)k_classify_long<LongSmemS, 4>, kLgThreads, sizeof(LongSmemS));
    occ_dual = occupancy((const void*)k_classify_dual, kW1Warps * 32, 0);
  }
  const mg_tuning& t = ix->tune;
  auto pick = [](uint32_t v, unsigned def, unsigned lo, unsigned hi) {
    return v ? std::min<unsigned>(hi, std::max<unsigned>(lo, v)) : def;
  };
  Shapes s;
  s.first_tier = pick(t.first_tier, 1, 1, 3);
  s.dual_blocks_per_sm = pick(t.dual_blocks_per_sm, (unsigned)occ_dual, 1, (unsigned)occ_dual);
  s.steal_chunk = pick(t.steal_chunk, kW1Chunk, 1, 64);
  // the 128-posting tier takes the first tier's few leftovers (one block per SM), or every read
  s.second_blocks_per_sm = pick(t.second_blocks_per_sm, s.first_tier == 2 ? (unsigned)occ_second : 1u, 1,
                                (unsigned)occ_second);
  s.third_blocks_per_sm = pick(t.third_blocks_per_sm, (unsigned)occ_third, 1, (unsigned)occ_third);
  s.pack_bases = pick(t.pack_bases, 1, 1, 2);
  s.finish_blocks_per_sm = pick(t.finish_blocks_per_sm, 8, 1, 8);
  s.long_blocks_per_sm = pick(t.long_blocks_per_sm, (unsigned)occ_long, 1, (unsigned)occ_long);
  s.long_small_blocks_per_sm = (unsigned)occ_long_s;
  s.chunks = pick(t.chunks, mg_index::kMaxChunks, 1, mg_index::kMaxChunks);
  s.weighted_chunks = pick(t.weighted_chunks, 1, 1, 2);
  return s;
}

// Density class of an index (postings per 28-bit hash), the key of the tuning file's entries.
static const char* density_class(uint64_t n_postings) {
  const double d = (double)n_postings / (double)(1ull << 28);
  return d < 0.25 ? "sparse" : d < 4.0 ? "dense" : "saturated";
}

// Launch shapes from the tuning file of this GPU model: MG_TUNING_FILE, else
// tuning/<device name, spaces as '_'>.txt beside the library. A line "<class> key=value ..."
// sets the fields it names for indexes of that density class; '#' starts a comment.
static void load_tuning(mg_index* ix) {
  std::string path;
  if (const char* e = std::getenv("MG_TUNING_FILE")) {
    path = e;
  } else {
    Dl_info info;
    if (!dladdr((const void*)&load_tuning, &info) || !info.dli_fname) return;
    std::string lib = info.dli_fname;
    const size_t slash = lib.rfind('/');
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, ix->device) != cudaSuccess) return;
    std::string name = p.name;
    for (char& c : name)
      if (c == ' ' || c == '/') c = '_';
    path = (slash == std::string::npos ? std::string(".") : lib.substr(0, slash)) + "/tuning/" + name + ".txt";
  }
  std::ifstream f(path);
  if (!f) return;
  const std::string cls = density_class(ix->info.n_postings);
  std::string line;
  while (std::getline(f, line)) {
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    size_t p = line.find_first_not_of(" \t");
    if (p == std::string::npos) continue;
    size_t q = line.find_first_of(" \t", p);
    if (line.substr(p, q == std::string::npos ? std::string::npos : q - p) != cls) continue;
    while (q != std::string::npos) {
      p = line.find_first_not_of(" \t", q);
      if (p == std::string::npos) break;
      q = line.find_first_of(" \t", p);
      const std::string kv = line.substr(p, q == std::string::npos ? std::string::npos : q - p);
      const size_t eq = kv.find('=');
      if (eq == std::string::npos) continue;
      const std::string k = kv.substr(0, eq);
      const uint32_t v = (uint32_t)std::strtoul(kv.c_str() + eq + 1, nullptr, 10);
      mg_tuning& t = ix->tune;
      if (k == "dual_blocks_per_sm") t.dual_blocks_per_sm = v;
      else if (k == "steal_chunk") t.steal_chunk = v;
      else if (k == "first_tier") t.first_tier = v;
      else if (k == "second_blocks_per_sm") t.second_blocks_per_sm = v;
      else if (k == "finish_blocks_per_sm") t.finish_blocks_per_sm = v;
      else if (k == "long_blocks_per_sm") t.long_blocks_per_sm = v;
      else if (k == "chunks") t.chunks = v;
      else if (k == "weighted_chunks") t.weighted_chunks = v;
      else if (k == "third_blocks_per_sm") t.third_blocks_per_sm = v;
      else if (k == "pack_bases") t.pack_bases = v;
    }
  }
}

int ensure_workspace(Workspace& w, uint64_t n_reads, uint64_t n_bases, bool host_io) {
  uint64_t arena_cap = std::max<uint64_t>(1 << 16, n_reads * 2);
  if (host_io) {
    if (w.offs.alloc((n_reads + 1) * 8) || w.bases.alloc(n_bases + 16) ||
        w.reads.alloc(n_reads * sizeof(mg_read_result) + 16))
      return set_error(MG_ERR_OOM, "batch buffers");
  }
  if (w.stage.alloc(n_reads * kSlots * sizeof(mg_candidate) + 16) ||
      w.arena.alloc(arena_cap * sizeof(mg_candidate)) || w.ctr.alloc(256) ||
      w.ovf.alloc(8 * (n_reads + 4) * 4 + 16) || w.sums.alloc(((n_reads + kScanBlock - 1) / kScanBlock + 1) * 8))
    return set_error(MG_ERR_OOM, "staging buffers");
  const WsLayout l3 = ws_layout(kB3Q, kB3Seeds, kB3E, kB3C);
  if (w.gws.alloc(l3.total * kB3Blocks)) return set_error(MG_ERR_OOM, "global workspace");
  return MG_OK;
}

// Counters in w_ctr (device): 0 n_cands(u64) | 8 arena_n(u64) | 16 err | 20 work | 24 n_ovf1 |
// 28 work2 | 32 n_ovf2 | 36 work3 | 40 total(u64) | 48 n_ovf0 | 52 work1 | 56 n_ovf0b | 60 work0b |
// 64 n_ovf1b | 68 work of the smaller long-read size | 72 n_ovf0c | 76 work0c | 80 n_ovf1c |
// 84 work of the larger long-read size | 88 n_ovf3 (the global tier's leftovers) | 92 work4 |
// 96 oversize need: most bases, seeds, postings, reads waiting (4 x u32)
int run_pipeline(mg_index* ix, Workspace& w, uint64_t n, const uint64_t* d_offs, const uint8_t* d_bases,
                        mg_read_result* d_reads, mg_candidate* d_out, uint64_t cap, cudaStream_t st,
                        bool plain, unsigned long long* chain, const ChainSync* cs) {
  uint8_t* ctr = w.ctr.as<uint8_t>();
  CU(cudaMemsetAsync(ctr, 0, 256, st));
  BatchDev b;
  b.n = n;
  b.offs = d_offs;
  b.bases = d_bases;
  b.reads = d_reads;
  b.cands = d_out;
  b.cand_cap = cap;
  b.n_cands = (unsigned long long*)(ctr + 0);
  b.err = chain ? (int*)(chain + 1) : (int*)(ctr + 16);
  b.work = (unsigned*)(ctr + 20);
  b.n_ovf1 = (unsigned*)(ctr + 24);
  b.work2 = (unsigned*)(ctr + 28);
  b.n_ovf2 = (unsigned*)(ctr + 32);
  b.work3 = (unsigned*)(ctr + 36);
  b.n_ovf0 = (unsigned*)(ctr + 48);
  b.work1 = (unsigned*)(ctr + 52);
  b.n_ovf0b = (unsigned*)(ctr + 56);
  b.work0b = (unsigned*)(ctr + 60);
  b.ovf0 = w.ovf.as<uint32_t>();
  b.ovf0b = w.ovf.as<uint32_t>() + 3 * (n + 4);
  b.ovf1 = w.ovf.as<uint32_t>() + n + 4;
  b.ovf2 = w.ovf.as<uint32_t>() + 2 * (n + 4);
  uint32_t* ovf1b = w.ovf.as<uint32_t>() + 4 * (n + 4);  // the long-read tier's leftovers
  unsigned* n_ovf1b = (unsigned*)(ctr + 64);
  unsigned* work_long = (unsigned*)(ctr + 68);
  uint32_t* ovf0c = w.ovf.as<uint32_t>() + 5 * (n + 4);  // the 128-posting tier's leftovers
  unsigned* n_ovf0c = (unsigned*)(ctr + 72);
  unsigned* work0c = (unsigned*)(ctr + 76);
  uint32_t* ovf1c = w.ovf.as<uint32_t>() + 6 * (n + 4);  // the smaller long-read size's leftovers
  unsigned* n_ovf1c = (unsigned*)(ctr + 80);
  unsigned* work_long2 = (unsigned*)(ctr + 84);
  uint32_t* ovf3 = w.ovf.as<uint32_t>() + 7 * (n + 4);  // the global tier's leftovers
  unsigned* n_ovf3 = (unsigned*)(ctr + 88);
  unsigned* work4 = (unsigned*)(ctr + 92);
  unsigned* huge_need = (unsigned*)(ctr + 96);
  StageDev sd;
  sd.stage = w.stage.as<mg_candidate>();
  sd.arena = w.arena.as<mg_candidate>();
  sd.arena_cap = w.arena.n / sizeof(mg_candidate);
  sd.arena_n = (unsigned long long*)(ctr + 8);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
  const WsLayout l2 = ws_layout(kB2Q, kB2Seeds, kB2E, kB2C);
  const WsLayout l3 = ws_layout(kB3Q, kB3Seeds, kB3E, kB3C);
  const Caps c2{kB2Q, kB2Seeds, kB2E, kB2C}, c3{kB3Q, kB3Seeds, kB3E, kB3C};
  const WsLayout lh = ws_layout((int)w.hq, (int)w.hseeds, (int)w.he, (int)w.hc, true);
  const Caps ch{(int)w.hq, (int)w.hseeds, (int)w.he, (int)w.hc};
  static bool attr_set = false;
  if (!attr_set) {
    CU(cudaFuncSetAttribute(k_classify_block<kB2Threads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l2.total));
    CU(cudaFuncSetAttribute(k_classify_long<LongSmem, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(LongSmem)));
    CU(cudaFuncSetAttribute(k_classify_long<LongSmemS, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(LongSmemS)));
    attr_set = true;
  }
  const bool tm = ix->timing && ix->events_made;
  if (n > 0) {
    // timing events (start, end) per tier: ev[0..1] first tier, ev[2..3] general warp tier,
    // ev[3..4] block tier, ev[4..5] global tier, ev[6..7] compaction
    if (tm) CU(cudaEventRecord(ix->ev[0], st));
    auto global_tier = [&](cudaStream_t s) {
      k_classify_block<kB3Threads><<<kB3Blocks, kB3Threads, 0, s>>>(ix->dix, b, sd, b.ovf2, b.n_ovf2, b.work3, ovf3,
                                                                    n_ovf3, w.gws.as<uint8_t>(), l3, c3, !w.hmode);
      // the oversize tier, once a batch of this workspace has needed it: one block while it has
      // no workspace (it only sizes the reads it gets)
      if (w.hmode)
        k_classify_huge<kHugeThreads><<<(unsigned)std::max(1, w.hslabs), kHugeThreads, 0, s>>>(
            ix->dix, b, sd, ovf3, n_ovf3, work4, w.hslabs ? w.hws.as<uint8_t>() : nullptr, lh, ch, huge_need);
    };
    if (plain) {
      // every read gets its own block (one launch for the batch)
      k_classify_block<kB2Threads><<<(unsigned)n, kB2Threads, l2.total, st>>>(
          ix->dix, b, sd, nullptr, nullptr, nullptr, b.ovf2, b.n_ovf2, nullptr, l2, c2, 0);
      if (tm) {
        CU(cudaEventRecord(ix->ev[1], st));
        CU(cudaEventRecord(ix->ev[2], st));
        CU(cudaEventRecord(ix->ev[3], st));
        CU(cudaEventRecord(ix->ev[4], st));
      }
      global_tier(st);
      if (tm) CU(cudaEventRecord(ix->ev[5], st));
    } else {
      if (!w.side) {
        CU(cudaStreamCreateWithFlags(&w.side, cudaStreamNonBlocking));
        CU(cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&w.join, cudaEventDisableTiming));
      }
      const Shapes sh = shapes(ix);
      if (sh.first_tier == 1)
        k_classify_dual<<<sh.dual_blocks_per_sm * sms, kW1Warps * 32, 0, st>>>(ix->dix, b, sd, sh.steal_chunk);
      // tiers of 64, 128 and 256 postings per strand, each over the one before's leftovers
      if (sh.first_tier <= 2)
        k_classify_dual_list<128, kW2Warps><<<sh.second_blocks_per_sm * sms, kW2Warps * 32, 0, st>>>(
            ix->dix, b, sd, b.ovf0, b.n_ovf0, b.work0b, ovf0c, n_ovf0c, sh.first_tier == 2);
      k_classify_dual_list<256, kW3Warps><<<sh.third_blocks_per_sm * sms, kW3Warps * 32, 0, st>>>(
          ix->dix, b, sd, ovf0c, n_ovf0c, work0c, b.ovf0b, b.n_ovf0b, sh.first_tier == 3);
      // the reads the dual tiers handed on go through the other tiers on the side stream, beside
      // the dual tier's finishing pass (different reads, disjoint slots; arena space by atomics)
      CU(cudaEventRecord(w.fork, st));
      CU(cudaStreamWaitEvent(w.side, w.fork, 0));
      if (tm) CU(cudaEventRecord(ix->ev[2], w.side));
      static int per_sm2 = 0;  // the same on every call (one architecture): queried once
      if (!per_sm2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_classify_warp_list, kW1Warps * 32, 0);
      k_classify_warp_list<<<(unsigned)std::max(1, per_sm2) * sms, kW1Warps * 32, 0, w.side>>>(ix->dix, b, sd);
      if (tm) CU(cudaEventRecord(ix->ev[3], w.side));
      k_classify_long<LongSmemS, 4><<<sh.long_small_blocks_per_sm * sms, kLgThreads, sizeof(LongSmemS), w.side>>>(
          ix->dix, b, sd, b.ovf1, b.n_ovf1, work_long, ovf1c, n_ovf1c);
      k_classify_long<LongSmem, 2><<<sh.long_blocks_per_sm * sms, kLgThreads, sizeof(LongSmem), w.side>>>(
          ix->dix, b, sd, ovf1c, n_ovf1c, work_long2, ovf1b, n_ovf1b);
      k_classify_block<kB2Threads><<<(unsigned)sms, kB2Threads, l2.total, w.side>>>(
          ix->dix, b, sd, ovf1b, n_ovf1b, b.work2, b.ovf2, b.n_ovf2, nullptr, l2, c2, 0);
      if (tm) CU(cudaEventRecord(ix->ev[4], w.side));
      global_tier(w.side);
      if (tm) CU(cudaEventRecord(ix->ev[5], w.side));
      CU(cudaEventRecord(w.join, w.side));
      k_finish_dual<<<(unsigned)std::min<uint64_t>((n + kFinThreads - 1) / kFinThreads,
                                                   (uint64_t)sms * sh.finish_blocks_per_sm),
                      kFinThreads, 0, st>>>(ix->dix, b, sd);
      if (tm) CU(cudaEventRecord(ix->ev[1], st));
      CU(cudaStreamWaitEvent(st, w.join, 0));
    }
    CU(cudaGetLastError());
    if (tm) CU(cudaEventRecord(ix->ev[6], st));
    const uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
    unsigned long long* sums = w.sums.as<unsigned long long>();
    k_count_sums<<<(unsigned)nb, kScanBlock, 0, st>>>(d_reads, n, sums);
    if (cs && cs->wait_prev) CU(cudaStreamWaitEvent(st, cs->wait_prev, 0));
    k_scan_sums<<<1, kScanBlock, 0, st>>>(sums, nb, (unsigned long long*)(ctr + 40), chain);
    if (cs && cs->snap) CU(cudaMemcpyAsync(cs->snap, chain, 8, cudaMemcpyDeviceToHost, st));
    if (cs && cs->scanned) CU(cudaEventRecord(cs->scanned, st));
    k_scatter<<<(unsigned)nb, kScanBlock, 0, st>>>(d_reads, n, sums, sd, d_out, cap, b.err);
    if (tm) CU(cudaEventRecord(ix->ev[7], st));
    CU(cudaGetLastError());
  }
  return MG_OK;
}

int read_counters(Workspace& w, cudaStream_t st, Counters* c) {
  uint8_t h[112];
  CU(cudaMemcpyAsync(h, w.ctr.p, 112, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  unsigned long long total, need;
  std::memcpy(&c->err, h + 16, 4);
  std::memcpy(&need, h + 8, 8);
  std::memcpy(&total, h + 40, 8);
  std::memcpy(c->huge_need, h + 96, 16);
  c->n_cands = total;
  c->arena_need = need;
  return MG_OK;
}

// Grow the oversize tier's slabs to hold every read the last run sized (and every read the old
// slabs held): one slab per waiting read, up to kHugeMaxSlabs and kHugeMaxBytes in all.
static int grow_oversize(mg_index* ix, Workspace& w, const Counters& c) {
  const uint32_t q = std::max(w.hq, c.huge_need[0]), seeds = std::max(w.hseeds, c.huge_need[1]);
  uint32_t e = 1;
  while (e < std::max(w.he, c.huge_need[2])) e <<= 1;
  const uint32_t cand = std::min<uint32_t>(std::min<uint32_t>(e, std::max<uint32_t>(ix->dix.n_refs, 1)), 65535);
  const WsLayout l = ws_layout((int)q, (int)seeds, (int)e, (int)cand, true);
  const uint64_t fit = std::max<uint64_t>(1, kHugeMaxBytes / l.total);
  const int slabs = (int)std::min<uint64_t>(std::min<uint64_t>(std::max<uint64_t>(w.hslabs, c.huge_need[3]), kHugeMaxSlabs), fit);
  if (w.hws.alloc(l.total * (size_t)slabs)) {
    w.hslabs = 0;
    w.hq = w.hseeds = w.he = w.hc = 0;
    return set_error(MG_ERR_OOM, "oversize-read workspace");
  }
  w.hslabs = slabs;
  w.hq = q;
  w.hseeds = seeds;
  w.he = e;
  w.hc = cand;
  return MG_OK;
}

int complete_pipeline(mg_index* ix, Workspace& w, uint64_t n, const uint64_t* d_offs, const uint8_t* d_bases,
                      mg_read_result* d_reads, mg_candidate* d_out, uint64_t cap, cudaStream_t st, bool plain,
                      Counters* c) {
  int rc = read_counters(w, st, c);
  // a rerun can need another: the first oversize read turns the oversize tier on, its next run
  // sizes the reads, and their candidates go to the arena only once they fit
  for (int attempt = 0; rc == MG_OK && attempt < 4 && (c->err & (kErrArena | kErrHuge)); attempt++) {
    if ((c->err & kErrArena) &&
        w.arena.alloc((c->arena_need + (c->arena_need >> 3) + 1024) * sizeof(mg_candidate)))
      return set_error(MG_ERR_OOM, "staging arena");
    if (c->err & kErrHuge) {
      if (!w.hmode) {
        w.hmode = 1;
      } else {
        rc = grow_oversize(ix, w, *c);
        if (rc) return rc;
      }
    }
    rc = run_pipeline(ix, w, n, d_offs, d_bases, d_reads, d_out, cap, st, plain);
    c->reran = true;
    if (rc == MG_OK) rc = read_counters(w, st, c);
  }
  return rc;
}

int finish_errors(Workspace& w, cudaStream_t st, uint64_t* n_cands) {
  Counters c;
  const int rc = read_counters(w, st, &c);
  *n_cands = c.n_cands;
  return rc ? rc : error_status(c.err);
}

int error_status(int err) {
  if (err & kErrBadInput) return set_error(MG_ERR_BADINPUT, "a read holds a byte without a reverse complement");
  if (err & kErrLimit) return set_error(MG_ERR_LIMIT, "a read exceeds the largest workspace tier");
  if (err & kErrOutput) return set_error(MG_ERR_OOM, "candidate output buffer too small");
  if (err & kErrLogRange) return set_error(MG_ERR_LIMIT, "relative-score logarithm outside its exact domain");
  if (err & kErrArena) return set_error(MG_ERR_OOM, "staging arena too small");
  if (err & kErrHuge) return set_error(MG_ERR_LIMIT, "a read needs a larger oversize-read workspace");
  if (err & kErrInternal) return set_error(MG_ERR_CUDA, "a device loop reached its bound (internal error)");
  return MG_OK;
}

// Smallest chunk of the batched form with host buffers: a batch of fewer than twice this runs in
// one piece, and from kMaxChunks times this on the chunks are weighted (1,000,000 reads: 8
// chunks, the first and last 55,556 reads).
constexpr uint64_t kChunkReads = 65536;
constexpr uint64_t kChunkBases = kChunkReads * 192;  // the same size in bases, for long reads

// Chunks of a host-buffer batch: by reads or by bases, whichever gives more (long reads fill a
// chunk with few of them); 1 or less runs the batch in one piece.
static uint64_t chunk_units(uint64_t n, uint64_t n_bases) {
  return std::min<uint64_t>(n, std::max<uint64_t>(n / kChunkReads, n_bases / kChunkBases));
}
constexpr int kRunWhole = 1;

// Threads of the packed upload's pool: one per CPU this process may run on, at most 32 (a thread
// packs at about the rate one core reads memory, 5-10 GB/s).
static int pack_threads() {
  cpu_set_t set;
  int n = 0;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) n = CPU_COUNT(&set);
  if (n <= 0) n = (int)std::thread::hardware_concurrency();
  return std::max(1, std::min(32, n));
}

// Batched form with host buffers, in chunks: chunk i's offsets and bases are copied on the index's h2d stream
// while chunk i-1 is classified on its compute stream, and chunk i's read results go back on the
// d2h stream while chunk i+1 is classified. The chunks share the device output: the compaction
// continues the candidate offsets of the earlier chunks (run_pipeline's chain), so cand_off is an
// offset into the whole batch's candidates, as in one piece. Returns kRunWhole when a chunk's
// staging arena overflowed (the caller then runs the batch in one piece, which grows it).
static int classify_chunked(mg_index* ix, Workspace& w, const mg_batch* batch, mg_result* out) {
  const uint64_t n = batch->n_reads;
  if (!ix->chunk_made) {
    CU(cudaStreamCreateWithFlags(&ix->h2d, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&ix->d2h, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&ix->stream2, cudaStreamNonBlocking));
    for (int i = 0; i < mg_index::kMaxChunks; i++) {
      CU(cudaEventCreateWithFlags(&ix->ev_in[i], cudaEventDisableTiming));
      CU(cudaEventCreateWithFlags(&ix->ev_done[i], cudaEventDisableTiming));
      CU(cudaEventCreateWithFlags(&ix->ev_scan[i], cudaEventDisableTiming));
    }
    CU(cudaMallocHost((void**)&ix->h_snap, mg_index::kMaxChunks * 8));
    ix->chunk_made = true;
  }
  if (w.chain.alloc(16)) return set_error(MG_ERR_OOM, "chunk counters");
  const Shapes sh = shapes(ix);
  const int nc = (int)std::min<uint64_t>(sh.chunks, chunk_units(n, batch->offsets[n]));
  // chunk boundaries, weighted so that the first chunk (whose upload nothing hides) and the last
  // (whose classification and copy back nothing hides) are the smallest
  static const int kWeight[mg_index::kMaxChunks] = {1, 2, 3, 3, 3, 3, 2, 1};
  uint64_t bound[mg_index::kMaxChunks + 1];
  {
    const bool weighted = nc == mg_index::kMaxChunks && sh.weighted_chunks == 1;
    uint64_t wsum = 0, acc = 0;
    for (int i = 0; i < nc; i++) wsum += weighted ? kWeight[i] : 1;
    bound[0] = 0;
    for (int i = 0; i < nc; i++) {
      acc += weighted ? kWeight[i] : 1;
      bound[i + 1] = n * acc / wsum;
    }
  }
  uint64_t max_chunk = 0;
  for (int i = 0; i < nc; i++) max_chunk = std::max(max_chunk, bound[i + 1] - bound[i]);
  // the odd chunks run on a second stream with their own scratch, so that one chunk's tail
  // overlaps the next chunk's start; the compaction scans stay in chunk order
  int rc = ensure_workspace(ix->ws2, max_chunk + 1, 0, false);
  if (rc) return rc;
  cudaStream_t cst[2] = {ix->stream, ix->stream2};
  Workspace* cws[2] = {&w, &ix->ws2};
  unsigned long long* chain = w.chain.as<unsigned long long>();
  CU(cudaMemsetAsync(chain, 0, 16, ix->h2d));
  // packed upload: pinned staging for every chunk's packed bases and exceptions (a chunk with more
  // exceptions than its share goes up as given)
  const bool pack = sh.pack_bases == 2;
  const uint64_t n_bases = batch->offsets[n];
  const uint64_t pack_need = n_bases / 4 + 64 * (uint64_t)(nc + 1), exc_need = n_bases / 32 + 4096 * (uint64_t)nc;
  if (pack) {
    if (!ix->pack_pool)
      ix->pack_pool = new PackPool(std::max(1, pack_threads() - 1));  // a CPU left for the launches
    if (ix->h_pack_cap < pack_need) {
      if (ix->h_pack) cudaFreeHost(ix->h_pack);
      ix->h_pack = nullptr;
      ix->h_pack_cap = 0;
      CU(cudaMallocHost((void**)&ix->h_pack, pack_need));
      ix->h_pack_cap = pack_need;
    }
    if (ix->h_exc_cap < exc_need) {
      if (ix->h_exc) cudaFreeHost(ix->h_exc);
      ix->h_exc = nullptr;
      ix->h_exc_cap = 0;
      CU(cudaMallocHost((void**)&ix->h_exc, exc_need * 8));
      ix->h_exc_cap = exc_need;
    }
    if (w.packed.alloc(pack_need) || w.exc.alloc(exc_need * 8)) return set_error(MG_ERR_OOM, "packed staging");
  }
  // the packed upload: a packer thread packs the chunks in order, ahead of this thread, which
  // enqueues each chunk's copies and kernels once its bytes are packed; each chunk has its own
  // staging region and an equal share of the exception staging (a chunk with more exceptions
  // goes up as given)
  uint64_t pk_at[mg_index::kMaxChunks + 1] = {0};
  const uint64_t exc_share = exc_need / (uint64_t)std::max(1, nc);
  for (int i = 0; i < nc; i++) {
    const uint64_t nb_i = batch->offsets[bound[i + 1]] - batch->offsets[bound[i]];
    pk_at[i + 1] = pk_at[i] + ((nb_i + 3) / 4 + 15) / 16 * 16;
  }
  struct Packer {
    std::mutex mu;
    std::condition_variable cv;
    int64_t n_exc[mg_index::kMaxChunks];  // per chunk: exceptions, -1 not packed yet, -2 too many
    std::atomic<bool> stop{false};
    std::thread th;
    ~Packer() {  // joined on every way out of the call
      stop = true;
      if (th.joinable()) th.join();
    }
  } packer;
  for (int i = 0; i < mg_index::kMaxChunks; i++) packer.n_exc[i] = -1;
  if (pack) {
    packer.th = std::thread([&] {
      for (int i = 0; i < nc && !packer.stop; i++) {
        const uint64_t b0 = batch->offsets[bound[i]], b1 = batch->offsets[bound[i + 1]];
        uint64_t ne = 0;
        if (b1 > b0)
          pack_bases(*ix->pack_pool, batch->bases + b0, b1 - b0, ix->h_pack + pk_at[i], ix->h_exc + i * exc_share,
                     exc_share, &ne);
        std::lock_guard<std::mutex> lk(packer.mu);
        packer.n_exc[i] = ne <= exc_share ? (int64_t)ne : -2;
        packer.cv.notify_one();
      }
    });
  }
  for (int i = 0; i < nc && rc == MG_OK; i++) {
    const uint64_t r0 = bound[i], r1 = bound[i + 1];
    const uint64_t b0 = batch->offsets[r0], b1 = batch->offsets[r1];
    cudaStream_t st = cst[i & 1];
    // each chunk's offsets travel with its bases (the shared boundary entry twice, same value)
    CU(cudaMemcpyAsync(w.offs.as<uint64_t>() + r0, batch->offsets + r0, (r1 - r0 + 1) * 8, cudaMemcpyHostToDevice,
                       ix->h2d));
    bool packed = false;
    uint64_t n_exc = 0;
    const uint64_t pb = (b1 - b0 + 3) / 4, pk = pk_at[i], ek = (uint64_t)i * exc_share;
    if (pack && b1 > b0) {
      std::unique_lock<std::mutex> lk(packer.mu);
      packer.cv.wait(lk, [&] { return packer.n_exc[i] != -1; });
      packed = packer.n_exc[i] >= 0;
      n_exc = packed ? (uint64_t)packer.n_exc[i] : 0;
    }
    if (packed) {
      CU(cudaMemcpyAsync(w.packed.as<uint8_t>() + pk, ix->h_pack + pk, pb, cudaMemcpyHostToDevice, ix->h2d));
      if (n_exc)
        CU(cudaMemcpyAsync(w.exc.as<uint64_t>() + ek, ix->h_exc + ek, n_exc * 8, cudaMemcpyHostToDevice, ix->h2d));
    } else if (b1 > b0) {
      CU(cudaMemcpyAsync(w.bases.as<uint8_t>() + b0, batch->bases + b0, b1 - b0, cudaMemcpyHostToDevice, ix->h2d));
    }
    CU(cudaEventRecord(ix->ev_in[i], ix->h2d));
    CU(cudaStreamWaitEvent(st, ix->ev_in[i], 0));
    if (packed) {
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
      k_unpack_bases<<<(unsigned)sms * 4, 256, 0, st>>>(w.packed.as<uint8_t>() + pk, b1 - b0, w.bases.as<uint8_t>() + b0);
      if (n_exc)
        k_unpack_exceptions<<<(unsigned)std::min<uint64_t>((n_exc + 255) / 256, (uint64_t)sms * 4), 256, 0, st>>>(
            w.exc.as<uint64_t>() + ek, n_exc, b1 - b0, w.bases.as<uint8_t>() + b0);
      CU(cudaGetLastError());
    }
    const ChainSync cs{i ? ix->ev_scan[i - 1] : nullptr, ix->ev_scan[i], ix->h_snap + i};
    rc = run_pipeline(ix, *cws[i & 1], r1 - r0, w.offs.as<uint64_t>() + r0, w.bases.as<uint8_t>(),
                      w.reads.as<mg_read_result>() + r0, w.cands.as<mg_candidate>(), out->cand_cap, st, false, chain,
                      &cs);
    if (rc) break;
    CU(cudaEventRecord(ix->ev_done[i], st));
  }
  // results back in chunk order as each chunk completes: its reads, then its candidates (whose
  // range the running total snapshot gives)
  uint64_t lo = 0;
  for (int i = 0; i < nc && rc == MG_OK; i++) {
    const uint64_t r0 = bound[i], r1 = bound[i + 1];
    CU(cudaEventSynchronize(ix->ev_scan[i]));
    const uint64_t hi = ix->h_snap[i];
    CU(cudaStreamWaitEvent(ix->d2h, ix->ev_done[i], 0));
    CU(cudaMemcpyAsync(out->reads + r0, w.reads.as<mg_read_result>() + r0, (r1 - r0) * sizeof(mg_read_result),
                       cudaMemcpyDeviceToHost, ix->d2h));
    const uint64_t a = std::min(lo, out->cand_cap), b = std::min(hi, out->cand_cap);
    if (b > a)
      CU(cudaMemcpyAsync(out->cands + a, w.cands.as<mg_candidate>() + a, (b - a) * sizeof(mg_candidate),
                         cudaMemcpyDeviceToHost, ix->d2h));
    lo = hi;
  }
  unsigned long long h[2] = {0, 0};
  CU(cudaStreamSynchronize(ix->h2d));
  CU(cudaStreamSynchronize(ix->stream));
  CU(cudaStreamSynchronize(ix->stream2));
  if (rc == MG_OK) CU(cudaMemcpy(h, chain, 16, cudaMemcpyDeviceToHost));
  CU(cudaStreamSynchronize(ix->d2h));
  if (rc) return rc;
  int err = 0;
  std::memcpy(&err, &h[1], 4);
  out->n_cands = h[0];
  if (err & (kErrArena | kErrHuge)) return kRunWhole;
  return error_status(err);
}

static int classify_host(mg_index* ix, const mg_batch* batch, mg_result* out, bool plain) {
  if (!ix || !batch || !out || (batch->n_reads && (!batch->offsets || !batch->bases || !out->reads)))
    return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  CU(cudaSetDevice(ix->device));
  const uint64_t n = batch->n_reads;
  if (n >= 0xFFFFFFF0ull) return set_error(MG_ERR_LIMIT, "too many reads in one batch");
  const uint64_t nb = n ? batch->offsets[n] : 0;
  if (n && batch->offsets[0] != 0) return set_error(MG_ERR_INVAL, "offsets[0] must be 0");
  Workspace& w = ix->ws;
  int rc = ensure_workspace(w, n, nb, true);
  if (rc) return rc;
  if (w.cands.alloc(std::max<uint64_t>(out->cand_cap, 1) * sizeof(mg_candidate)))
    return set_error(MG_ERR_OOM, "candidate buffer");
  bool chunks_overflowed = false;
  if (!plain && chunk_units(n, nb) >= 2 && shapes(ix).chunks > 1) {
    rc = classify_chunked(ix, w, batch, out);
    if (rc != kRunWhole) return rc;
    chunks_overflowed = true;
  }
  cudaStream_t st = ix->stream;
  if (n) {
    CU(cudaMemcpyAsync(w.offs.p, batch->offsets, (n + 1) * 8, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(w.bases.p, batch->bases, nb, cudaMemcpyHostToDevice, st));
  }
  rc = run_pipeline(ix, w, n, w.offs.as<uint64_t>(), w.bases.as<uint8_t>(), w.reads.as<mg_read_result>(),
                    w.cands.as<mg_candidate>(), out->cand_cap, st, plain);
  if (rc) return rc;
  Counters c;
  rc = complete_pipeline(ix, w, n, w.offs.as<uint64_t>(), w.bases.as<uint8_t>(), w.reads.as<mg_read_result>(),
                         w.cands.as<mg_candidate>(), out->cand_cap, st, plain, &c);
  const uint64_t total = c.n_cands;
  out->n_cands = total;
  if (rc) return rc;
  rc = error_status(c.err);
  if (rc) return rc;
  // a chunk's staging arena ran out: the odd chunks' workspace, sized for one chunk, gets the
  // arena the whole batch needed (no chunk needs more), so that batches like this one stay in
  // chunks from now on (a failed allocation only leaves them on this path)
  if (chunks_overflowed) ix->ws2.arena.alloc(w.arena.n);
  // the same for the oversize tier's slabs (the even chunks run on w itself)
  if (chunks_overflowed && w.hmode) ix->ws2.hmode = 1;
  if (chunks_overflowed && w.hslabs > 0 && ix->ws2.hws.n < w.hws.n) {
    Workspace& o = ix->ws2;
    if (o.hws.alloc(w.hws.n)) {
      o.hslabs = 0;
      o.hq = o.hseeds = o.he = o.hc = 0;
    } else {
      o.hslabs = w.hslabs;
      o.hq = w.hq;
      o.hseeds = w.hseeds;
      o.he = w.he;
      o.hc = w.hc;
    }
  }
  if (n) {
    CU(cudaMemcpyAsync(out->reads, w.reads.p, n * sizeof(mg_read_result), cudaMemcpyDeviceToHost, st));
    if (total) CU(cudaMemcpyAsync(out->cands, w.cands.p, total * sizeof(mg_candidate), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
  }
  return MG_OK;
}

}  // namespace mg

using namespace mg;

extern "C" {

const char* mg_last_error(void) { return g_last_error.c_str(); }

const char* mg_strerror(int code) {
  switch (code) {
    case MG_OK: return "ok";
    case MG_ERR_IO: return "I/O error";
    case MG_ERR_BADFMT: return "not a readable MirAge hashmap database";
    case MG_ERR_OOM: return "out of memory or output buffer too small";
    case MG_ERR_LIMIT: return "size outside the supported limits";
    case MG_ERR_CUDA: return "CUDA error";
    case MG_ERR_BADINPUT: return "read contains a byte without a reverse complement";
    case MG_ERR_TIMEOUT: return "device wait timed out";
    case MG_ERR_INVAL: return "invalid argument";
    case MG_ERR_BUSY: return "server busy";
    default: return "unknown error";
  }
}

int mg_open(const char* path, int k, int device, mg_index** out) {
  if (!path || !out) return set_error(MG_ERR_INVAL, "null argument");
  *out = nullptr;
  auto t0 = std::chrono::steady_clock::now();
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return set_error(MG_ERR_IO, std::string("cannot open ") + path);
  const uint64_t len = (uint64_t)f.tellg();
  f.seekg(0);
  std::vector<uint8_t> buf;
  try {
    buf.resize(len);
  } catch (...) {
    return set_error(MG_ERR_OOM, "host memory for the hashmap file");
  }
  if (!f.read((char*)buf.data(), (std::streamsize)len)) return set_error(MG_ERR_IO, std::string("read error on ") + path);
  mg_index* ix = new mg_index();
  ix->info.load_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const int rc = open_image(ix, buf.data(), len, k, device);
  if (rc) {
    mg_close(ix);
    return rc;
  }
  *out = ix;
  return MG_OK;
}

int mg_open_image(const uint8_t* image, uint64_t len, int k, int device, mg_index** out) {
  if (!image || !out) return set_error(MG_ERR_INVAL, "null argument");
  *out = nullptr;
  mg_index* ix = new mg_index();
  const int rc = open_image(ix, image, len, k, device);
  if (rc) {
    mg_close(ix);
    return rc;
  }
  *out = ix;
  return MG_OK;
}

void mg_close(mg_index* ix) {
  if (!ix) return;
  cudaSetDevice(ix->device);
  for (DevBuf* b : {&ix->dir, &ix->post, &ix->slots, &ix->bases, &ix->ref_off, &ix->ref_len, &ix->logx_bitmap,
                    &ix->logx_keys, &ix->logx_vals, &ix->log_den})
    b->release();
  ix->ws.release();
  if (ix->stream) cudaStreamDestroy(ix->stream);
  if (ix->events_made)
    for (auto& e : ix->ev) cudaEventDestroy(e);
  ix->ws2.release();
  if (ix->chunk_made) {
    cudaStreamDestroy(ix->h2d);
    cudaStreamDestroy(ix->d2h);
    cudaStreamDestroy(ix->stream2);
    for (int i = 0; i < mg_index::kMaxChunks; i++) {
      cudaEventDestroy(ix->ev_in[i]);
      cudaEventDestroy(ix->ev_done[i]);
      cudaEventDestroy(ix->ev_scan[i]);
    }
    cudaFreeHost(ix->h_snap);
  }
  delete ix->pack_pool;
  if (ix->h_pack) cudaFreeHost(ix->h_pack);
  if (ix->h_exc) cudaFreeHost(ix->h_exc);
  delete ix;
}

int mg_index_get_info(const mg_index* ix, mg_index_info* info) {
  if (!ix || !info) return set_error(MG_ERR_INVAL, "null argument");
  *info = ix->info;
  info->device_bytes = ix->device_bytes + ix->slots.n;
  info->probe_slots = ix->dix.slots != nullptr;
  return MG_OK;
}

int mg_build_image(const uint8_t* bases, const uint64_t* offsets, uint32_t n_refs, const char* const* names,
                   const int32_t* taxids, int k, int word, uint8_t** image, uint64_t* len) {
  if (!bases || !offsets || !names || !image || !len) return set_error(MG_ERR_INVAL, "null argument");
  std::vector<std::string> hdr(n_refs);
  for (uint32_t r = 0; r < n_refs; r++) hdr[r] = names[r];
  std::vector<int32_t> tax;
  if (taxids) tax.assign(taxids, taxids + n_refs);
  std::vector<uint8_t> img;
  std::string err;
  int rc = mhm_build(bases, offsets, n_refs, hdr, tax, k, word, (int)std::max(1u, std::thread::hardware_concurrency()),
                     &img, &err);
  if (rc) return set_error(rc == MHM_ERR_OOM ? MG_ERR_OOM : MG_ERR_LIMIT, err);
  uint8_t* p = (uint8_t*)std::malloc(img.size() ? img.size() : 1);
  if (!p) return set_error(MG_ERR_OOM, "image");
  std::memcpy(p, img.data(), img.size());
  *image = p;
  *len = img.size();
  return MG_OK;
}

void mg_free(void* p) { std::free(p); }

int mg_inspect_image(const uint8_t* image, uint64_t len, int k, mg_index_info* info) {
  if (!image || !info) return set_error(MG_ERR_INVAL, "null argument");
  MhmIndex h;
  std::string err;
  auto t0 = std::chrono::steady_clock::now();
  int rc = mhm_parse(image, len, k, (int)std::max(1u, std::thread::hardware_concurrency()), &h, &err);
  if (rc != MHM_OK)
    return set_error(rc == MHM_ERR_IO ? MG_ERR_IO : rc == MHM_ERR_OOM ? MG_ERR_OOM : rc == MHM_ERR_LIMIT ? MG_ERR_LIMIT : MG_ERR_BADFMT, err);
  *info = mg_index_info{};
  info->n_hashes = h.n_hash;
  info->n_postings = h.postings.size();
  info->n_refs = h.n_refs;
  info->ref_bases = h.bases.size();
  info->k = k;
  info->word = h.word;
  info->load_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return MG_OK;
}

int mg_set_probe_slots(mg_index* ix, int on) {
  if (!ix) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  if (ix->n_servers.load() > 0) return set_error(MG_ERR_BUSY, "a server is attached to the index");
  CU(cudaSetDevice(ix->device));
  CU(cudaDeviceSynchronize());  // no kernel of an earlier call still reads the table
  return set_probe_slots(ix, on != 0);
}

int mg_set_tuning(mg_index* ix, const mg_tuning* t) {
  if (!ix || !t) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  ix->tune = *t;
  return MG_OK;
}

int mg_get_tuning(const mg_index* ix, mg_tuning* t, char* cls, uint64_t cls_len) {
  if (!ix || !t) return set_error(MG_ERR_INVAL, "null argument");
  CU(cudaSetDevice(ix->device));
  const Shapes s = shapes(ix);
  *t = mg_tuning{s.dual_blocks_per_sm, s.steal_chunk, s.first_tier, s.second_blocks_per_sm,
                 s.finish_blocks_per_sm, s.long_blocks_per_sm, s.chunks, s.weighted_chunks, s.third_blocks_per_sm,
                 s.pack_bases};
  if (cls && cls_len) std::snprintf(cls, cls_len, "%s", density_class(ix->info.n_postings));
  return MG_OK;
}

int mg_set_timing(mg_index* ix, int on) {
  if (!ix) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  CU(cudaSetDevice(ix->device));
  if (on && !ix->events_made) {
    for (auto& e : ix->ev) CU(cudaEventCreate(&e));
    ix->events_made = true;
  }
  ix->timing = on != 0;
  return MG_OK;
}

int mg_last_kernel_times(mg_index* ix, float* ms) {
  if (!ix || !ms) return set_error(MG_ERR_INVAL, "null argument");
  if (!ix->timing || !ix->events_made) return set_error(MG_ERR_INVAL, "timing is off");
  static const int from[5] = {0, 2, 3, 4, 6}, to[5] = {1, 3, 4, 5, 7};
  for (int i = 0; i < 5; i++) {
    CU(cudaEventSynchronize(ix->ev[to[i]]));
    CU(cudaEventElapsedTime(&ms[i], ix->ev[from[i]], ix->ev[to[i]]));
  }
  return MG_OK;
}

int mg_last_tier_counts(mg_index* ix, uint32_t* counts7) {
  if (!ix || !counts7) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  CU(cudaSetDevice(ix->device));
  if (!ix->ws.ctr.p) return set_error(MG_ERR_INVAL, "no batched call yet");
  uint8_t h[128];
  CU(cudaStreamSynchronize(ix->stream));
  CU(cudaMemcpy(h, ix->ws.ctr.p, sizeof(h), cudaMemcpyDeviceToHost));
  // the lists' counters (run_pipeline): left by the 64-, 128- and 256-posting dual tiers, the
  // general warp tier, the two long-read sizes and the block tier
  static const int at[7] = {48, 72, 56, 24, 80, 64, 32};
  for (int i = 0; i < 7; i++) std::memcpy(&counts7[i], h + at[i], 4);
  return MG_OK;
}

__global__ void k_bucket_sizes(const uint32_t* dir, const uint32_t* h, uint32_t* out, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const uint32_t x = h[i] & 0x0FFFFFFFu;
    out[i] = dir[x + 1] - dir[x];
  }
}

// Random 32-byte-sector gathers, the access pattern of the directory and posting probes: each
// group of 8 lanes reads one whole sector (4 bytes per lane, so a warp instruction reads 4
// sectors) at a pseudo-random sector index (splitmix64 of the gather number, masked to the
// power-of-two number of sectors), through L2 only, 8 gathers in flight per group.
__global__ void __launch_bounds__(256) k_gather_sectors(const uint32_t* buf, uint64_t sec_mask, uint64_t n_gathers,
                                                        unsigned long long* sink) {
  const uint32_t sub = threadIdx.x & 7;
  const uint64_t stride = ((uint64_t)gridDim.x * blockDim.x) >> 3;
  uint32_t acc = 0;
  for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3; g < n_gathers; g += 8 * stride) {
    uint32_t v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const uint64_t gg = g + u * stride;
      uint64_t x = gg + 0x9E3779B97F4A7C15ull;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      x ^= x >> 31;
      const uint64_t s = gg < n_gathers ? (x & sec_mask) : 0;
      v[u] = __ldcg(buf + 8 * s + sub);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) acc ^= v[u];
  }
  if (acc == 0x9E3779B9u) atomicAdd(sink, 1ull);
}

int mg_gather_bandwidth(int device, uint64_t buffer_bytes, double* gbs) {
  if (!gbs || buffer_bytes < (1u << 20)) return set_error(MG_ERR_INVAL, "buffer below 1 MiB or null output");
  CU(cudaSetDevice(device));
  uint64_t n_sec = 1;
  while (n_sec * 2 <= buffer_bytes / 32) n_sec *= 2;  // the largest power of two that fits
  DevBuf buf, sink;
  if (buf.alloc(n_sec * 32) || sink.alloc(8)) return set_error(MG_ERR_OOM, "gather buffer");
  CU(cudaMemset(buf.p, 0x5A, n_sec * 32));
  CU(cudaMemset(sink.p, 0, 8));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const uint64_t n_gathers = 1ull << 26;  // 2 GiB of sectors per launch
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  float best = 0.0f;
  for (int rep = 0; rep < 4; rep++) {
    CU(cudaEventRecord(e0, 0));
    k_gather_sectors<<<(unsigned)sms * 8, 256>>>(buf.as<uint32_t>(), n_sec - 1, n_gathers, sink.as<unsigned long long>());
    CU(cudaEventRecord(e1, 0));
    CU(cudaEventSynchronize(e1));
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0 && (best == 0.0f || ms < best)) best = ms;  // the first launch is a warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(cudaGetLastError());
  *gbs = (double)n_gathers * 32.0 / (best * 1e-3) / 1e9;
  return MG_OK;
}

int mg_bucket_sizes(mg_index* ix, const uint32_t* hashes, uint32_t* counts, uint64_t n) {
  if (!ix || (n && (!hashes || !counts))) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  CU(cudaSetDevice(ix->device));
  DevBuf dh, dc;
  if (dh.alloc(n * 4 + 4) || dc.alloc(n * 4 + 4)) return set_error(MG_ERR_OOM, "bucket size buffers");
  cudaStream_t st = ix->stream;
  if (n) {
    CU(cudaMemcpyAsync(dh.p, hashes, n * 4, cudaMemcpyHostToDevice, st));
    k_bucket_sizes<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ix->dix.dir, dh.as<uint32_t>(), dc.as<uint32_t>(), n);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(counts, dc.p, n * 4, cudaMemcpyDeviceToHost, st));
  }
  CU(cudaStreamSynchronize(st));
  return MG_OK;
}

int mg_eval_logf(mg_index* ix, const float* x, float* out, uint64_t n) {
  if (!ix || (n && (!x || !out))) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  CU(cudaSetDevice(ix->device));
  DevBuf dx, dout, derr;
  if (dx.alloc(n * 4 + 4) || dout.alloc(n * 4 + 4) || derr.alloc(4)) return set_error(MG_ERR_OOM, "logf buffers");
  cudaStream_t st = ix->stream;
  CU(cudaMemsetAsync(derr.p, 0, 4, st));
  if (n) {
    CU(cudaMemcpyAsync(dx.p, x, n * 4, cudaMemcpyHostToDevice, st));
    k_eval_logf<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ix->dix, dx.as<float>(), dout.as<float>(), n, derr.as<int>());
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, dout.p, n * 4, cudaMemcpyDeviceToHost, st));
  }
  int err = 0;
  CU(cudaMemcpyAsync(&err, derr.p, 4, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if (err & kErrLogRange) return set_error(MG_ERR_LIMIT, "input outside [1, 2^20)");
  return MG_OK;
}

int mg_score_batch(mg_index* ix, const mg_batch* batch, mg_result* out) { return classify_host(ix, batch, out, true); }

int mg_classify(mg_index* ix, const mg_batch* batch, mg_result* out) { return classify_host(ix, batch, out, false); }

int mg_classify_device(mg_index* ix, uint64_t n, const uint64_t* d_offs, const uint8_t* d_bases,
                       mg_read_result* d_reads, mg_candidate* d_cands, uint64_t cand_cap, uint64_t* d_n_cands,
                       void* stream) {
  if (!ix || (n && (!d_offs || !d_bases || !d_reads))) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  CU(cudaSetDevice(ix->device));
  Workspace& w = ix->ws;
  int rc = ensure_workspace(w, n, 0, false);
  if (rc) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : ix->stream;
  rc = run_pipeline(ix, w, n, d_offs, d_bases, d_reads, d_cands, cand_cap, st, false);
  if (rc) return rc;
  if (d_n_cands) CU(cudaMemcpyAsync(d_n_cands, w.ctr.as<uint8_t>() + 40, 8, cudaMemcpyDeviceToDevice, st));
  ix->last.n = n;
  ix->last.cap = cand_cap;
  ix->last.offs = d_offs;
  ix->last.bases = d_bases;
  ix->last.reads = d_reads;
  ix->last.cands = d_cands;
  ix->last.d_n_cands = d_n_cands;
  return MG_OK;
}

int mg_classify_device_sync(mg_index* ix, void* stream, uint64_t* n_cands) {
  if (!ix || !n_cands) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : ix->stream;
  Counters c;
  const auto& a = ix->last;
  int rc = complete_pipeline(ix, ix->ws, a.n, a.offs, a.bases, a.reads, a.cands, a.cap, st, false, &c);
  *n_cands = c.n_cands;
  return rc ? rc : error_status(c.err);
}

int mg_score_candidates(mg_index* ix, uint64_t n_strands, const uint64_t* q_off, const uint8_t* bases,
                        const uint64_t* c_off, const uint32_t* cand_ref, const uint64_t* r_off, const uint32_t* runs,
                        float* score, float* pct, float* rel, float* highest) {
  if (!ix || !q_off || !c_off) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(ix->mu);
  CU(cudaSetDevice(ix->device));
  const uint64_t nc = c_off[n_strands];
  const uint64_t nr = nc ? r_off[nc] : 0;
  const uint64_t nb = q_off[n_strands];
  uint32_t maxL = 0;
  for (uint64_t s = 0; s < n_strands; s++) maxL = std::max<uint32_t>(maxL, (uint32_t)(q_off[s + 1] - q_off[s]));
  for (uint64_t c = 0; c < nc; c++)
    if (cand_ref[c] >= ix->dix.n_refs) return set_error(MG_ERR_INVAL, "candidate reference out of range");
  std::vector<uint64_t> cs(nc);
  for (uint64_t s = 0; s < n_strands; s++)
    for (uint64_t c = c_off[s]; c < c_off[s + 1]; c++) cs[c] = s;
  // a run the kernel walks (Start.Query <= Last.Query) must lie inside its query and reference:
  // its coverage ends at Last.Query + tail <= L and its head walk starts at Start.Reference
  for (uint64_t c = 0; c < nc; c++) {
    const uint64_t L = q_off[cs[c] + 1] - q_off[cs[c]];
    const uint32_t rlen = ix->host.ref_len[cand_ref[c]];
    for (uint64_t r = r_off[c]; r < r_off[c + 1]; r++) {
      const uint32_t sref = runs[4 * r], sq = runs[4 * r + 1], lq = runs[4 * r + 3];
      if (sq <= lq && (lq > L || sref >= rlen))
        return set_error(MG_ERR_INVAL, "a candidate run lies outside its reference or query");
    }
  }
  const uint64_t hw = (maxL + 31) / 32 + 1;
  DevBuf dq, db, dr, drun, dcs, dro, dsc, dpc, drl, dhit, derr;
  if (dq.alloc((n_strands + 1) * 8) || db.alloc(nb + 16) || dr.alloc(nc * 4 + 4) || drun.alloc(nr * 16 + 16) ||
      dcs.alloc(nc * 8 + 8) || dro.alloc((nc + 1) * 8) || dsc.alloc(nc * 4 + 4) || dpc.alloc(nc * 4 + 4) ||
      drl.alloc(nc * 4 + 4) || dhit.alloc(nc * hw * 4 + 4) || derr.alloc(4))
    return set_error(MG_ERR_OOM, "scoring buffers");
  cudaStream_t st = ix->stream;
  CU(cudaMemcpyAsync(dq.p, q_off, (n_strands + 1) * 8, cudaMemcpyHostToDevice, st));
  if (nb) CU(cudaMemcpyAsync(db.p, bases, nb, cudaMemcpyHostToDevice, st));
  if (nc) {
    CU(cudaMemcpyAsync(dr.p, cand_ref, nc * 4, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(dcs.p, cs.data(), nc * 8, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(dro.p, r_off, (nc + 1) * 8, cudaMemcpyHostToDevice, st));
  }
  if (nr) CU(cudaMemcpyAsync(drun.p, runs, nr * 16, cudaMemcpyHostToDevice, st));
  CU(cudaMemsetAsync(derr.p, 0, 4, st));
  if (nc)
    k_score_candidates<<<(unsigned)((nc + 127) / 128), 128, 0, st>>>(
        ix->dix, n_strands, dq.as<uint64_t>(), db.as<uint8_t>(), nullptr, dr.as<uint32_t>(), dro.as<uint64_t>(),
        drun.as<uint32_t>(), nc, dcs.as<uint64_t>(), dsc.as<float>(), dpc.as<float>(), drl.as<float>(),
        dhit.as<uint32_t>(), hw, derr.as<int>());
  CU(cudaGetLastError());
  int err = 0;
  CU(cudaMemcpyAsync(&err, derr.p, 4, cudaMemcpyDeviceToHost, st));
  if (nc) {
    CU(cudaMemcpyAsync(score, dsc.p, nc * 4, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(pct, dpc.p, nc * 4, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(rel, drl.p, nc * 4, cudaMemcpyDeviceToHost, st));
  }
  CU(cudaStreamSynchronize(st));
  for (uint64_t s = 0; s < n_strands; s++) {
    float h = -1.0f;
    for (uint64_t c = c_off[s]; c < c_off[s + 1]; c++)
      if (score[c] > -1 && rel[c] > h) h = rel[c];
    highest[s] = h;
  }
  if (err & kErrLogRange) return set_error(MG_ERR_LIMIT, "relative-score logarithm outside its exact domain");
  return MG_OK;
}

}  // extern "C"
