// Candidate scoring for callers that cannot allocate device memory.
//
// Some callers may not call cudaMalloc or cudaFree: a host whose device memory is already
// reserved by another allocator (a framework's caching allocator or a pool sized at start-up,
// where a stray cudaMalloc fails or breaks the budget), or a latency-bound path where the
// device-wide synchronisation of cudaFree would stall other streams. mg_score_candidates_noalloc
// serves them: inputs and outputs are the caller's device buffers, and the only working memory
// is the fixed array below, which the library holds on every GPU that loads it until exit.
//
// Its kernel is a variant of k_score_candidates (mg_lib.cu) with a fixed grid: each thread owns
// one slot of the array for its coverage bitmap and strides over the candidates, so the array's
// size bounds the query length (kNaMaxLen bases) and not the number of candidates.
#include <cuda_runtime.h>

#include <mutex>

#include "mg_internal.h"
#include "mg_kernels.cuh"

namespace mg {
namespace {

constexpr int kNaBlocks = 148;                   // one block per SM of a B200
constexpr int kNaThreads = 128;
constexpr uint32_t kNaMaxLen = 2048;             // longest query strand, in bases
constexpr uint32_t kNaWords = kNaMaxLen / 32;    // coverage bitmap words per thread
constexpr size_t kNaHeaderWords = 64;            // 256 bytes; word 0 holds the error bits
constexpr size_t kNaScratchWords = kNaHeaderWords + (size_t)kNaBlocks * kNaThreads * kNaWords;
constexpr int kNaMaxDevices = 64;

}  // namespace
}  // namespace mg

// The working memory of every call on a device (4,849,920 bytes). Host code sees only a
// host-side stand-in under this name; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) uint32_t mg_noalloc_scratch[mg::kNaScratchWords];

namespace mg {
namespace {

// Score, percentageMatch and relative score of every candidate (MatrixCPU.cpp:57-176 and
// MatrixResult.cpp:60-79, as k_score_candidates). Runs that would read outside their query or
// reference set kErrBadInput and are skipped; a query longer than kNaMaxLen sets kErrLimit.
__global__ void __launch_bounds__(kNaThreads)
    k_score_candidates_static(DevIndex ix, uint64_t n_strands, const uint64_t* q_off, const uint8_t* bases,
                              const uint64_t* c_off, const uint32_t* cand_ref, const uint64_t* r_off,
                              const uint32_t* runs, float* score_out, float* pct_out, float* rel_out,
                              uint32_t* scratch) {
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t* hit = scratch + kNaHeaderWords + gtid * kNaWords;
  const uint64_t nc = c_off[n_strands];
  const uint32_t k = (uint32_t)ix.k;
  int err = 0;
  for (uint64_t c = gtid; c < nc; c += stride) {
    uint64_t lo = 0, hi = n_strands - 1;  // the strand of c: last s with c_off[s] <= c
    while (lo < hi) {
      const uint64_t mid = (lo + hi + 1) / 2;
      if (c_off[mid] <= c) lo = mid;
      else hi = mid - 1;
    }
    const uint64_t Lq = q_off[lo + 1] - q_off[lo];
    const uint32_t ref = cand_ref[c];
    float score = -2.0f, pct = 0.0f, rel = -1.0f;
    if (ref >= ix.n_refs) {
      err |= kErrBadInput;
    } else if (Lq > kNaMaxLen) {
      err |= kErrLimit;
    } else {
      const uint32_t L = (uint32_t)Lq;
      const uint8_t* q = bases + q_off[lo];
      const uint8_t* rs = ix.bases + ix.ref_off[ref];
      const uint32_t rlen = ix.ref_len[ref];
      const uint32_t nw = (L + 31) / 32;
      for (uint32_t w = 0; w < nw; w++) hit[w] = 0;
      uint64_t sc = 0, sr = 0;
      for (uint64_t r = r_off[c]; r < r_off[c + 1]; r++) {
        const uint32_t sref = runs[4 * r], sq = runs[4 * r + 1], lref = runs[4 * r + 2], lq = runs[4 * r + 3];
        if (sq > lq) continue;
        if (lq > L || sref >= rlen) {
          err |= kErrBadInput;
          continue;
        }
        const uint32_t tail = tail_walk(q, rs, L, rlen, lq, lref, k);
        const uint32_t head = head_walk(q, rs, sq, sref, k);
        const uint64_t tot = (uint64_t)tail + head + (lq - sq);
        if (tot >= k) {
          sc += tot;
          sr += tot * (tot + 1) / 2;
          for (uint64_t p = sq - head; p < sq - head + tot; p++) hit[p >> 5] |= 1u << (p & 31);
        }
      }
      if (sc > 0) {
        uint32_t hits = 0;
        for (uint32_t w = 0; w < nw; w++) hits += __popc(hit[w]);
        final_score(sr, sc, hits, L, &score, &pct);
        rel = relative_score(ix, __uint2float_rn(L), __uint2float_rn(rlen), score, &err);
      }
    }
    score_out[c] = score;
    pct_out[c] = pct;
    rel_out[c] = rel;
  }
  if (err) atomicOr((int*)scratch, err);
}

// HighestScore per strand: the largest relative score among its scored candidates, -1 when it
// has none (MatrixCPU.cpp:323-370).
__global__ void k_strand_highest(uint64_t n_strands, const uint64_t* c_off, const float* score, const float* rel,
                                 float* highest) {
  const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_strands) return;
  float h = -1.0f;
  for (uint64_t c = c_off[s]; c < c_off[s + 1]; c++)
    if (score[c] > -1.0f && rel[c] > h) h = rel[c];
  highest[s] = h;
}

std::mutex g_na_mu[kNaMaxDevices];          // serialises the calls on each device (one array each)
void* g_na_addr[kNaMaxDevices] = {};        // device address of the array, per device

}  // namespace
}  // namespace mg

using namespace mg;

extern "C" int mg_score_candidates_noalloc(mg_index* ix, uint64_t n_strands, const uint64_t* d_q_off,
                                           const uint8_t* d_bases, const uint64_t* d_c_off,
                                           const uint32_t* d_cand_ref, const uint64_t* d_r_off,
                                           const uint32_t* d_runs, float* d_score, float* d_pct, float* d_rel,
                                           float* d_highest, void* stream) {
  if (!ix) return set_error(MG_ERR_INVAL, "null index");
  if (n_strands == 0) return MG_OK;
  if (!d_q_off || !d_bases || !d_c_off || !d_cand_ref || !d_r_off || !d_runs || !d_score || !d_pct || !d_rel ||
      !d_highest)
    return set_error(MG_ERR_INVAL, "null argument");
  if (n_strands >= (1ull << 40)) return set_error(MG_ERR_LIMIT, "too many query strands");
  const int dev = ix->device;
  if (dev < 0 || dev >= kNaMaxDevices) return set_error(MG_ERR_LIMIT, "device ordinal beyond the supported range");
  std::lock_guard<std::mutex> lk(g_na_mu[dev]);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return set_error(MG_ERR_CUDA, "cudaGetDevice");
  if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return set_error(MG_ERR_CUDA, "cudaSetDevice");
  int rc = MG_OK;
  int bits = 0;
  do {
    // set-up, once per device with that device current: the array's device address
    if (!g_na_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, mg_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        rc = set_error(MG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        break;
      }
      g_na_addr[dev] = p;
    }
    uint32_t* scratch = (uint32_t*)g_na_addr[dev];
    cudaStream_t st = stream ? (cudaStream_t)stream : ix->stream;
    // the error word keeps the previous call's bits; each bitmap slot is cleared by its thread
    if (cudaMemsetAsync(scratch, 0, kNaHeaderWords * 4, st) != cudaSuccess) {
      rc = set_error(MG_ERR_CUDA, "cudaMemsetAsync");
      break;
    }
    k_score_candidates_static<<<kNaBlocks, kNaThreads, 0, st>>>(ix->dix, n_strands, d_q_off, d_bases, d_c_off,
                                                                 d_cand_ref, d_r_off, d_runs, d_score, d_pct, d_rel,
                                                                 scratch);
    k_strand_highest<<<(unsigned)((n_strands + 255) / 256), 256, 0, st>>>(n_strands, d_c_off, d_score, d_rel,
                                                                          d_highest);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, scratch, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = set_error(MG_ERR_CUDA, cudaGetErrorString(e));
  } while (false);
  if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  if (rc) return rc;
  if (bits & kErrLimit) return set_error(MG_ERR_LIMIT, "a query strand is longer than 2048 bases");
  if (bits & kErrBadInput) return set_error(MG_ERR_INVAL, "a candidate reference or run lies outside its reference or query");
  if (bits & kErrLogRange) return set_error(MG_ERR_LIMIT, "relative-score logarithm outside its exact domain");
  return MG_OK;
}
