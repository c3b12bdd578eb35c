// Index build on the device: the .mhm image of a reference set, byte-identical to the host
// builder (mhm_build) and so to the reference's own builder (BuildHashmapTable /
// TBuildHashmapForReference / SaveHashmapTableV3, Hashmap.cpp:967-1292, 2771-2976, 1701-2533).
//
//   1. every window of every reference: key = hash << 32 | position, value = refID, in
//      (reference, position) order; the first window that hashes like an all-N window ends its
//      reference (the writer's pointer stops there, Hashmap.cpp:2887-2895)
//   2. one stable radix sort of the keys: (hash, position, refID) order, the host builder's
//   3. buckets = runs of equal hash; per bucket the byte widths and record size of the writer
//      (Hashmap.cpp:1619-1697); with k < 20 the fragmented-database rule drops large buckets
//   4. record offsets by scan; bucket TOC entries and records encoded on the device
//   5. the host writes the header, reference TOCs and sequence block (mhm_write_head) and copies
//      the TOC and records in
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mg_device.cuh"
#include "mg_internal.h"
#include "mhm.h"

namespace mg {
namespace {

constexpr unsigned long long kCutKey = 1ull << 60;  // above every (hash << 32 | position)
constexpr int kSortBits = 61;

__device__ __forceinline__ int width_dev(unsigned long long v) {
  const int bits = v ? 64 - __clzll((long long)v) : 0;
  return ((bits - 1) / 8) + 1;
}
__device__ __forceinline__ void wr_dev(uint8_t* p, unsigned long long v, int w) {
  for (int i = 0; i < w; i++) p[i] = (uint8_t)(v >> (8 * i));
}

__global__ void k_build_hash(const uint8_t* bases, const uint64_t* roff, const uint64_t* wfirst, uint32_t n_refs,
                             int hlen, uint32_t h_nnn, uint64_t nwin, unsigned long long* keys, uint32_t* vals,
                             uint32_t* cut) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwin; w += stride) {
    uint32_t lo = 0, hi = n_refs - 1;  // last r with wfirst[r] <= w
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) / 2;
      if (wfirst[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t i = (uint32_t)(w - wfirst[lo]);
    const uint32_t h = hash28_dev(bases + roff[lo] + i, hlen);
    keys[w] = ((unsigned long long)h << 32) | i;
    vals[w] = lo;
    if (h == h_nnn) atomicMin(cut + lo, i);
  }
}

__global__ void k_build_cut(unsigned long long* keys, const uint32_t* vals, const uint32_t* cut, uint64_t nwin) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwin; w += stride)
    if ((uint32_t)keys[w] >= cut[vals[w]]) keys[w] = kCutKey;
}

__global__ void k_build_heads(const unsigned long long* keys, uint64_t m, uint32_t* head) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    head[i] = (i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32)) ? 1u : 0u;
}

__global__ void k_build_starts(const uint32_t* head, const uint32_t* gid, uint64_t m, uint32_t* gstart) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    if (head[i]) gstart[gid[i]] = (uint32_t)i;
}

// Per bucket: entry count, record size (0 for a dropped bucket), kept flag; error bit when a
// repeat count does not fit its width; the size histogram (clipped at 20) for the k < 20 rule.
__global__ void k_build_sizes(const unsigned long long* keys, const uint32_t* vals, const uint32_t* gstart,
                              uint32_t ng, uint32_t keep_max, unsigned long long* rec_size, uint32_t* keep,
                              unsigned* max_group, unsigned long long* hist21, int* err) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += stride) {
    const uint32_t s = gstart[g], e = gstart[g + 1], n = e - s;
    if (hist21) atomicAdd(hist21 + (n < 20 ? n : 20), 1ull);
    const bool kept = n <= keep_max;
    keep[g] = kept ? 1u : 0u;
    if (!kept) {
      rec_size[g] = 0;
      continue;
    }
    uint32_t idmin = 0xFFFFFFFFu, idmax = 0;
    unsigned long long nrep = 1;
    for (uint32_t i = s; i < e; i++) {
      const uint32_t id = vals[i];
      idmin = id < idmin ? id : idmin;
      idmax = id > idmax ? id : idmax;
      if (i > s && (uint32_t)keys[i] != (uint32_t)keys[i - 1]) nrep++;
    }
    const uint32_t pmin = (uint32_t)keys[s], pmax = (uint32_t)keys[e - 1];
    const int wid = width_dev(idmax - idmin), wpos = width_dev(pmax - pmin);
    const int wo = width_dev(idmin > pmin ? idmin : pmin), wnum = width_dev(n), wrep = width_dev(n);
    if (wpos < 8 && nrep > ((1ull << (8 * wpos)) - 1ull)) atomicOr(err, 1);
    rec_size[g] = 4ull + 2ull * wo + wnum + (unsigned long long)wid * n + 1 + wpos + nrep * (unsigned long long)(wrep + wpos);
    atomicMax(max_group, n);
  }
}

// The TOC entry (hash, record stream position) and the record of every kept bucket.
__global__ void k_build_encode(const unsigned long long* keys, const uint32_t* vals, const uint32_t* gstart,
                               const uint32_t* keep, const uint32_t* kidx, const unsigned long long* rec_off,
                               uint32_t ng, int W, unsigned long long first_rec, uint8_t* toc, uint8_t* rec) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += stride) {
    if (!keep[g]) continue;
    const uint32_t s = gstart[g], e = gstart[g + 1], n = e - s;
    const uint32_t t = kidx[g];
    wr_dev(toc + (uint64_t)t * 2 * W, keys[s] >> 32, W);
    wr_dev(toc + (uint64_t)t * 2 * W + W, first_rec + rec_off[g], W);
    uint32_t idmin = 0xFFFFFFFFu, idmax = 0;
    unsigned long long nrep = 1;
    for (uint32_t i = s; i < e; i++) {
      const uint32_t id = vals[i];
      idmin = id < idmin ? id : idmin;
      idmax = id > idmax ? id : idmax;
      if (i > s && (uint32_t)keys[i] != (uint32_t)keys[i - 1]) nrep++;
    }
    const uint32_t pmin = (uint32_t)keys[s], pmax = (uint32_t)keys[e - 1];
    const int wid = width_dev(idmax - idmin), wpos = width_dev(pmax - pmin);
    const int wo = width_dev(idmin > pmin ? idmin : pmin), wnum = width_dev(n), wrep = width_dev(n);
    uint8_t* p = rec + rec_off[g];
    p[0] = (uint8_t)wo;
    p[1] = (uint8_t)wid;
    p[2] = (uint8_t)wpos;
    p[3] = (uint8_t)wnum;
    p += 4;
    wr_dev(p, idmin, wo);
    wr_dev(p + wo, pmin, wo);
    wr_dev(p + 2 * wo, n, wnum);
    p += 2 * wo + wnum;
    for (uint32_t i = s; i < e; i++) {
      wr_dev(p, vals[i] - idmin, wid);
      p += wid;
    }
    *p++ = (uint8_t)wrep;
    wr_dev(p, nrep, wpos);
    p += wpos;
    uint32_t i0 = s;
    for (uint32_t i = s + 1; i <= e; i++) {
      if (i == e || (uint32_t)keys[i] != (uint32_t)keys[i - 1]) {
        wr_dev(p, i - i0, wrep);
        wr_dev(p + wrep, (uint32_t)keys[i0] - pmin, wpos);
        p += wrep + wpos;
        i0 = i;
      }
    }
  }
}

struct Fail {
  int code;
};

}  // namespace
}  // namespace mg

using namespace mg;

#define BCU(x)                                                                             \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) return set_error(MG_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

extern "C" int mg_build_image_device(int device, const uint8_t* bases, const uint64_t* offsets, uint32_t n_refs,
                                     const char* const* names, const int32_t* taxids, int k, int word,
                                     uint8_t** image, uint64_t* len) {
  if (!bases || !offsets || !names || !image || !len || n_refs == 0) return set_error(MG_ERR_INVAL, "null argument");
  if (k < 2) return set_error(MG_ERR_LIMIT, "k too small");
  const uint32_t step = (uint32_t)k / 2;
  const int hlen = k - (int)step + 1;  // Hashmap.cpp:2790
  std::vector<std::string> hdr(n_refs);
  for (uint32_t r = 0; r < n_refs; r++) hdr[r] = names[r];
  std::vector<int32_t> tax;
  if (taxids) tax.assign(taxids, taxids + n_refs);
  std::vector<uint64_t> roff(n_refs + 1), wfirst(n_refs + 1, 0);
  for (uint32_t r = 0; r < n_refs; r++) {
    const uint64_t l = offsets[r + 1] - offsets[r];
    if (l <= (uint64_t)hlen) return set_error(MG_ERR_LIMIT, "reference shorter than the hash window");
    if (l > 0xFFFFFFFFull) return set_error(MG_ERR_LIMIT, "reference longer than 2^32");
    roff[r] = offsets[r] - offsets[0];
    wfirst[r + 1] = wfirst[r] + (l - hlen);
  }
  roff[n_refs] = offsets[n_refs] - offsets[0];
  const uint64_t nwin = wfirst[n_refs];
  if (nwin >= 0xFFFFFFFFull) return set_error(MG_ERR_LIMIT, "more than 2^32 indexed positions");
  const std::string nn(hlen, 'N');
  const uint32_t h_nnn = hash28((const uint8_t*)nn.data(), hlen);
  BCU(cudaSetDevice(device));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const unsigned grid = (unsigned)sms * 8;
  cudaStream_t st = 0;
  // 1. windows
  DevBuf d_bases, d_roff, d_wfirst, d_cut, keys, vals, keys2, vals2, tmp;
  if (d_bases.alloc(roff[n_refs] + 64) || d_roff.alloc((n_refs + 1) * 8) || d_wfirst.alloc((n_refs + 1) * 8) ||
      d_cut.alloc(n_refs * 4) || keys.alloc(nwin * 8 + 8) || vals.alloc(nwin * 4 + 4) || keys2.alloc(nwin * 8 + 8) ||
      vals2.alloc(nwin * 4 + 4))
    return set_error(MG_ERR_OOM, "device memory for the index build");
  BCU(cudaMemcpy(d_bases.p, bases + offsets[0], roff[n_refs], cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(d_roff.p, roff.data(), (n_refs + 1) * 8, cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(d_wfirst.p, wfirst.data(), (n_refs + 1) * 8, cudaMemcpyHostToDevice));
  BCU(cudaMemset(d_cut.p, 0xFF, n_refs * 4));
  k_build_hash<<<grid, 256, 0, st>>>(d_bases.as<uint8_t>(), d_roff.as<uint64_t>(), d_wfirst.as<uint64_t>(), n_refs,
                                     hlen, h_nnn, nwin, keys.as<unsigned long long>(), vals.as<uint32_t>(),
                                     d_cut.as<uint32_t>());
  BCU(cudaGetLastError());
  k_build_cut<<<grid, 256, 0, st>>>(keys.as<unsigned long long>(), vals.as<uint32_t>(), d_cut.as<uint32_t>(), nwin);
  BCU(cudaGetLastError());
  std::vector<uint32_t> cut(n_refs);
  BCU(cudaMemcpy(cut.data(), d_cut.p, n_refs * 4, cudaMemcpyDeviceToHost));
  uint64_t m = 0;
  for (uint32_t r = 0; r < n_refs; r++) m += std::min<uint64_t>(cut[r], wfirst[r + 1] - wfirst[r]);
  d_bases.release();
  // 2. stable sort by (hash, position); refID order kept among equal keys
  size_t tmp_bytes = 0;
  BCU(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.as<unsigned long long>(),
                                      keys2.as<unsigned long long>(), vals.as<uint32_t>(), vals2.as<uint32_t>(),
                                      (int64_t)nwin, 0, kSortBits, st));
  if (tmp.alloc(tmp_bytes + 16)) return set_error(MG_ERR_OOM, "device memory for the index sort");
  BCU(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys.as<unsigned long long>(), keys2.as<unsigned long long>(),
                                      vals.as<uint32_t>(), vals2.as<uint32_t>(), (int64_t)nwin, 0, kSortBits, st));
  keys.release();
  vals.release();
  tmp.release();
  const unsigned long long* sk = keys2.as<unsigned long long>();
  const uint32_t* sv = vals2.as<uint32_t>();
  // 3. buckets
  DevBuf head, gid;
  if (head.alloc(m * 4 + 4) || gid.alloc(m * 4 + 4)) return set_error(MG_ERR_OOM, "device memory for the buckets");
  uint32_t ng = 0;
  if (m) {
    k_build_heads<<<grid, 256, 0, st>>>(sk, m, head.as<uint32_t>());
    BCU(cudaGetLastError());
    BCU(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, head.as<uint32_t>(), gid.as<uint32_t>(), (int64_t)m, st));
    if (tmp.alloc(tmp_bytes + 16)) return set_error(MG_ERR_OOM, "device memory for the bucket scan");
    BCU(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, head.as<uint32_t>(), gid.as<uint32_t>(), (int64_t)m, st));
    uint32_t last_gid, last_head;
    BCU(cudaMemcpy(&last_gid, gid.as<uint32_t>() + m - 1, 4, cudaMemcpyDeviceToHost));
    BCU(cudaMemcpy(&last_head, head.as<uint32_t>() + m - 1, 4, cudaMemcpyDeviceToHost));
    ng = last_gid + last_head;
  }
  DevBuf gstart, rsz, keep, kidx, roffs, misc;
  if (gstart.alloc((uint64_t)(ng + 1) * 4) || rsz.alloc((uint64_t)ng * 8 + 8) || keep.alloc((uint64_t)ng * 4 + 4) ||
      kidx.alloc((uint64_t)ng * 4 + 4) || roffs.alloc((uint64_t)ng * 8 + 8) || misc.alloc(256))
    return set_error(MG_ERR_OOM, "device memory for the buckets");
  const uint32_t m32 = (uint32_t)m;
  BCU(cudaMemcpy(gstart.as<uint32_t>() + ng, &m32, 4, cudaMemcpyHostToDevice));
  if (m) {
    k_build_starts<<<grid, 256, 0, st>>>(head.as<uint32_t>(), gid.as<uint32_t>(), m, gstart.as<uint32_t>());
    BCU(cudaGetLastError());
  }
  head.release();
  gid.release();
  // misc: 0 max_group (u32) | 8 err (int) | 16 hist21 (21 x u64)
  unsigned* d_maxg = (unsigned*)misc.p;
  int* d_err = (int*)(misc.as<uint8_t>() + 8);
  unsigned long long* d_hist = (unsigned long long*)(misc.as<uint8_t>() + 16);
  uint32_t keep_max = 0xFFFFFFFFu;
  if (k < 20 && ng) {
    // EnableFragmentedDatabase (Hashmap.cpp:1759-1840): drop the buckets larger than
    // min(20, the 30th-percentile bucket size)
    BCU(cudaMemset(misc.p, 0, 256));
    k_build_sizes<<<grid, 256, 0, st>>>(sk, sv, gstart.as<uint32_t>(), ng, 0xFFFFFFFFu, rsz.as<unsigned long long>(),
                                        keep.as<uint32_t>(), d_maxg, d_hist, d_err);
    BCU(cudaGetLastError());
    unsigned long long hist[21];
    BCU(cudaMemcpy(hist, d_hist, sizeof(hist), cudaMemcpyDeviceToHost));
    const uint64_t idx = (uint64_t)(((double)ng / 100.0) * 30);
    uint64_t below = 0;
    keep_max = 20;
    for (uint32_t v = 0; v < 20; v++) {
      below += hist[v];
      if (below > idx) {
        keep_max = v;
        break;
      }
    }
  }
  BCU(cudaMemset(misc.p, 0, 256));
  if (ng) {
    k_build_sizes<<<grid, 256, 0, st>>>(sk, sv, gstart.as<uint32_t>(), ng, keep_max, rsz.as<unsigned long long>(),
                                        keep.as<uint32_t>(), d_maxg, nullptr, d_err);
    BCU(cudaGetLastError());
  }
  int err = 0;
  unsigned max_group = 0;
  BCU(cudaMemcpy(&err, d_err, 4, cudaMemcpyDeviceToHost));
  BCU(cudaMemcpy(&max_group, d_maxg, 4, cudaMemcpyDeviceToHost));
  if (err) return set_error(MG_ERR_LIMIT, "a bucket has more distinct positions than its width can count");
  // 4. record offsets and kept-bucket TOC slots
  uint64_t rec_total = 0, last_rec = 0;
  uint32_t n_kept = 0;
  if (ng) {
    BCU(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, rsz.as<unsigned long long>(),
                                      roffs.as<unsigned long long>(), (int64_t)ng, st));
    size_t tb2 = 0;
    BCU(cub::DeviceScan::ExclusiveSum(nullptr, tb2, keep.as<uint32_t>(), kidx.as<uint32_t>(), (int64_t)ng, st));
    if (tmp.alloc(std::max(tmp_bytes, tb2) + 16)) return set_error(MG_ERR_OOM, "device memory for the record scan");
    BCU(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, rsz.as<unsigned long long>(), roffs.as<unsigned long long>(),
                                      (int64_t)ng, st));
    BCU(cub::DeviceScan::ExclusiveSum(tmp.p, tb2, keep.as<uint32_t>(), kidx.as<uint32_t>(), (int64_t)ng, st));
    unsigned long long lo, ls;
    uint32_t lk, lki;
    BCU(cudaMemcpy(&lo, roffs.as<unsigned long long>() + ng - 1, 8, cudaMemcpyDeviceToHost));
    BCU(cudaMemcpy(&ls, rsz.as<unsigned long long>() + ng - 1, 8, cudaMemcpyDeviceToHost));
    BCU(cudaMemcpy(&lk, keep.as<uint32_t>() + ng - 1, 4, cudaMemcpyDeviceToHost));
    BCU(cudaMemcpy(&lki, kidx.as<uint32_t>() + ng - 1, 4, cudaMemcpyDeviceToHost));
    rec_total = lo + ls;
    n_kept = lki + lk;
    // the size of the last kept bucket's record (the 32-bit limit excludes it)
    if (n_kept) {
      std::vector<unsigned long long> tail;
      uint64_t at = ng;
      const uint64_t chunk = 4096;
      while (at > 0 && !last_rec) {
        const uint64_t from = at > chunk ? at - chunk : 0;
        tail.resize(at - from);
        BCU(cudaMemcpy(tail.data(), rsz.as<unsigned long long>() + from, (at - from) * 8, cudaMemcpyDeviceToHost));
        for (uint64_t i = at - from; i-- > 0;)
          if (tail[i]) {
            last_rec = tail[i];
            break;
          }
        at = from;
      }
    }
  }
  MhmPlan plan;
  std::string perr;
  int rc = mhm_plan(offsets, n_refs, hdr, word, n_kept, rec_total, last_rec, &plan, &perr);
  if (rc) return set_error(rc == MHM_ERR_OOM ? MG_ERR_OOM : MG_ERR_LIMIT, perr);
  // 5. records and TOC on the device, the rest on the host
  DevBuf d_toc, d_rec;
  if (d_toc.alloc((uint64_t)n_kept * 2 * plan.W + 16) || d_rec.alloc(rec_total + 16))
    return set_error(MG_ERR_OOM, "device memory for the records");
  if (ng) {
    k_build_encode<<<grid, 256, 0, st>>>(sk, sv, gstart.as<uint32_t>(), keep.as<uint32_t>(), kidx.as<uint32_t>(),
                                         roffs.as<unsigned long long>(), ng, (int)plan.W, plan.first_rec,
                                         d_toc.as<uint8_t>(), d_rec.as<uint8_t>());
    BCU(cudaGetLastError());
  }
  uint8_t* img = (uint8_t*)std::malloc(plan.total ? plan.total : 1);
  if (!img) return set_error(MG_ERR_OOM, "host memory for the image");
  rc = mhm_write_head(img, plan, bases, offsets, n_refs, hdr, tax, k, n_kept, max_group, &perr);
  cudaError_t e = cudaSuccess;
  if (!rc && n_kept) e = cudaMemcpy(img + plan.toc_at, d_toc.p, (uint64_t)n_kept * 2 * plan.W, cudaMemcpyDeviceToHost);
  if (!rc && e == cudaSuccess && rec_total) e = cudaMemcpy(img + plan.first_rec, d_rec.p, rec_total, cudaMemcpyDeviceToHost);
  if (rc || e != cudaSuccess) {
    std::free(img);
    return rc ? set_error(MG_ERR_LIMIT, perr) : set_error(MG_ERR_CUDA, cudaGetErrorString(e));
  }
  *image = img;
  *len = plan.total;
  return MG_OK;
}
