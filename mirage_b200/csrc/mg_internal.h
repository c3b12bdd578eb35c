// Host-side internals shared by the library's translation units (index, pipeline, server).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/mirage_b200.h"
#include "mg_device.cuh"
#include "mg_pack.h"
#include "mhm.h"

namespace mg {

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  int alloc(size_t bytes) {
    if (bytes <= n && p) return 0;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      cudaGetLastError();  // an allocation failure is not sticky: clear it for the next launch check
      p = nullptr;
      return -1;
    }
    n = bytes;
    return 0;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// Device buffers of one classification call in flight (a call owns one at a time).
struct Workspace {
  DevBuf offs, bases, reads, stage, arena, cands, ctr, ovf, sums, gws, chain;
  DevBuf packed, exc;  // 2-bit packed bases and their exceptions (mg_classify with pack_bases)
  // the oversize tier: off (hmode 0: the global tier marks what it cannot take) until a batch on
  // this workspace needs it; its workspace, hslabs slabs, each for a read of up to hq bases,
  // hseeds seeds and he postings per strand (a power of two) with up to hc candidates per strand,
  // grown on demand by complete_pipeline
  DevBuf hws;
  int hmode = 0;
  int hslabs = 0;
  uint32_t hq = 0, hseeds = 0, he = 0, hc = 0;
  // the stream on which the tiers after the dual tier run beside its finishing pass, and the
  // events that fork it from and join it back to the call's stream (made at first use)
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  void release() {
    for (DevBuf* b : {&offs, &bases, &reads, &stage, &arena, &cands, &ctr, &ovf, &sums, &gws, &chain, &packed, &exc,
                      &hws})
      b->release();
    hmode = hslabs = 0;
    hq = hseeds = he = hc = 0;
    if (side) cudaStreamDestroy(side);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    side = nullptr;
    fork = join = nullptr;
  }
  size_t bytes() const {
    return offs.n + bases.n + reads.n + stage.n + arena.n + cands.n + ctr.n + ovf.n + sums.n + gws.n + chain.n +
           packed.n + exc.n + hws.n;
  }
};

int set_error(int code, const std::string& msg);
// Size ws for n_reads reads (n_bases bases when host_io: the input and result buffers too).
int ensure_workspace(Workspace& ws, uint64_t n_reads, uint64_t n_bases, bool host_io);
// Queue the fused pipeline (warp, block and global tiers, then compaction) on stream st.
// chain (optional, device, 16 bytes): for one chunk of a larger batch, [0] the candidates of the
// earlier chunks (output offsets continue from there and the count is advanced), [8] the batch's
// error bits (accumulated instead of the per-call counter).
// For chunks on two streams: the scan waits for the previous chunk's (wait_prev), then the
// running total is copied to *snap (pinned host memory) and `scanned` is recorded.
struct ChainSync {
  cudaEvent_t wait_prev = nullptr;
  cudaEvent_t scanned = nullptr;
  unsigned long long* snap = nullptr;
};
int run_pipeline(mg_index* ix, Workspace& ws, uint64_t n, const uint64_t* d_offs, const uint8_t* d_bases,
                 mg_read_result* d_reads, mg_candidate* d_out, uint64_t cap, cudaStream_t st, bool plain,
                 unsigned long long* chain = nullptr, const ChainSync* cs = nullptr);
// Wait for st, read the error word and the candidate count of the call that used ws.
int finish_errors(Workspace& ws, cudaStream_t st, uint64_t* n_cands);
// The pipeline's counters after the stream drains.
struct Counters {
  uint64_t n_cands = 0;     // candidates of the batch (written when they fit the output)
  uint64_t arena_need = 0;  // staging arena entries the batch asked for
  int err = 0;              // error bits
  bool reran = false;       // the batch ran again with a larger staging arena or oversize workspace
  uint32_t huge_need[4] = {0, 0, 0, 0};  // oversize reads that did not fit: most bases, seeds,
                                         // postings per strand; how many
};
int read_counters(Workspace& ws, cudaStream_t st, Counters* c);
// Waits for a launched pipeline and, when the staging arena or the oversize tier's workspace was
// too small, grows it to what the kernels asked for and runs the batch again (same arguments as
// the launch), up to three times.
int complete_pipeline(mg_index* ix, Workspace& ws, uint64_t n, const uint64_t* d_offs, const uint8_t* d_bases,
                      mg_read_result* d_reads, mg_candidate* d_out, uint64_t cap, cudaStream_t st, bool plain,
                      Counters* c);
// Status of error bits as finish_errors reports them.
int error_status(int err_bits);

}  // namespace mg

struct mg_index {
  int device = 0;
  mg::DevIndex dix{};
  mg::MhmIndex host;  // refs, headers, taxids kept; postings released after upload
  mg::DevBuf dir, post, slots, bases, ref_off, ref_len, logx_bitmap, logx_keys, logx_vals, log_den;
  mg::Workspace ws;   // workspace of the synchronous entry points
  cudaStream_t stream = nullptr;
  // chunked batched form: copy streams and per-chunk events (made on first use)
  static constexpr int kMaxChunks = 8;
  cudaStream_t h2d = nullptr, d2h = nullptr, stream2 = nullptr;  // stream2: odd chunks
  cudaEvent_t ev_in[kMaxChunks], ev_done[kMaxChunks], ev_scan[kMaxChunks];
  unsigned long long* h_snap = nullptr;  // pinned: running candidate totals after each chunk
  mg::Workspace ws2;                     // scratch of the odd chunks
  bool chunk_made = false;
  std::mutex mu;
  std::atomic<int> n_servers{0};  // mg_server objects attached to this index
  mg_tuning tune{};               // launch shapes (mg_set_tuning); zero fields: defaults
  // 2-bit packing of the uploaded bases (mg_classify): host threads and pinned staging
  mg::PackPool* pack_pool = nullptr;
  uint8_t* h_pack = nullptr;
  uint64_t h_pack_cap = 0;
  uint64_t* h_exc = nullptr;
  uint64_t h_exc_cap = 0;
  mg_index_info info{};
  uint64_t device_bytes = 0;
  // optional per-kernel timing of the last pipeline (events on the launching stream)
  bool timing = false;
  bool events_made = false;
  cudaEvent_t ev[8];
  // arguments of the last mg_classify_device launch, for its completion in the sync call
  struct {
    uint64_t n = 0, cap = 0;
    const uint64_t* offs = nullptr;
    const uint8_t* bases = nullptr;
    mg_read_result* reads = nullptr;
    mg_candidate* cands = nullptr;
    uint64_t* d_n_cands = nullptr;
  } last;
};
