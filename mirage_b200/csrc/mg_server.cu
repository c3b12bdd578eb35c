// Served form: continuous batching of classification requests against an HBM-resident index.
//
// Requests are copied on submit and queued. A server thread forms "steps": it takes reads from
// the queued requests in arrival order (a request larger than a step spans several steps, and
// one step carries reads of many requests) and runs the fused pipeline on them. Two step slots
// each own a device workspace, pinned host staging buffers and a stream, so the next step's
// copies and kernels run while the previous step's results are drained. A request that arrives
// while steps are on the device joins the next step formed. Every read is classified
// independently, so its result is the same alone and in any mix.
//
// Admission: a request is refused with MG_ERR_BUSY (retry later) when the tracked request
// count or the bytes of queued-but-unfinished reads would pass their limits; the step size is
// fixed at creation from the device memory available.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "mg_internal.h"

namespace mg {

struct Request {
  uint64_t ticket = 0;
  uint64_t n = 0;
  std::vector<uint64_t> offs;
  std::vector<uint8_t> bases;
  uint64_t next = 0;  // next read to schedule
  uint64_t done = 0;  // reads with results
  std::vector<mg_read_result> reads;
  std::vector<mg_candidate> cands;
  int error = 0;
  bool complete = false;
};

struct Part {
  Request* req;
  uint64_t first, count;  // reads [first, first+count) of req
};

struct Slot {
  Workspace ws;
  cudaStream_t st = nullptr;
  uint64_t* h_offs = nullptr;
  uint8_t* h_bases = nullptr;
  mg_read_result* h_reads = nullptr;
  mg_candidate* h_cands = nullptr;
  uint64_t cap_reads = 0, cap_bases = 0, cap_cands = 0;
  std::vector<Part> parts;
  uint64_t n = 0;
  bool busy = false;
  int launch_rc = 0;
};

static bool has_complement(uint8_t c) {
  const uint8_t u = ((int8_t)c > 96) ? (uint8_t)(c - 32) : c;  // Sequences.cpp:43-55
  switch (u) {
    case 'A': case 'T': case 'U': case 'G': case 'C': case 'Y': case 'R': case 'S': case 'W':
    case 'K': case 'M': case 'B': case 'D': case 'H': case 'V': case 'N': case '-': case '~':
      return true;
    default:
      return false;
  }
}

}  // namespace mg

struct mg_server {
  mg_index* ix = nullptr;
  uint64_t step_reads = 0, step_bases = 0;
  uint32_t max_requests = 0;
  uint64_t queue_budget = 0;   // bytes of queued reads
  uint64_t queued_bytes = 0;
  uint64_t next_ticket = 1;
  std::deque<mg::Request*> queue;                           // requests with unscheduled reads
  std::map<uint64_t, std::unique_ptr<mg::Request>> live;    // every tracked request
  mg::Slot slot[2];
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::thread th;
};

namespace mg {

static int slot_alloc(Slot& s, uint64_t reads, uint64_t bases, uint64_t cands) {
  if (reads > s.cap_reads) {
    if (s.h_offs) cudaFreeHost(s.h_offs);
    if (s.h_reads) cudaFreeHost(s.h_reads);
    s.h_offs = nullptr;
    s.h_reads = nullptr;
    if (cudaMallocHost((void**)&s.h_offs, (reads + 1) * 8) != cudaSuccess ||
        cudaMallocHost((void**)&s.h_reads, reads * sizeof(mg_read_result)) != cudaSuccess)
      return set_error(MG_ERR_OOM, "pinned step buffers");
    s.cap_reads = reads;
  }
  if (bases > s.cap_bases) {
    if (s.h_bases) cudaFreeHost(s.h_bases);
    s.h_bases = nullptr;
    if (cudaMallocHost((void**)&s.h_bases, bases) != cudaSuccess) return set_error(MG_ERR_OOM, "pinned step buffers");
    s.cap_bases = bases;
  }
  if (cands > s.cap_cands) {
    if (s.h_cands) cudaFreeHost(s.h_cands);
    s.h_cands = nullptr;
    if (cudaMallocHost((void**)&s.h_cands, cands * sizeof(mg_candidate)) != cudaSuccess)
      return set_error(MG_ERR_OOM, "pinned step buffers");
    s.cap_cands = cands;
  }
  if (ensure_workspace(s.ws, reads, bases, true)) return MG_ERR_OOM;
  if (s.ws.cands.alloc(std::max<uint64_t>(cands, 1) * sizeof(mg_candidate))) return set_error(MG_ERR_OOM, "step candidates");
  return MG_OK;
}

static void slot_free(Slot& s) {
  if (s.st) cudaStreamDestroy(s.st);
  if (s.h_offs) cudaFreeHost(s.h_offs);
  if (s.h_bases) cudaFreeHost(s.h_bases);
  if (s.h_reads) cudaFreeHost(s.h_reads);
  if (s.h_cands) cudaFreeHost(s.h_cands);
  s.ws.release();
}

// Form a step from the queue (server lock held) and launch it on the slot's stream.
static bool form_step(mg_server* sv, Slot& s) {
  s.parts.clear();
  s.n = 0;
  uint64_t nb = 0;
  while (!sv->queue.empty() && s.n < sv->step_reads) {
    Request* r = sv->queue.front();
    uint64_t take = std::min(r->n - r->next, sv->step_reads - s.n);
    // respect the base budget, but always take at least one read
    uint64_t got = 0, b = 0;
    while (got < take) {
      uint64_t L = r->offs[r->next + got + 1] - r->offs[r->next + got];
      if (nb + b + L > sv->step_bases && (s.n + got) > 0) break;
      b += L;
      got++;
    }
    if (got == 0) break;
    s.parts.push_back(Part{r, r->next, got});
    r->next += got;
    s.n += got;
    nb += b;
    if (r->next == r->n) sv->queue.pop_front();
    if (nb >= sv->step_bases) break;
  }
  if (s.n == 0) return false;
  if (slot_alloc(s, s.n, std::max<uint64_t>(nb, sv->step_bases), std::max<uint64_t>(s.cap_cands, 16 * s.n + 1024))) {
    s.launch_rc = MG_ERR_OOM;
    s.busy = true;
    return true;
  }
  // pack the reads (offsets rebased) into the pinned staging buffers
  uint64_t at = 0, ob = 0;
  s.h_offs[0] = 0;
  for (const Part& p : s.parts) {
    const uint64_t b0 = p.req->offs[p.first], b1 = p.req->offs[p.first + p.count];
    std::memcpy(s.h_bases + ob, p.req->bases.data() + b0, b1 - b0);
    for (uint64_t i = 0; i < p.count; i++) s.h_offs[at + i + 1] = ob + (p.req->offs[p.first + i + 1] - b0);
    at += p.count;
    ob += b1 - b0;
  }
  mg_index* ix = sv->ix;
  s.launch_rc = MG_OK;
  cudaError_t e = cudaMemcpyAsync(s.ws.offs.p, s.h_offs, (s.n + 1) * 8, cudaMemcpyHostToDevice, s.st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s.ws.bases.p, s.h_bases, ob, cudaMemcpyHostToDevice, s.st);
  if (e != cudaSuccess) {
    s.launch_rc = set_error(MG_ERR_CUDA, cudaGetErrorString(e));
  } else {
    s.launch_rc = run_pipeline(ix, s.ws, s.n, s.ws.offs.as<uint64_t>(), s.ws.bases.as<uint8_t>(),
                               s.ws.reads.as<mg_read_result>(), s.ws.cands.as<mg_candidate>(), s.cap_cands, s.st, false);
    if (s.launch_rc == MG_OK &&
        cudaMemcpyAsync(s.h_reads, s.ws.reads.p, s.n * sizeof(mg_read_result), cudaMemcpyDeviceToHost, s.st) !=
            cudaSuccess)
      s.launch_rc = MG_ERR_CUDA;
  }
  s.busy = true;
  return true;
}

// Wait for a launched step and hand its results to the requests (server lock not held while
// waiting).
static void drain_step(mg_server* sv, Slot& s) {
  int rc = s.launch_rc;
  uint64_t total = 0;
  if (rc == MG_OK) rc = finish_errors(s.ws, s.st, &total);
  if (rc == MG_ERR_OOM && total > s.cap_cands) {
    // the step produced more candidates than its buffer holds: rerun it with room for all
    if (slot_alloc(s, s.n, s.cap_bases, total + 1024) == MG_OK) {
      rc = run_pipeline(sv->ix, s.ws, s.n, s.ws.offs.as<uint64_t>(), s.ws.bases.as<uint8_t>(),
                        s.ws.reads.as<mg_read_result>(), s.ws.cands.as<mg_candidate>(), s.cap_cands, s.st, false);
      if (rc == MG_OK &&
          cudaMemcpyAsync(s.h_reads, s.ws.reads.p, s.n * sizeof(mg_read_result), cudaMemcpyDeviceToHost, s.st) !=
              cudaSuccess)
        rc = MG_ERR_CUDA;
      if (rc == MG_OK) rc = finish_errors(s.ws, s.st, &total);
    }
  }
  if (rc == MG_OK && total) {
    if (cudaMemcpyAsync(s.h_cands, s.ws.cands.p, total * sizeof(mg_candidate), cudaMemcpyDeviceToHost, s.st) !=
            cudaSuccess ||
        cudaStreamSynchronize(s.st) != cudaSuccess)
      rc = MG_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  uint64_t at = 0;
  for (const Part& p : s.parts) {
    Request* r = p.req;
    if (rc != MG_OK) {
      r->error = rc;
    } else {
      for (uint64_t i = 0; i < p.count; i++) {
        mg_read_result rr = s.h_reads[at + i];
        const uint32_t nc = rr.n_fwd + rr.n_rc;
        const uint64_t dst = r->cands.size();
        r->cands.insert(r->cands.end(), s.h_cands + rr.cand_off, s.h_cands + rr.cand_off + nc);
        rr.cand_off = (uint32_t)dst;
        r->reads[p.first + i] = rr;
      }
    }
    r->done += p.count;
    at += p.count;
    if (r->done == r->n) {
      r->complete = true;
      sv->queued_bytes -= r->bases.size() + r->offs.size() * 8;
    }
  }
  s.parts.clear();
  s.busy = false;
  sv->cv_done.notify_all();
}

static void server_loop(mg_server* sv) {
  cudaSetDevice(sv->ix->device);
  int oldest = 0;
  std::unique_lock<std::mutex> lk(sv->mu);
  for (;;) {
    sv->cv_work.wait(lk, [&] { return sv->stop || !sv->queue.empty() || sv->slot[0].busy || sv->slot[1].busy; });
    if (sv->stop && !sv->slot[0].busy && !sv->slot[1].busy) break;
    // launch into every free slot while there is work (the launch is asynchronous)
    for (int i = 0; i < 2; i++) {
      Slot& s = sv->slot[(oldest + i) % 2];
      if (!s.busy && !sv->queue.empty()) form_step(sv, s);
    }
    // drain the oldest busy slot
    Slot* d = nullptr;
    for (int i = 0; i < 2; i++)
      if (sv->slot[(oldest + i) % 2].busy) {
        d = &sv->slot[(oldest + i) % 2];
        oldest = (oldest + i + 1) % 2;
        break;
      }
    if (!d) continue;
    lk.unlock();
    drain_step(sv, *d);
    lk.lock();
  }
}

}  // namespace mg

using namespace mg;

extern "C" {

int mg_server_create(mg_index* ix, const mg_server_config* cfg, mg_server** out) {
  if (!ix || !out) return set_error(MG_ERR_INVAL, "null argument");
  *out = nullptr;
  if (cudaSetDevice(ix->device) != cudaSuccess) return set_error(MG_ERR_CUDA, "cudaSetDevice");
  mg_server* sv = new mg_server();
  sv->ix = ix;
  mg_server_config c = cfg ? *cfg : mg_server_config{0, 0, 0};
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  uint64_t budget = c.device_budget ? c.device_budget : (uint64_t)(free_b / 4);
  // per read of a step: ~300 bases, the result, 4 staging + 16 output candidates, overflow lists
  const uint64_t per_read = 320 + 16 + 20 * sizeof(mg_candidate) + 16;
  uint64_t reads = c.max_inflight_reads ? c.max_inflight_reads : 262144;
  reads = std::max<uint64_t>(1024, std::min<uint64_t>(reads, budget / 2 / per_read));
  sv->step_reads = reads;
  sv->step_bases = reads * 320;
  sv->max_requests = c.max_requests ? c.max_requests : 4096;
  sv->queue_budget = std::max<uint64_t>(budget, 64ull << 20);
  for (auto& s : sv->slot) {
    if (cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) != cudaSuccess ||
        slot_alloc(s, sv->step_reads, sv->step_bases, 16 * sv->step_reads + 1024) != MG_OK) {
      for (auto& t : sv->slot) slot_free(t);
      delete sv;
      return set_error(MG_ERR_OOM, "server step buffers");
    }
  }
  sv->th = std::thread(server_loop, sv);
  *out = sv;
  return MG_OK;
}

int mg_server_submit(mg_server* sv, const mg_batch* b, uint64_t* ticket) {
  if (!sv || !b || !ticket || (b->n_reads && (!b->offsets || !b->bases))) return set_error(MG_ERR_INVAL, "null argument");
  const uint64_t n = b->n_reads;
  const uint64_t nb = n ? b->offsets[n] : 0;
  if (n && b->offsets[0] != 0) return set_error(MG_ERR_INVAL, "offsets[0] must be 0");
  for (uint64_t i = 0; i < nb; i++)
    if (!has_complement(b->bases[i])) return set_error(MG_ERR_BADINPUT, "a read holds a byte without a reverse complement");
  for (uint64_t i = 0; i < n; i++)
    if (b->offsets[i + 1] < b->offsets[i] || b->offsets[i + 1] - b->offsets[i] > 65535)
      return set_error(MG_ERR_LIMIT, "read longer than 65535 bases");
  const uint64_t bytes = nb + (n + 1) * 8;
  std::unique_ptr<Request> r(new Request());
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->live.size() >= sv->max_requests || (sv->queued_bytes > 0 && sv->queued_bytes + bytes > sv->queue_budget))
      return set_error(MG_ERR_BUSY, "server at capacity");
    sv->queued_bytes += bytes;  // reserved before the copy
  }
  r->n = n;
  try {
    r->offs.assign(b->offsets, b->offsets + n + 1);
    r->bases.assign(b->bases, b->bases + nb);
    r->reads.resize(n);
  } catch (...) {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->queued_bytes -= bytes;
    return set_error(MG_ERR_OOM, "host memory for the request copy");
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  r->ticket = sv->next_ticket++;
  *ticket = r->ticket;
  if (n == 0) {
    r->complete = true;
    sv->queued_bytes -= bytes;
  } else {
    sv->queue.push_back(r.get());
  }
  sv->live[r->ticket] = std::move(r);
  sv->cv_work.notify_one();
  return MG_OK;
}

static int take_result(mg_server* sv, std::map<uint64_t, std::unique_ptr<Request>>::iterator it, mg_result* out) {
  Request* r = it->second.get();
  if (r->error) {
    int e = r->error;
    sv->live.erase(it);
    return set_error(e, "request failed on the device");
  }
  out->n_cands = r->cands.size();
  if (r->cands.size() > out->cand_cap) return set_error(MG_ERR_OOM, "candidate output buffer too small");
  if (r->n) std::memcpy(out->reads, r->reads.data(), r->n * sizeof(mg_read_result));
  if (!r->cands.empty()) std::memcpy(out->cands, r->cands.data(), r->cands.size() * sizeof(mg_candidate));
  sv->live.erase(it);
  return 1;
}

int mg_server_poll(mg_server* sv, uint64_t ticket, mg_result* out) {
  if (!sv || !out) return set_error(MG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->live.find(ticket);
  if (it == sv->live.end()) return set_error(MG_ERR_INVAL, "unknown ticket");
  if (!it->second->complete) return 0;
  return take_result(sv, it, out);
}

int mg_server_wait(mg_server* sv, uint64_t ticket, mg_result* out, uint32_t timeout_ms) {
  if (!sv || !out) return set_error(MG_ERR_INVAL, "null argument");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->live.find(ticket);
  if (it == sv->live.end()) return set_error(MG_ERR_INVAL, "unknown ticket");
  Request* r = it->second.get();
  if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->complete; }))
    return set_error(MG_ERR_TIMEOUT, "request not complete within the timeout");
  return take_result(sv, sv->live.find(ticket), out);
}

void mg_server_destroy(mg_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
    sv->queue.clear();
  }
  sv->cv_work.notify_all();
  if (sv->th.joinable()) sv->th.join();
  cudaSetDevice(sv->ix->device);
  for (auto& s : sv->slot) slot_free(s);
  delete sv;
}

}  // extern "C"
