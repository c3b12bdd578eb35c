// Served form: continuous batching of classification requests against an HBM-resident index.
//
// Submit copies a request's reads once, into a pinned host ring shared by all requests; the
// ring is the admission budget (MG_ERR_BUSY when a request does not fit now, MG_ERR_LIMIT when
// it can never fit). A server thread forms "steps" from the queued reads in arrival order (a
// large request spans several steps, one step carries reads of many requests) and runs the
// fused pipeline on them; each request segment of a step is one host->device copy straight from
// the ring. Step slots (2 to 4), each with its own device workspace and stream, let the next
// step's copies and kernels run while earlier steps finish. A request arriving while steps are on
// the device joins the next step formed. Each read is classified on its own, so a request's
// results are the same alone and in any mix.
//
// Threads: the server thread carves, launches and waits for steps; a delivery thread hands each
// finished step's results to its requests, in launch order, and frees its slot. Each has a few
// worker threads for the per-read host work (rebasing offsets into the step; copying results out),
// split in pieces of at most 32,768 reads.
//
// Admission also holds device memory: each admitted request books the device bytes its reads
// take in a step (bases, offsets, results and a candidate allowance) against a budget, which
// follows the device's free memory as steps complete (another user's allocations shrink it).
// A request submitted with caller buffers (mg_server_submit_into) has its results written into
// them by the delivery thread, with no copy at completion. A request whose bases lie in
// host memory the server has page-locked for the caller (mg_server_register_host) is copied to
// the device from there, so submit copies only its offsets.
#include <cuda_runtime.h>
#include <sched.h>

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
#include "mg_pack.h"
#include "mg_ring.h"

namespace mg {

struct Request {
  uint64_t ticket = 0;
  uint64_t n = 0;
  uint64_t* offs = nullptr;     // in the pinned ring: n + 1 offsets
  const uint8_t* bases = nullptr;  // in the pinned ring, or in a range registered by the caller
  uint64_t ring_at = 0;
  uint64_t next = 0;  // next read to schedule
  uint64_t done = 0;  // reads with results
  std::vector<mg_read_result> reads;
  std::vector<mg_candidate> cands;
  mg_result* dst = nullptr;   // caller buffers (mg_server_submit_into), written as segments finish
  uint64_t n_cands = 0;       // candidates delivered (or needed, when dst's capacity ran out)
  uint64_t dev_bytes = 0;     // device bytes booked at admission
  int error = 0;
  bool complete = false;
  bool released = false;  // ring space returned
};

struct Part {
  Request* req;
  uint64_t first, count;  // reads [first, first+count) of req
};

// A run of at most kPieceReads consecutive reads of one part: the unit the worker threads rebase
// offsets and deliver results in.
struct Piece {
  uint32_t part;
  uint64_t at;            // first read of the piece in the step
  uint64_t in_part;       // first read of the piece in its part
  uint64_t count;
  uint64_t bases_at = 0;  // launch: first base of the piece in the step
  uint64_t base = 0;      // delivery: where the piece's first candidate goes in the request's output
  int err = 0;            // delivery: a rejected read's error
  bool deliver = false;   // delivery: copy this piece (the request takes it)
};
constexpr uint64_t kPieceReads = 32768;

struct Slot {
  Workspace ws;
  cudaStream_t st = nullptr;
  uint64_t* h_offs = nullptr;
  mg_read_result* h_reads = nullptr;
  mg_candidate* h_cands = nullptr;
  uint64_t cap_reads = 0, cap_cands = 0;
  std::vector<Part> parts;
  std::vector<Piece> pieces;
  uint64_t n = 0;
  bool busy = false;      // from carving until its results are delivered
  int launch_rc = 0;
  int drain_rc = 0;       // the step's status after the device part of draining
  mg_server* owner = nullptr;
  std::atomic<bool> device_done{false};  // the step's device work and read-result copy have finished
  std::chrono::steady_clock::time_point t_launch, t_done;  // launch start; end of the device work
};

}  // namespace mg

struct mg_server {
  mg_index* ix = nullptr;
  uint64_t step_reads = 0, step_bases = 0;
  uint64_t dev_budget = 0, dev_booked = 0;  // admission: device bytes of the admitted requests
  uint64_t dev_cap = 0;                     // the budget set at creation (the budget's ceiling)
  uint64_t dev_reserve = 0;                 // free device memory kept for the step buffers' growth
  std::chrono::steady_clock::time_point budget_read{};  // last read of the device's free memory
  uint32_t max_requests = 0;
  mg::Ring ring;
  uint64_t next_ticket = 1;
  std::deque<mg::Request*> queue;                          // requests with unscheduled reads
  std::map<uint64_t, std::unique_ptr<mg::Request>> live;   // every tracked request
  static constexpr int kMaxSlots = 4;
  mg::Slot slot[kMaxSlots];
  int n_slots = 3;                  // step slots in use (mg_server_config.step_slots)
  std::deque<int> in_flight;        // launched slots in launch order
  std::deque<int> to_deliver;       // drained slots in launch order, for the delivery thread
  std::condition_variable cv_deliver;
  bool stop_deliver = false;
  std::thread th_deliver;
  std::unique_ptr<mg::PackPool> pool_launch, pool_deliver;  // workers of the two threads
  struct HostRange {
    uintptr_t p;
    uint64_t len;
  };
  std::vector<HostRange> host_ranges;  // page-locked by mg_server_register_host (under mu)
  // mg_server_get_stats
  std::atomic<uint64_t> n_steps{0}, n_reads{0}, n_requests{0}, ring_bytes{0}, direct_bytes{0};
  std::atomic<uint64_t> ns_submit{0}, ns_launch{0}, ns_device{0}, ns_deliver{0}, ns_idle{0}, ns_step{0};
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
  if (cands > s.cap_cands) {
    if (s.h_cands) cudaFreeHost(s.h_cands);
    s.h_cands = nullptr;
    if (cudaMallocHost((void**)&s.h_cands, cands * sizeof(mg_candidate)) != cudaSuccess)
      return set_error(MG_ERR_OOM, "pinned step buffers");
    s.cap_cands = cands;
  }
  if (ensure_workspace(s.ws, reads, bases, true)) return MG_ERR_OOM;
  if (s.ws.cands.alloc(std::max<uint64_t>(s.cap_cands, 1) * sizeof(mg_candidate)))
    return set_error(MG_ERR_OOM, "step candidates");
  return MG_OK;
}

static void slot_free(Slot& s) {
  if (s.st) cudaStreamDestroy(s.st);
  if (s.h_offs) cudaFreeHost(s.h_offs);
  if (s.h_reads) cudaFreeHost(s.h_reads);
  if (s.h_cands) cudaFreeHost(s.h_cands);
  s.ws.release();
}

constexpr std::chrono::milliseconds kBudgetRefresh{50};
using Clock = std::chrono::steady_clock;

static uint64_t ns_since(Clock::time_point t0) {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t0).count();
}

// Take a step's worth of request segments from the queue (server lock held).
static void carve_step(mg_server* sv, Slot& s) {
  s.parts.clear();
  s.n = 0;
  uint64_t nb = 0;
  while (!sv->queue.empty() && s.n < sv->step_reads && nb < sv->step_bases) {
    Request* r = sv->queue.front();
    const uint64_t take = std::min(r->n - r->next, sv->step_reads - s.n);
    uint64_t got = take;
    // respect the base budget, but a step always carries at least one read
    const uint64_t room = sv->step_bases - nb;
    if (r->offs[r->next + got] - r->offs[r->next] > room) {
      uint64_t lo = 0, hi = take;  // largest got with bytes <= room
      while (lo < hi) {
        uint64_t mid = (lo + hi + 1) / 2;
        if (r->offs[r->next + mid] - r->offs[r->next] <= room) lo = mid;
        else hi = mid - 1;
      }
      got = std::max<uint64_t>(lo, s.n == 0 ? 1 : 0);
    }
    if (got == 0) break;
    s.parts.push_back(Part{r, r->next, got});
    nb += r->offs[r->next + got] - r->offs[r->next];
    r->next += got;
    s.n += got;
    if (r->next == r->n) sv->queue.pop_front();
  }
  s.busy = true;
  s.launch_rc = MG_OK;
  s.device_done = false;
}

// Split a step's parts into pieces of at most kPieceReads reads.
static void make_pieces(Slot& s) {
  s.pieces.clear();
  uint64_t at = 0;
  for (size_t i = 0; i < s.parts.size(); i++) {
    for (uint64_t f = 0; f < s.parts[i].count; f += kPieceReads) {
      Piece pc;
      pc.part = (uint32_t)i;
      pc.at = at + f;
      pc.in_part = f;
      pc.count = std::min(kPieceReads, s.parts[i].count - f);
      s.pieces.push_back(pc);
    }
    at += s.parts[i].count;
  }
}

// fn(piece) for every piece, on the pool's threads when the step is large enough to share
template <class F>
static void for_pieces(PackPool* pool, Slot& s, F&& fn) {
  const size_t np = s.pieces.size();
  if (!pool || np < 2 || s.n < 2 * kPieceReads) {
    for (size_t i = 0; i < np; i++) fn(s.pieces[i]);
    return;
  }
  const size_t T = (size_t)pool->threads();
  pool->run([&](int t) {
    for (size_t i = (size_t)t; i < np; i += T) fn(s.pieces[i]);
  });
}

// Copy a carved step's segments from the ring (or the caller's registered memory) and launch it on
// the slot's stream (server lock not held: the segments' requests stay queued-or-running, so their
// memory stays in place). The offsets, rebased into the step, are written by the launch workers.
static void launch_step_work(mg_server* sv, Slot& s) {
  if (s.n == 0) return;
  make_pieces(s);
  uint64_t nb = 0;
  for (Piece& pc : s.pieces) {
    const Part& p = s.parts[pc.part];
    pc.bases_at = nb;
    const uint64_t r0 = p.first + pc.in_part;
    nb += p.req->offs[r0 + pc.count] - p.req->offs[r0];
  }
  if (slot_alloc(s, s.n, std::max<uint64_t>(nb, sv->step_bases), std::max<uint64_t>(s.cap_cands, 16 * s.n + 1024))) {
    s.launch_rc = MG_ERR_OOM;
    return;
  }
  s.h_offs[0] = 0;
  for_pieces(sv->pool_launch.get(), s, [&](const Piece& pc) {
    const Part& p = s.parts[pc.part];
    const uint64_t* ro = p.req->offs + p.first + pc.in_part;
    const uint64_t d = pc.bases_at - ro[0];  // modulo 2^64: ro[j] - ro[0] + bases_at
    uint64_t* out = s.h_offs + pc.at + 1;
    for (uint64_t j = 0; j < pc.count; j++) out[j] = ro[j + 1] + d;
  });
  // bases: one copy per part (its pieces are contiguous in the source and in the step)
  cudaError_t e = cudaSuccess;
  uint64_t ob = 0;
  for (const Part& p : s.parts) {
    const uint64_t b0 = p.req->offs[p.first], b1 = p.req->offs[p.first + p.count];
    if (e == cudaSuccess && b1 > b0)
      e = cudaMemcpyAsync(s.ws.bases.as<uint8_t>() + ob, p.req->bases + b0, b1 - b0, cudaMemcpyHostToDevice, s.st);
    ob += b1 - b0;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(s.ws.offs.p, s.h_offs, (s.n + 1) * 8, cudaMemcpyHostToDevice, s.st);
  if (e != cudaSuccess) {
    s.launch_rc = set_error(MG_ERR_CUDA, cudaGetErrorString(e));
    return;
  }
  s.launch_rc = run_pipeline(sv->ix, s.ws, s.n, s.ws.offs.as<uint64_t>(), s.ws.bases.as<uint8_t>(),
                             s.ws.reads.as<mg_read_result>(), s.ws.cands.as<mg_candidate>(), s.cap_cands, s.st, false);
  if (s.launch_rc == MG_OK &&
      cudaMemcpyAsync(s.h_reads, s.ws.reads.p, s.n * sizeof(mg_read_result), cudaMemcpyDeviceToHost, s.st) != cudaSuccess)
    s.launch_rc = MG_ERR_CUDA;
}

// Host function enqueued after a step's work: marks the step done on the device and wakes the
// server thread (no CUDA call here). The notify happens under the lock, so once the lock is
// released this function touches the server no more (the server may then be destroyed).
static void CUDART_CB step_done(void* p) {
  Slot* s = static_cast<Slot*>(p);
  mg_server* sv = s->owner;
  std::lock_guard<std::mutex> lk(sv->mu);
  s->t_done = Clock::now();
  s->device_done = true;
  sv->cv_work.notify_one();
}

static void launch_step(mg_server* sv, Slot& s) {
  s.t_launch = Clock::now();
  s.t_done = s.t_launch;
  launch_step_work(sv, s);
  if (s.launch_rc == MG_OK && s.n) {
    if (cudaLaunchHostFunc(s.st, step_done, &s) == cudaSuccess) return;
    s.launch_rc = set_error(MG_ERR_CUDA, "cudaLaunchHostFunc");
  }
  s.device_done = true;  // nothing to wait for (drain_device synchronises the stream on an error)
}

// Bring a step that has finished on the device to the slot's pinned buffers (server thread;
// lock not held). The step's status goes to s.drain_rc for the delivery thread.
static void drain_device(mg_server* sv, Slot& s) {
  const auto t_wait = Clock::now();
  int rc = s.launch_rc;
  Counters c;
  if (rc != MG_OK) cudaStreamSynchronize(s.st);  // copies from the ring may still be in flight
  auto run = [&]() {
    return run_pipeline(sv->ix, s.ws, s.n, s.ws.offs.as<uint64_t>(), s.ws.bases.as<uint8_t>(),
                        s.ws.reads.as<mg_read_result>(), s.ws.cands.as<mg_candidate>(), s.cap_cands, s.st, false);
  };
  auto complete = [&]() {
    return complete_pipeline(sv->ix, s.ws, s.n, s.ws.offs.as<uint64_t>(), s.ws.bases.as<uint8_t>(),
                             s.ws.reads.as<mg_read_result>(), s.ws.cands.as<mg_candidate>(), s.cap_cands, s.st,
                             false, &c);
  };
  bool reran = false;
  if (rc == MG_OK && s.n) {
    rc = complete();
    reran = c.reran;
  }
  if (rc == MG_OK && (c.err & kErrOutput) && c.n_cands > s.cap_cands) {
    // more candidates than the step buffer holds: rerun the step with room for all of them
    rc = slot_alloc(s, s.n, s.ws.bases.n, c.n_cands + 1024);
    if (rc == MG_OK) rc = run();
    if (rc == MG_OK) rc = complete();
    reran = true;
  }
  // a rejected read fails its own request only (at delivery); any other error fails the step
  const int step_bits = c.err & ~(kErrBadInput | kErrLimit);
  if (rc == MG_OK && step_bits) rc = error_status(step_bits);
  if (rc == MG_OK && s.n) {
    if ((reran && cudaMemcpyAsync(s.h_reads, s.ws.reads.p, s.n * sizeof(mg_read_result), cudaMemcpyDeviceToHost,
                                  s.st) != cudaSuccess) ||
        (c.n_cands && cudaMemcpyAsync(s.h_cands, s.ws.cands.p, c.n_cands * sizeof(mg_candidate),
                                      cudaMemcpyDeviceToHost, s.st) != cudaSuccess) ||
        cudaStreamSynchronize(s.st) != cudaSuccess)
      rc = set_error(MG_ERR_CUDA, "step results");
  }
  s.drain_rc = rc;
  if (s.t_done > s.t_launch)
    sv->ns_step += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(s.t_done - s.t_launch).count();
  // the device budget follows the device's free memory, read at most every kBudgetRefresh (the
  // query is a driver call, too slow for every step)
  const auto now = Clock::now();
  if (now - sv->budget_read >= kBudgetRefresh) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      std::lock_guard<std::mutex> lk(sv->mu);
      const uint64_t room = free_b > sv->dev_reserve ? free_b - sv->dev_reserve : 0;
      sv->dev_budget = std::min(sv->dev_cap, room + sv->dev_booked);
    }
    sv->budget_read = now;
  }
  sv->ns_device += ns_since(t_wait);
}

// Hand a drained step's results to its requests (delivery thread; lock not held). Until a request
// completes only this thread writes its results, count and error code, and steps are delivered in
// launch order, so a request's segments arrive in read order. A first pass over the pieces, in
// order, places each one in its request's output; the copies then run on the delivery workers.
static void deliver_step(mg_server* sv, Slot& s) {
  const auto t0 = Clock::now();
  const int rc = s.drain_rc;
  uint64_t c0 = 0, base = 0;  // the current part's first candidate in the step and in its request
  for (Piece& pc : s.pieces) {
    const Part& p = s.parts[pc.part];
    Request* r = p.req;
    pc.deliver = false;
    pc.err = 0;
    const mg_read_result* src = s.h_reads + pc.at;
    const uint64_t pc0 = src[0].cand_off;
    const mg_read_result& last = src[pc.count - 1];
    const uint64_t pc1 = (uint64_t)last.cand_off + last.n_fwd + last.n_rc;
    if (pc.in_part == 0) {  // the part's first piece: the part's candidates go after the request's
      c0 = pc0;
      base = r->n_cands;
      if (rc != MG_OK) r->error = rc;
    }
    if (rc != MG_OK) continue;
    if (r->error) {
      // a request whose error came from an earlier segment still counts the candidates it needs
      if (r->dst && r->error == MG_ERR_OOM) r->n_cands += pc1 - pc0;
      continue;
    }
    r->n_cands += pc1 - pc0;
    pc.base = base + (pc0 - c0);
    if (r->dst) {
      if (r->n_cands > r->dst->cand_cap) {
        r->error = MG_ERR_OOM;  // n_cands keeps counting what the request needs
        continue;
      }
    } else {
      try {
        r->cands.resize(r->n_cands);
      } catch (...) {
        r->error = MG_ERR_OOM;
        continue;
      }
    }
    pc.deliver = true;
  }
  for_pieces(sv->pool_deliver.get(), s, [&](Piece& pc) {
    if (!pc.deliver) return;
    const Part& p = s.parts[pc.part];
    Request* r = p.req;
    const mg_read_result* src = s.h_reads + pc.at;
    const uint64_t pc0 = src[0].cand_off;
    const mg_read_result& last = src[pc.count - 1];
    const uint64_t pc1 = (uint64_t)last.cand_off + last.n_fwd + last.n_rc;
    mg_candidate* cd = r->dst ? r->dst->cands : r->cands.data();
    if (pc1 > pc0) std::memcpy(cd + pc.base, s.h_cands + pc0, (pc1 - pc0) * sizeof(mg_candidate));
    mg_read_result* dst = (r->dst ? r->dst->reads : r->reads.data()) + p.first + pc.in_part;
    for (uint64_t i = 0; i < pc.count; i++) {
      mg_read_result rr = src[i];
      if (rr.strand == MG_READ_BAD_BYTE || rr.strand == MG_READ_TOO_LARGE) {
        pc.err = rr.strand == MG_READ_BAD_BYTE ? MG_ERR_BADINPUT : MG_ERR_LIMIT;
        break;
      }
      rr.cand_off = (uint32_t)(rr.cand_off - pc0 + pc.base);
      dst[i] = rr;
    }
  });
  for (const Piece& pc : s.pieces)
    if (pc.err && !s.parts[pc.part].req->error) s.parts[pc.part].req->error = pc.err;
  sv->ns_deliver += ns_since(t0);
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->n_steps++;
  sv->n_reads += s.n;
  for (const Part& p : s.parts) {
    Request* r = p.req;
    r->done += p.count;
    if (r->done == r->n) {
      r->complete = true;
      sv->n_requests++;
      if (!r->released) {
        sv->ring.release(r->ring_at);
        r->released = true;
      }
      sv->dev_booked -= r->dev_bytes;
      r->dev_bytes = 0;
    }
  }
  s.parts.clear();
  s.pieces.clear();
  s.busy = false;
  sv->cv_done.notify_all();
  sv->cv_work.notify_one();  // a slot is free for the server thread
}

static bool slot_free_now(const mg_server* sv) {
  for (int i = 0; i < sv->n_slots; i++)
    if (!sv->slot[i].busy) return true;
  return false;
}

// Server thread: carves and launches steps into free slots, and drains the oldest launched step
// once it has finished on the device; the delivery thread then hands its results out and frees
// the slot. It sleeps until one of those can happen: work and a free slot (a delivery freed
// one, or a request came), or the oldest step done (its host function).
static void server_loop(mg_server* sv) {
  cudaSetDevice(sv->ix->device);
  std::unique_lock<std::mutex> lk(sv->mu);
  auto oldest_done = [&] { return !sv->in_flight.empty() && sv->slot[sv->in_flight.front()].device_done; };
  for (;;) {
    const auto t_idle = Clock::now();
    sv->cv_work.wait(lk, [&] {
      return (sv->stop && sv->in_flight.empty()) || (!sv->stop && !sv->queue.empty() && slot_free_now(sv)) ||
             oldest_done();
    });
    sv->ns_idle += ns_since(t_idle);
    if (sv->stop && sv->in_flight.empty()) break;
    // launch into every free slot while there is work (asynchronous)
    for (int i = 0; i < sv->n_slots && !sv->queue.empty(); i++) {
      Slot& s = sv->slot[i];
      if (!s.busy) {
        carve_step(sv, s);
        sv->in_flight.push_back(i);
        lk.unlock();
        const auto t_launch = Clock::now();
        launch_step(sv, s);
        sv->ns_launch += ns_since(t_launch);
        lk.lock();
      }
    }
    // drain the oldest launched step when it is done, then pass it to the delivery thread
    if (!oldest_done()) continue;
    const int d = sv->in_flight.front();
    sv->in_flight.pop_front();
    lk.unlock();
    drain_device(sv, sv->slot[d]);
    lk.lock();
    sv->to_deliver.push_back(d);
    sv->cv_deliver.notify_one();
  }
}

static void deliver_loop(mg_server* sv) {
  std::unique_lock<std::mutex> lk(sv->mu);
  for (;;) {
    sv->cv_deliver.wait(lk, [&] { return sv->stop_deliver || !sv->to_deliver.empty(); });
    if (sv->to_deliver.empty()) break;  // stop_deliver, nothing left
    const int d = sv->to_deliver.front();
    sv->to_deliver.pop_front();
    lk.unlock();
    deliver_step(sv, sv->slot[d]);
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
  mg_server_config c = cfg ? *cfg : mg_server_config{0, 0, 0, 0};
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  // device memory for the two step slots: ~0.6 KB per read of a step
  const uint64_t per_read = 320 + 16 + 20 * sizeof(mg_candidate) + 16;
  const uint64_t dev_budget = c.device_budget ? c.device_budget : (uint64_t)(free_b / 4);
  uint64_t reads = c.max_inflight_reads ? c.max_inflight_reads : 262144;
  reads = std::max<uint64_t>(1024, std::min<uint64_t>(reads, dev_budget / 2 / per_read));
  sv->dev_cap = sv->dev_budget = dev_budget;
  sv->dev_reserve = (uint64_t)(free_b / 8);  // kept free beyond the budget
  sv->step_reads = reads;
  sv->step_bases = reads * 320;
  sv->max_requests = c.max_requests ? c.max_requests : 4096;
  sv->n_slots = c.step_slots ? (int)std::min<uint32_t>(std::max<uint32_t>(c.step_slots, 2), mg_server::kMaxSlots) : 3;
  // pinned ring for queued requests: (slots + 2) steps' worth of reads, at least 64 MB
  sv->ring.cap = std::max<uint64_t>(64ull << 20, (uint64_t)(sv->n_slots + 2) * (sv->step_bases + (sv->step_reads + 1) * 8));
  if (cudaMallocHost((void**)&sv->ring.base, sv->ring.cap) != cudaSuccess) {
    delete sv;
    return set_error(MG_ERR_OOM, "pinned request ring");
  }
  for (int i = 0; i < sv->n_slots; i++) {
    Slot& s = sv->slot[i];
    s.owner = sv;
    if (cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) != cudaSuccess ||
        slot_alloc(s, sv->step_reads, sv->step_bases, 16 * sv->step_reads + 1024) != MG_OK) {
      for (auto& t : sv->slot) slot_free(t);
      cudaFreeHost(sv->ring.base);
      delete sv;
      return set_error(MG_ERR_OOM, "server step buffers");
    }
  }
  // workers for the offsets (server thread) and the results (delivery thread): a quarter of the
  // CPUs this process may use, 1 to 4 each
  {
    cpu_set_t set;
    int cpus = 0;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) cpus = CPU_COUNT(&set);
    if (cpus <= 0) cpus = (int)std::thread::hardware_concurrency();
    const int w = std::max(1, std::min(4, cpus / 4));
    sv->pool_launch.reset(new PackPool(w));
    sv->pool_deliver.reset(new PackPool(w));
  }
  sv->th_deliver = std::thread(deliver_loop, sv);
  sv->th = std::thread(server_loop, sv);
  ix->n_servers++;
  *out = sv;
  return MG_OK;
}

// Device bytes a request books: its bases and offsets on the device, its read results and an
// allowance of 8 candidates per read (the step buffers grow beyond it when needed).
static uint64_t request_device_bytes(uint64_t n, uint64_t nb) {
  return nb + (n + 1) * 8 + n * (sizeof(mg_read_result) + 8 * sizeof(mg_candidate));
}

static int submit(mg_server* sv, const mg_batch* b, mg_result* dst, uint64_t* ticket) {
  if (!sv || !b || !ticket || (b->n_reads && (!b->offsets || !b->bases))) return set_error(MG_ERR_INVAL, "null argument");
  if (dst && b->n_reads && (!dst->reads || (dst->cand_cap && !dst->cands)))
    return set_error(MG_ERR_INVAL, "null output buffer");
  const uint64_t n = b->n_reads;
  const uint64_t nb = n ? b->offsets[n] : 0;
  if (n && b->offsets[0] != 0) return set_error(MG_ERR_INVAL, "offsets[0] must be 0");
  for (uint64_t i = 0; i < n; i++)
    if (b->offsets[i + 1] < b->offsets[i] || b->offsets[i + 1] - b->offsets[i] > 65535)
      return set_error(MG_ERR_LIMIT, "read longer than 65535 bases");
  std::unique_ptr<Request> r(new Request());
  r->n = n;
  r->dst = dst;
  const uint64_t dev = request_device_bytes(n, nb);
  bool direct = false;  // bases read in place, from a range registered with the server
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    const uintptr_t b0 = (uintptr_t)b->bases;
    for (const auto& h : sv->host_ranges)
      if (nb && b0 >= h.p && b0 - h.p <= h.len && nb <= h.len - (b0 - h.p)) {
        direct = true;
        break;
      }
    const uint64_t len = (direct ? 0 : nb) + (n + 1) * 8 + 16;
    if (len > sv->ring.cap) return set_error(MG_ERR_LIMIT, "request larger than the server's request memory");
    if (dev > sv->dev_cap) return set_error(MG_ERR_LIMIT, "request larger than the server's device budget");
    if (sv->dev_booked + dev > sv->dev_budget) return set_error(MG_ERR_BUSY, "not enough free device memory now");
    if (sv->live.size() >= sv->max_requests || !sv->ring.alloc(len, &r->ring_at))
      return set_error(MG_ERR_BUSY, "server at capacity");
    sv->dev_booked += dev;
    r->dev_bytes = dev;
    r->offs = (uint64_t*)(sv->ring.base + r->ring_at);
    r->bases = direct ? b->bases : sv->ring.base + r->ring_at + (n + 1) * 8;
  }
  const auto t_copy = Clock::now();
  std::memcpy(r->offs, b->offsets, (n + 1) * 8);
  if (direct) {
    sv->direct_bytes += nb;
  } else {
    std::memcpy(sv->ring.base + r->ring_at + (n + 1) * 8, b->bases, nb);
    sv->ring_bytes += nb;
  }
  sv->ns_submit += ns_since(t_copy);
  if (!dst) {
    try {
      r->reads.resize(n);
    } catch (...) {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->ring.release(r->ring_at);
      sv->dev_booked -= dev;
      return set_error(MG_ERR_OOM, "host memory for the results");
    }
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  r->ticket = sv->next_ticket++;
  *ticket = r->ticket;
  if (n == 0) {
    r->complete = true;
    r->released = true;
    sv->ring.release(r->ring_at);
    sv->dev_booked -= r->dev_bytes;
    r->dev_bytes = 0;
  } else {
    sv->queue.push_back(r.get());
  }
  sv->live[r->ticket] = std::move(r);
  sv->cv_work.notify_one();
  return MG_OK;
}

int mg_server_submit(mg_server* sv, const mg_batch* b, uint64_t* ticket) { return submit(sv, b, nullptr, ticket); }

int mg_server_submit_into(mg_server* sv, const mg_batch* b, mg_result* out, uint64_t* ticket) {
  if (!out) return set_error(MG_ERR_INVAL, "null output");
  return submit(sv, b, out, ticket);
}

// Hand a completed request to its caller: detached from the server under the lock, copied out and
// freed after the lock is released. A request whose candidates do not fit stays for a retry.
static int take_result(mg_server* sv, std::map<uint64_t, std::unique_ptr<Request>>::iterator it, mg_result* out,
                       std::unique_lock<std::mutex>& lk) {
  Request* r0 = it->second.get();
  if (r0->dst) {  // results are in the caller's buffers already
    std::unique_ptr<Request> r = std::move(it->second);
    sv->live.erase(it);
    lk.unlock();
    r->dst->n_cands = r->n_cands;
    if (out) out->n_cands = r->n_cands;
    if (r->error == MG_ERR_OOM) return set_error(MG_ERR_OOM, "candidate output buffer too small");
    if (r->error) return set_error(r->error, mg_strerror(r->error));
    return 1;
  }
  if (!out) return set_error(MG_ERR_INVAL, "null output");
  if (!r0->error && r0->cands.size() > out->cand_cap) {
    out->n_cands = r0->cands.size();
    return set_error(MG_ERR_OOM, "candidate output buffer too small");
  }
  std::unique_ptr<Request> r = std::move(it->second);
  sv->live.erase(it);
  lk.unlock();
  if (r->error) return set_error(r->error, mg_strerror(r->error));
  out->n_cands = r->cands.size();
  if (r->n) std::memcpy(out->reads, r->reads.data(), r->n * sizeof(mg_read_result));
  if (!r->cands.empty()) std::memcpy(out->cands, r->cands.data(), r->cands.size() * sizeof(mg_candidate));
  return 1;
}

int mg_server_poll(mg_server* sv, uint64_t ticket, mg_result* out) {
  if (!sv) return set_error(MG_ERR_INVAL, "null argument");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->live.find(ticket);
  if (it == sv->live.end()) return set_error(MG_ERR_INVAL, "unknown ticket");
  if (!it->second->complete) return 0;
  return take_result(sv, it, out, lk);
}

int mg_server_wait(mg_server* sv, uint64_t ticket, mg_result* out, uint32_t timeout_ms) {
  if (!sv) return set_error(MG_ERR_INVAL, "null argument");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->live.find(ticket);
  if (it == sv->live.end()) return set_error(MG_ERR_INVAL, "unknown ticket");
  Request* r = it->second.get();
  if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->complete; }))
    return set_error(MG_ERR_TIMEOUT, "request not complete within the timeout");
  return take_result(sv, sv->live.find(ticket), out, lk);
}

int mg_server_register_host(mg_server* sv, const void* ptr, uint64_t len) {
  if (!sv || !ptr || !len) return set_error(MG_ERR_INVAL, "null argument");
  if (cudaSetDevice(sv->ix->device) != cudaSuccess) return set_error(MG_ERR_CUDA, "cudaSetDevice");
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, ptr) == cudaSuccess && at.type != cudaMemoryTypeUnregistered)
    return set_error(MG_ERR_INVAL, "range is page-locked already, or device memory");
  cudaGetLastError();
  const cudaError_t e = cudaHostRegister(const_cast<void*>(ptr), len, cudaHostRegisterDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();  // not sticky: clear it
    if (e == cudaErrorHostMemoryAlreadyRegistered) return set_error(MG_ERR_INVAL, "range is page-locked already");
    return set_error(MG_ERR_CUDA, cudaGetErrorString(e));
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->host_ranges.push_back(mg_server::HostRange{(uintptr_t)ptr, len});
  return MG_OK;
}

int mg_server_get_stats(mg_server* sv, mg_server_stats* out) {
  if (!sv || !out) return set_error(MG_ERR_INVAL, "null argument");
  out->steps = sv->n_steps;
  out->reads = sv->n_reads;
  out->requests = sv->n_requests;
  out->ring_bytes = sv->ring_bytes;
  out->direct_bytes = sv->direct_bytes;
  out->submit_copy_s = sv->ns_submit * 1e-9;
  out->launch_s = sv->ns_launch * 1e-9;
  out->device_s = sv->ns_device * 1e-9;
  out->deliver_s = sv->ns_deliver * 1e-9;
  out->idle_s = sv->ns_idle * 1e-9;
  out->step_s = sv->ns_step * 1e-9;
  return MG_OK;
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
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop_deliver = true;
  }
  sv->cv_deliver.notify_all();
  if (sv->th_deliver.joinable()) sv->th_deliver.join();
  cudaSetDevice(sv->ix->device);
  for (auto& s : sv->slot) slot_free(s);
  if (sv->ring.base) cudaFreeHost(sv->ring.base);
  for (const auto& h : sv->host_ranges) cudaHostUnregister((void*)h.p);
  sv->ix->n_servers--;
  delete sv;
}

}  // extern "C"
