// Load generator for the served form: client threads that drive an mg_server through the public
// C ABI (mg_server_submit_into / mg_server_wait) the way a C++ caller would, for throughput and
// latency measurement. Requests are contiguous slices of a pool of reads, with log-uniform sizes
// in [1, max_req] reads; each client rebases its slice's offsets into its own buffer and submits
// it (which copies it) with result buffers from its own pool, into which the server writes the
// results; a request whose candidates overflow its buffer is submitted again with a larger one.
//
//   rate_reads_s == 0: closed loop, each client keeps `depth` requests outstanding
//   rate_reads_s  > 0: open loop, Poisson arrivals split evenly over the clients; latency is
//                      measured from the scheduled arrival to the end of the wait
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "../../include/mirage_b200.h"

extern "C" {
typedef struct {
  double reads_per_s;  // reads completed / wall time of the run
  uint64_t requests, reads;
  double p50_ms, p99_ms, mean_ms;  // request latency (open loop: from the scheduled arrival)
  int error;                       // first MG_ERR_* seen, 0 if none
} mg_loadgen_report;
}

namespace {

using Clock = std::chrono::steady_clock;

struct Pool {
  const uint64_t* offs;
  const uint8_t* bases;
  uint64_t n;
  uint32_t max_req;
};

// Result buffers of one request, reused across requests (allocated and touched by the client,
// so the server's delivery threads write into resident pages).
struct Buf {
  std::vector<mg_read_result> reads;
  std::vector<mg_candidate> cands;
  mg_result res{};
  mg_batch batch{};
};

struct Client {
  std::mt19937_64 rng;
  std::vector<uint64_t> o;
  std::vector<double> lat_ms;
  std::mutex pool_mu;
  std::vector<std::unique_ptr<Buf>> pool;
  uint64_t reads_done = 0, requests = 0;
  int error = 0;
  explicit Client(uint64_t seed, uint32_t max_req) : rng(seed), o(max_req + 1), buf_reads(max_req) {}

  // a request: (first read, size); its offsets rebased into o
  mg_batch draw(const Pool& p, uint32_t* size_out) {
    std::uniform_real_distribution<double> u(0.0, std::log((double)p.max_req + 1.0));
    uint64_t size = (uint64_t)std::exp(u(rng));
    size = std::max<uint64_t>(1, std::min<uint64_t>(size, p.max_req));
    std::uniform_int_distribution<uint64_t> pick(0, p.n - size);
    const uint64_t st = pick(rng);
    const uint64_t b0 = p.offs[st];
    for (uint64_t i = 0; i <= size; i++) o[i] = p.offs[st + i] - b0;
    *size_out = (uint32_t)size;
    return mg_batch{size, o.data(), p.bases + b0};
  }
  // Buffers of one size, for the largest request (max_req reads, 4 candidates per read, more
  // on demand), made and touched before the measurement (warm), reused last in, first out.
  uint64_t buf_reads = 0;
  Buf* make_buf() {
    Buf* b = new Buf();
    b->reads.assign(buf_reads, mg_read_result{});
    b->cands.assign(4 * buf_reads + 64, mg_candidate{});
    return b;
  }
  void warm(int n) {
    for (int i = 0; i < n; i++) pool.emplace_back(make_buf());
  }
  Buf* acquire() {
    {
      std::lock_guard<std::mutex> lk(pool_mu);
      if (!pool.empty()) {
        Buf* b = pool.back().release();
        pool.pop_back();
        return b;
      }
    }
    return make_buf();  // more requests outstanding than were warmed
  }
  void release(Buf* b) {
    std::lock_guard<std::mutex> lk(pool_mu);
    pool.emplace_back(b);
  }
  int submit(mg_server* sv, const mg_batch& bt, Buf* b, uint64_t* t) {
    b->batch = bt;
    b->res = mg_result{b->reads.data(), b->cands.data(), b->cands.size(), 0};
    for (;;) {
      const int rc = mg_server_submit_into(sv, &bt, &b->res, t);
      if (rc != MG_ERR_BUSY) return rc;
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
  // waits for the request; one whose candidates did not fit goes again with a larger buffer (its
  // batch still points at the pool's reads; the rebased offsets are copied first)
  int wait(mg_server* sv, uint64_t t, Buf*& b) {
    for (;;) {
      const int rc = mg_server_wait(sv, t, nullptr, 600000);
      if (rc == 1) return MG_OK;
      if (rc != MG_ERR_OOM || b->res.n_cands <= b->cands.size()) return rc ? rc : MG_ERR_TIMEOUT;
      b->cands.assign(b->res.n_cands + 1024, mg_candidate{});
      std::vector<uint64_t> offs(b->batch.offsets, b->batch.offsets + b->batch.n_reads + 1);
      const mg_batch bt{b->batch.n_reads, offs.data(), b->batch.bases};
      if (int s = submit(sv, bt, b, &t)) return s;
    }
  }
};

// an outstanding request: ticket, (scheduled) submission time, reads, result buffers
struct Out {
  uint64_t ticket;
  Clock::time_point t0;
  uint32_t size;
  Buf* buf;
};

void closed_loop(mg_server* sv, const Pool& p, Client& c, Clock::time_point end, int depth) {
  std::deque<Out> q;
  while (Clock::now() < end && !c.error) {
    uint32_t size;
    const mg_batch b = c.draw(p, &size);
    uint64_t t;
    Buf* buf = c.acquire();
    const auto t0 = Clock::now();
    if (int rc = c.submit(sv, b, buf, &t)) {
      c.release(buf);
      c.error = rc;
      break;
    }
    q.push_back(Out{t, t0, size, buf});
    if ((int)q.size() >= depth) {
      Out f = q.front();
      q.pop_front();
      if (int rc = c.wait(sv, f.ticket, f.buf)) c.error = rc;
      c.lat_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - f.t0).count());
      c.reads_done += f.size;
      c.requests++;
      c.release(f.buf);
    }
  }
  while (!q.empty()) {
    Out f = q.front();
    q.pop_front();
    if (int rc = c.wait(sv, f.ticket, f.buf)) c.error = c.error ? c.error : rc;
    c.lat_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - f.t0).count());
    c.reads_done += f.size;
    c.requests++;
    c.release(f.buf);
  }
}

void open_loop(mg_server* sv, const Pool& p, Client& c, Clock::time_point start, double seconds,
               double req_per_s) {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Out> q;
  bool fin = false;
  std::thread waiter([&] {
    for (;;) {
      Out f;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return fin || !q.empty(); });
        if (q.empty()) return;
        f = q.front();
        q.pop_front();
      }
      if (int rc = c.wait(sv, f.ticket, f.buf)) c.error = c.error ? c.error : rc;
      c.lat_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - f.t0).count());
      c.reads_done += f.size;
      c.requests++;
      c.release(f.buf);
    }
  });
  std::exponential_distribution<double> gap(req_per_s);
  auto arrive = start;
  const auto end = start + std::chrono::duration<double>(seconds);
  while (!c.error) {
    arrive += std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(gap(c.rng)));
    if (arrive >= end) break;
    std::this_thread::sleep_until(arrive);
    uint32_t size;
    const mg_batch b = c.draw(p, &size);
    uint64_t t;
    Buf* buf = c.acquire();
    if (int rc = c.submit(sv, b, buf, &t)) {
      c.release(buf);
      c.error = rc;
      break;
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      q.push_back(Out{t, arrive, size, buf});
    }
    cv.notify_one();
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    fin = true;
  }
  cv.notify_one();
  waiter.join();
}

}  // namespace

extern "C" int mg_loadgen_run(mg_server* sv, const uint64_t* offs, const uint8_t* bases, uint64_t n_reads,
                              int clients, double seconds, uint32_t max_req, double rate_reads_s, int depth,
                              uint64_t seed, mg_loadgen_report* out) {
  if (!sv || !offs || !bases || !out || n_reads == 0 || clients < 1 || max_req < 1 || seconds <= 0)
    return MG_ERR_INVAL;
  Pool p{offs, bases, n_reads, (uint32_t)std::min<uint64_t>(max_req, n_reads)};
  std::vector<std::unique_ptr<Client>> cl;
  for (int i = 0; i < clients; i++) {
    cl.emplace_back(new Client(seed + 7919ull * (uint64_t)i, p.max_req));
    cl.back()->warm(rate_reads_s > 0 ? 16 : std::max(1, depth) + 1);  // before the clock starts
  }
  const double mean_size = p.max_req > 1 ? (double)(p.max_req - 1) / std::log((double)p.max_req) : 1.0;
  const auto t0 = Clock::now();
  std::vector<std::thread> th;
  for (int i = 0; i < clients; i++)
    th.emplace_back([&, i] {
      if (rate_reads_s > 0)
        open_loop(sv, p, *cl[i], t0, seconds, rate_reads_s / mean_size / clients);
      else
        closed_loop(sv, p, *cl[i], t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(seconds)),
                    std::max(1, depth));
    });
  for (auto& t : th) t.join();
  const double wall = std::chrono::duration<double>(Clock::now() - t0).count();
  std::vector<double> lat;
  std::memset(out, 0, sizeof(*out));
  for (auto& cp : cl) {
    const Client& c = *cp;
    lat.insert(lat.end(), c.lat_ms.begin(), c.lat_ms.end());
    out->reads += c.reads_done;
    out->requests += c.requests;
    if (c.error && !out->error) out->error = c.error;
  }
  out->reads_per_s = out->reads / wall;
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) { return lat[std::min(lat.size() - 1, (size_t)(q * (double)(lat.size() - 1) + 0.5))]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    double s = 0;
    for (double x : lat) s += x;
    out->mean_ms = s / lat.size();
  }
  return out->error;
}
