// Load generator for the served form: client threads that drive an mg_server through the public
// C ABI (mg_server_submit / mg_server_wait) the way a C++ caller would, for throughput and
// latency measurement. Requests are contiguous slices of a pool of reads, with log-uniform sizes
// in [1, max_req] reads; each client rebases its slice's offsets into its own buffer, submits it
// (which copies it) and collects the results into its own buffers.
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

struct Client {
  std::mt19937_64 rng;
  std::vector<uint64_t> o;
  std::vector<mg_read_result> reads;
  std::vector<mg_candidate> cands;
  std::vector<double> lat_ms;
  uint64_t reads_done = 0, requests = 0;
  int error = 0;
  explicit Client(uint64_t seed, uint32_t max_req)
      : rng(seed), o(max_req + 1), reads(max_req), cands((size_t)64 * max_req) {}

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
  int submit(mg_server* sv, const mg_batch& b, uint64_t* t) {
    for (;;) {
      const int rc = mg_server_submit(sv, &b, t);
      if (rc != MG_ERR_BUSY) return rc;
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
  int wait(mg_server* sv, uint64_t t) {
    mg_result r{reads.data(), cands.data(), cands.size(), 0};
    const int rc = mg_server_wait(sv, t, &r, 600000);
    return rc == 1 ? MG_OK : (rc ? rc : MG_ERR_TIMEOUT);
  }
};

void closed_loop(mg_server* sv, const Pool& p, Client& c, Clock::time_point end, int depth) {
  std::deque<std::pair<uint64_t, std::pair<Clock::time_point, uint32_t>>> q;
  while (Clock::now() < end && !c.error) {
    uint32_t size;
    const mg_batch b = c.draw(p, &size);
    uint64_t t;
    const auto t0 = Clock::now();
    if (int rc = c.submit(sv, b, &t)) {
      c.error = rc;
      break;
    }
    q.push_back({t, {t0, size}});
    if ((int)q.size() >= depth) {
      auto f = q.front();
      q.pop_front();
      if (int rc = c.wait(sv, f.first)) c.error = rc;
      c.lat_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - f.second.first).count());
      c.reads_done += f.second.second;
      c.requests++;
    }
  }
  while (!q.empty()) {
    auto f = q.front();
    q.pop_front();
    if (int rc = c.wait(sv, f.first)) c.error = c.error ? c.error : rc;
    c.lat_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - f.second.first).count());
    c.reads_done += f.second.second;
    c.requests++;
  }
}

void open_loop(mg_server* sv, const Pool& p, Client& c, Clock::time_point start, double seconds,
               double req_per_s) {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::pair<uint64_t, std::pair<Clock::time_point, uint32_t>>> q;
  bool fin = false;
  std::thread waiter([&] {
    for (;;) {
      std::pair<uint64_t, std::pair<Clock::time_point, uint32_t>> f;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return fin || !q.empty(); });
        if (q.empty()) return;
        f = q.front();
        q.pop_front();
      }
      if (int rc = c.wait(sv, f.first)) c.error = c.error ? c.error : rc;
      c.lat_ms.push_back(std::chrono::duration<double, std::milli>(Clock::now() - f.second.first).count());
      c.reads_done += f.second.second;
      c.requests++;
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
    if (int rc = c.submit(sv, b, &t)) {
      c.error = rc;
      break;
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      q.push_back({t, {arrive, size}});
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
  std::vector<Client> cl;
  cl.reserve(clients);
  for (int i = 0; i < clients; i++) cl.emplace_back(seed + 7919ull * (uint64_t)i, p.max_req);
  const double mean_size = p.max_req > 1 ? (double)(p.max_req - 1) / std::log((double)p.max_req) : 1.0;
  const auto t0 = Clock::now();
  std::vector<std::thread> th;
  for (int i = 0; i < clients; i++)
    th.emplace_back([&, i] {
      if (rate_reads_s > 0)
        open_loop(sv, p, cl[i], t0, seconds, rate_reads_s / mean_size / clients);
      else
        closed_loop(sv, p, cl[i], t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(seconds)),
                    std::max(1, depth));
    });
  for (auto& t : th) t.join();
  const double wall = std::chrono::duration<double>(Clock::now() - t0).count();
  std::vector<double> lat;
  std::memset(out, 0, sizeof(*out));
  for (auto& c : cl) {
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
