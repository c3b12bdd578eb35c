// Randomised check of the served form's request ring (mg_ring.h): live regions stay inside the
// ring and never overlap, an allocation that fails leaves the ring unchanged, and once every
// region is released the whole ring is available again. Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "mg_ring.h"

struct Live {
  uint64_t at, len;
};

static bool overlap(const Live& a, const Live& b) { return a.at < b.at + b.len && b.at < a.at + a.len; }

int main(int argc, char** argv) {
  const unsigned seed = argc > 1 ? (unsigned)atoi(argv[1]) : 1;
  std::mt19937_64 rng(seed);
  for (int trial = 0; trial < 200; trial++) {
    mg::Ring ring;
    ring.cap = 16 * (1 + rng() % 64);
    std::vector<Live> live;
    uint64_t ok = 0, refused = 0;
    for (int op = 0; op < 2000; op++) {
      if (live.empty() || rng() % 3) {
        const uint64_t want = 1 + rng() % (ring.cap / 2 + 1);
        uint64_t at = ~0ull;
        if (ring.alloc(want, &at)) {
          Live l{at, (want + 15) & ~15ull};
          if (l.at + l.len > ring.cap) {
            std::printf("trial %d op %d: region [%llu,+%llu) beyond cap %llu\n", trial, op,
                        (unsigned long long)l.at, (unsigned long long)l.len, (unsigned long long)ring.cap);
            return 1;
          }
          for (const Live& o : live)
            if (overlap(o, l)) {
              std::printf("trial %d op %d: overlap\n", trial, op);
              return 1;
            }
          live.push_back(l);
          ok++;
        } else {
          refused++;
        }
      } else {
        const size_t i = rng() % live.size();
        ring.release(live[i].at);
        live.erase(live.begin() + i);
      }
    }
    for (const Live& l : live) ring.release(l.at);
    uint64_t at = 1;
    if (!ring.alloc(ring.cap, &at) || at != 0) {
      std::printf("trial %d: empty ring refused a full-size region\n", trial);
      return 1;
    }
    if (!ok || !refused) {
      std::printf("trial %d: degenerate run (ok %llu refused %llu)\n", trial, (unsigned long long)ok,
                  (unsigned long long)refused);
      return 1;
    }
  }
  std::printf("ring ok\n");
  return 0;
}
