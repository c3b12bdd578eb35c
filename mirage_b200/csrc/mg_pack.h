// 2-bit packing of read bases for the host-to-device copy (mg_pack.cpp) and its device unpack.
#pragma once
#include <cstdint>
#include <functional>

namespace mg {

// A fixed set of host threads that run one job at a time, the calling thread as thread 0.
class PackPool {
 public:
  explicit PackPool(int threads);
  ~PackPool();
  int threads() const { return n_; }
  void run(const std::function<void(int)>& job);  // job(t) for t in [0, threads), returns when all end

 private:
  struct Impl;
  Impl* impl_;
  int n_;
};

// Packs n bases of src into dst ((n + 3) / 4 bytes, four bases per byte, the first in the low
// bits) and lists every byte that is not A, C, G or T (either case) in exc as (offset << 8 | byte),
// in offset order. Returns the number of exceptions; when it exceeds exc_cap, exc is not written.
uint64_t pack_bases(PackPool& pool, const uint8_t* src, uint64_t n, uint8_t* dst, uint64_t* exc, uint64_t exc_cap,
                    uint64_t* n_exc);

}  // namespace mg
