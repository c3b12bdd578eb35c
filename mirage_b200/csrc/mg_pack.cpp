// 2-bit packing of read bases on the host, for the host-to-device copy of the batched form.
//
// A base A, C, G or T (either case) becomes its 2-bit code ((b >> 1) ^ (b >> 2)) & 3: A 0, C 1,
// G 2, T 3, the same for a, c, g, t, four per byte, the first base in the low bits. Every other
// byte is an exception: its offset and the byte itself go to a list, and its 2-bit slot holds
// whatever the formula gives. The device unpacks a chunk into upper-case ASCII and then writes
// the exceptions back, so the bytes the kernels read differ from the caller's only in the case
// of a, c, g and t, which the kernels fold to upper case on reading (Sequences.cpp:43-55) before
// any use. The copy moves a quarter of the bytes.
#include <immintrin.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "mg_pack.h"

namespace mg {

namespace {

inline bool is_base(uint8_t b) {
  const uint8_t l = b | 0x20;
  return l == 'a' || l == 'c' || l == 'g' || l == 't';
}
inline uint32_t code(uint8_t b) { return ((b >> 1) ^ (b >> 2)) & 3u; }

// Bases [a, b) of src (a and b multiples of 4 or b == n): packed bytes to dst[a / 4 ..], exceptions
// appended to exc as (offset << 8 | byte).
void pack_scalar(const uint8_t* src, uint64_t a, uint64_t b, uint8_t* dst, std::vector<uint64_t>& exc) {
  for (uint64_t i = a; i < b; i += 4) {
    uint32_t v = 0;
    for (uint64_t t = 0; t < 4 && i + t < b; t++) {
      const uint8_t c = src[i + t];
      if (!is_base(c)) exc.push_back(((i + t) << 8) | c);
      v |= code(c) << (2 * t);
    }
    dst[i >> 2] = (uint8_t)v;
  }
}

// 128 bases per step: each byte's code c, then its validity as (byte | 0x20) == "acgt"[c] (a byte
// passes exactly when it is one of A, C, G, T in either case: those are the only bytes whose
// lower-case form is a, c, g or t, and each maps to its own letter), one branch per step; the codes
// of 4 consecutive bytes summed into one byte (c0 + 4 c1 + 16 c2 + 64 c3) per 32-bit lane, and
// the four vectors' lanes narrowed and put in order for one 32-byte store.
__attribute__((target("avx2"))) void pack_avx2(const uint8_t* src, uint64_t a, uint64_t b, uint8_t* dst,
                                               std::vector<uint64_t>& exc) {
  const __m256i lo20 = _mm256_set1_epi8(0x20), three = _mm256_set1_epi8(3);
  const __m256i letters = _mm256_setr_epi8('a', 'c', 'g', 't', 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 'a', 'c', 'g', 't',
                                           0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0);
  const __m256i w14 = _mm256_set1_epi16(0x0401);       // bytes (1, 4): c0 + 4 c1 per 16 bits
  const __m256i w116 = _mm256_set1_epi32(0x00100001);  // halves (1, 16): + 16 (c2 + 4 c3)
  const __m256i order = _mm256_setr_epi32(0, 4, 1, 5, 2, 6, 3, 7);
  uint64_t i = a;
  for (; i + 128 <= b; i += 128) {
    __m256i p[4], ok = _mm256_set1_epi8(-1);
    for (int v = 0; v < 4; v++) {
      const __m256i x = _mm256_loadu_si256((const __m256i*)(src + i + 32 * v));
      // per-byte codes: the 16-bit shifts carry bits across bytes only above bit 1, which & 3 drops
      const __m256i c = _mm256_and_si256(_mm256_xor_si256(_mm256_srli_epi16(x, 1), _mm256_srli_epi16(x, 2)), three);
      ok = _mm256_and_si256(ok, _mm256_cmpeq_epi8(_mm256_or_si256(x, lo20), _mm256_shuffle_epi8(letters, c)));
      p[v] = _mm256_madd_epi16(_mm256_maddubs_epi16(c, w14), w116);  // one packed byte per 32-bit lane
    }
    if ((uint32_t)_mm256_movemask_epi8(ok) != 0xFFFFFFFFu) {
      for (uint64_t t = i; t < i + 128; t++)
        if (!is_base(src[t])) exc.push_back((t << 8) | src[t]);
    }
    // dwords after the two narrowings: [A0-3 B0-3 C0-3 D0-3 | A4-7 B4-7 C4-7 D4-7] -> A B C D
    const __m256i n16 = _mm256_packus_epi16(_mm256_packus_epi32(p[0], p[1]), _mm256_packus_epi32(p[2], p[3]));
    _mm256_storeu_si256((__m256i*)(dst + (i >> 2)), _mm256_permutevar8x32_epi32(n16, order));
  }
  pack_scalar(src, i, b, dst, exc);
}

bool have_avx2() {
  static const bool v = __builtin_cpu_supports("avx2");
  return v;
}

}  // namespace

// Worker threads that pack the slices of a chunk.
struct PackPool::Impl {
  std::vector<std::thread> th;
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::function<void(int)> job;
  uint64_t gen = 0;
  int pending = 0;
  bool stop = false;
};

PackPool::PackPool(int threads) : impl_(new Impl()), n_(std::max(1, threads)) {
  for (int t = 1; t < n_; t++)
    impl_->th.emplace_back([this, t] {
      uint64_t seen = 0;
      for (;;) {
        std::function<void(int)> job;
        {
          std::unique_lock<std::mutex> lk(impl_->mu);
          impl_->cv.wait(lk, [&] { return impl_->stop || impl_->gen != seen; });
          if (impl_->stop) return;
          seen = impl_->gen;
          job = impl_->job;
        }
        job(t);
        std::lock_guard<std::mutex> lk(impl_->mu);
        if (--impl_->pending == 0) impl_->cv_done.notify_all();
      }
    });
}

PackPool::~PackPool() {
  {
    std::lock_guard<std::mutex> lk(impl_->mu);
    impl_->stop = true;
  }
  impl_->cv.notify_all();
  for (auto& t : impl_->th) t.join();
  delete impl_;
}

void PackPool::run(const std::function<void(int)>& job) {
  {
    std::lock_guard<std::mutex> lk(impl_->mu);
    impl_->job = job;
    impl_->pending = n_ - 1;
    impl_->gen++;
  }
  impl_->cv.notify_all();
  job(0);
  std::unique_lock<std::mutex> lk(impl_->mu);
  impl_->cv_done.wait(lk, [&] { return impl_->pending == 0; });
}

uint64_t pack_bases(PackPool& pool, const uint8_t* src, uint64_t n, uint8_t* dst, uint64_t* exc, uint64_t exc_cap,
                    uint64_t* n_exc) {
  const int T = pool.threads();
  // slices of whole 128-byte steps, so every slice but the last starts and ends on a packed byte
  const uint64_t per = ((n + T - 1) / T + 127) / 128 * 128;
  std::vector<std::vector<uint64_t>> local(T);
  pool.run([&](int t) {
    const uint64_t a = std::min(n, per * (uint64_t)t), b = std::min(n, a + per);
    if (a < b) {
      if (have_avx2()) pack_avx2(src, a, b, dst, local[t]);
      else pack_scalar(src, a, b, dst, local[t]);
    }
  });
  uint64_t total = 0;
  for (auto& v : local) total += v.size();
  *n_exc = total;
  if (total > exc_cap) return total;
  uint64_t at = 0;
  for (auto& v : local) {
    if (!v.empty()) std::memcpy(exc + at, v.data(), v.size() * 8);
    at += v.size();
  }
  return total;
}

}  // namespace mg
