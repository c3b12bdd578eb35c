// .mhm reader and writer; see mhm.h for the layout and the reference sources it follows.
#include "mhm.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <thread>

namespace mg {

static const char kMagic[] = "MirAge - Maarten Pater - www.mirdesign.nl - mirage@mirdesign.nl - Hashmap";
static const int kVersion = 4;  // Hashmap.h:252

// CreateHash32 / CreateHash24 with HashBits = 28 (Hashmap.cpp:3197-3268, Hashmap.h:111).
uint32_t hash28(const uint8_t* p, int len) {
  uint32_t h = 2166136261u;
  for (int i = 0; i < len; i++) h = (h * 16777619u) ^ p[i];
  return ((h >> 28) ^ h) & 0x0FFFFFFFu;
}

static inline uint64_t rd(const uint8_t* p, int w) {
  uint64_t v = 0;
  for (int i = 0; i < w; i++) v |= (uint64_t)p[i] << (8 * i);
  return v;
}
static inline void wr(uint8_t* p, uint64_t v, int w) {
  for (int i = 0; i < w; i++) p[i] = (uint8_t)(v >> (8 * i));
}
static inline uint64_t wmask(int w) { return w >= 8 ? ~0ull : ((1ull << (8 * w)) - 1); }

template <class F>
static void parallel_for(uint64_t n, int nthreads, F f) {
  if (nthreads < 1) nthreads = 1;
  if (n < 4096 || nthreads == 1) {
    f(0, n, 0);
    return;
  }
  std::vector<std::thread> th;
  uint64_t per = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; t++) {
    uint64_t lo = std::min(n, per * t), hi = std::min(n, lo + per);
    th.emplace_back([=] { f(lo, hi, t); });
  }
  for (auto& x : th) x.join();
}

// ------------------------------------------------------------------------------------ reader

// Posting record (writer Hashmap.cpp:2397-2507, reader Analyser.cpp:1631-1750):
//   [w_off, w_id, w_pos, w_num] refIDMin (w_off) refPOSMin (w_off) numIDs (w_num)
//   numIDs x (refID - refIDMin) (w_id)   w_rep (1)   numRep (w_pos)
//   numRep x (count (w_rep), pos - refPOSMin (w_pos))
// Returns the number of postings, or -1 when the record is malformed. Every width the writer
// emits is at least one byte, so a record cannot hold more postings than it has bytes left; the
// bound also keeps the sum of the counts from overflowing.
static int64_t record_count(const uint8_t* p, const uint8_t* end) {
  if (p + 4 > end) return -1;
  int wo = p[0], wnum = p[3];
  if (p + 4 + 2 * wo + wnum > end || wnum > 8 || wnum < 1) return -1;
  const uint64_t c = rd(p + 4 + 2 * wo, wnum);
  if (c > (uint64_t)(end - p) || c > 0xFFFFFFFFull) return -1;
  return (int64_t)c;
}

static bool decode_record(const uint8_t* p, const uint8_t* end, int word, uint32_t n_refs,
                          Posting* out, uint64_t num) {
  const uint64_t M = wmask(word);
  int wo = p[0], wid = p[1], wpos = p[2], wnum = p[3];
  if (wo > word || wid > word || wpos > word || wo < 1 || wid < 1 || wpos < 1) return false;
  p += 4;
  uint64_t id_min = rd(p, wo), pos_min = rd(p + wo, wo);
  p += 2 * wo + wnum;
  if (p + (uint64_t)wid * num + 1 + wpos > end) return false;
  for (uint64_t j = 0; j < num; j++) {
    uint64_t id = (rd(p + j * wid, wid) + id_min) & M;  // "raise" of Analyser.cpp:1666-1686
    if (id >= n_refs) return false;
    out[j].ref = (uint32_t)id;
  }
  p += (uint64_t)wid * num;
  int wrep = p[0];
  uint64_t nrep = rd(p + 1, wpos);
  p += 1 + wpos;
  if (wrep > word || wrep < 1 || nrep > num || p + nrep * (uint64_t)(wrep + wpos) > end) return false;
  uint64_t filled = 0;
  for (uint64_t r = 0; r < nrep; r++) {
    uint64_t c = rd(p, wrep);
    uint64_t v = (rd(p + wrep, wpos) + pos_min) & M;
    p += wrep + wpos;
    if (filled + c > num || v > 0xFFFFFFFFull) return false;
    for (uint64_t i = 0; i < c; i++) out[filled + i].pos = (uint32_t)v;
    filled += c;
  }
  // The reference pairs vSeqIDs[k] with vPos[k]; both must hold numIDs values.
  return filled == num;
}

int mhm_parse_meta(const uint8_t* b, uint64_t L, int k, MhmIndex* ix, MhmMeta* meta, bool copy_bases,
                   std::string* err) {
  auto fail = [&](int code, const char* msg) {
    if (err) *err = msg;
    return code;
  };
  const uint64_t ml = sizeof(kMagic) - 1;
  uint64_t o = 0;
  if (L < ml + 24 || std::memcmp(b, kMagic, ml) != 0) return fail(MHM_ERR_FORMAT, "not a MirAge hashmap database");
  o = ml;
  ix->n_hash = rd(b + o, 8);
  o += 8;
  int32_t version = (int32_t)rd(b + o, 4);
  int32_t word = (int32_t)rd(b + o + 4, 4);
  ix->threshold = (int32_t)rd(b + o + 8, 4);
  o += 12;
  int bsp = b[o];
  o += 4;
  if (version != kVersion) return fail(MHM_ERR_FORMAT, "unsupported hashmap version");
  if (word != 4 && word != 8) return fail(MHM_ERR_FORMAT, "unsupported hashmap bit size");
  if (bsp != word) return fail(MHM_ERR_FORMAT, "unexpected stream position width");
  // Hashmap.cpp:457-463: the configured k may not be below the one the index was built with.
  if (k < ix->threshold) return fail(MHM_ERR_FORMAT, "k is below the threshold the hashmap was built with");
  ix->word = word;
  const uint64_t n = ix->n_hash;
  const uint64_t W = (uint64_t)word;
  if (n > (L - o) / (2 * W)) return fail(MHM_ERR_FORMAT, "truncated TOC");
  if (n > 0xFFFFFFFFull) return fail(MHM_ERR_LIMIT, "too many hashes");
  meta->toc_at = o;
  o += n * 2 * W;
  // TaxIDs
  if (o + W > L) return fail(MHM_ERR_FORMAT, "truncated TaxIDs");
  uint64_t ntax = rd(b + o, word);
  o += W;
  if (ntax > (L - o) / 4) return fail(MHM_ERR_FORMAT, "truncated TaxIDs");
  ix->taxids.resize(ntax);
  for (uint64_t i = 0; i < ntax; i++) ix->taxids[i] = (int32_t)rd(b + o + 4 * i, 4);
  o += 4 * ntax;
  // sequence and header TOCs (LoadReferenceDataFromHashmapDB_SuperLazy)
  auto read_toc = [&](std::vector<uint64_t>* sizes, std::vector<uint64_t>* pos, uint64_t* count) -> bool {
    if (o + 2 * W > L) return false;
    *count = rd(b + o + W, word);
    o += 2 * W;
    if (*count > (L - o) / (2 * W)) return false;
    sizes->resize(*count);
    pos->resize(*count);
    for (uint64_t i = 0; i < *count; i++) (*sizes)[i] = rd(b + o + W * i, word);
    o += W * *count;
    for (uint64_t i = 0; i < *count; i++) (*pos)[i] = rd(b + o + W * i, word);
    o += W * *count;
    return true;
  };
  std::vector<uint64_t> ssz, spos, hsz, hpos;
  uint64_t nseq = 0, nhdr = 0;
  if (!read_toc(&ssz, &spos, &nseq)) return fail(MHM_ERR_FORMAT, "truncated sequence TOC");
  if (!read_toc(&hsz, &hpos, &nhdr)) return fail(MHM_ERR_FORMAT, "truncated header TOC");
  if (nseq > 0xFFFFFFFFull) return fail(MHM_ERR_LIMIT, "too many references");
  ix->n_refs = (uint32_t)nseq;
  ix->ref_len.resize(nseq);
  ix->ref_off.resize(nseq);
  meta->bases_at = meta->bases_len = 0;
  if (nseq) {
    uint64_t first = spos[0];
    uint64_t last_end = spos[nseq - 1] + ssz[nseq - 1];
    if (last_end > L || first > last_end) return fail(MHM_ERR_FORMAT, "truncated reference bases");
    for (uint64_t r = 0; r < nseq; r++) {
      if (ssz[r] > 0xFFFFFFFFull || spos[r] < first || spos[r] + ssz[r] > last_end)
        return fail(MHM_ERR_FORMAT, "bad reference position");
      ix->ref_len[r] = (uint32_t)ssz[r];
      ix->ref_off[r] = spos[r] - first;
    }
    meta->bases_at = first;
    meta->bases_len = last_end - first;
    if (copy_bases) ix->bases.assign(b + first, b + last_end);
  }
  ix->headers.resize(nhdr);
  for (uint64_t r = 0; r < nhdr; r++) {
    if (hpos[r] + hsz[r] > L) return fail(MHM_ERR_FORMAT, "truncated headers");
    uint64_t len = hsz[r];
    if (len && b[hpos[r] + len - 1] == 0) len--;
    ix->headers[r].assign((const char*)b + hpos[r], len);
  }
  return MHM_OK;
}

int mhm_parse(const uint8_t* b, uint64_t L, int k, int nthreads, MhmIndex* ix, std::string* err) {
  auto fail = [&](int code, const char* msg) {
    if (err) *err = msg;
    return code;
  };
  MhmMeta meta;
  int rc = mhm_parse_meta(b, L, k, ix, &meta, true, err);
  if (rc) return rc;
  const uint64_t n = ix->n_hash;
  const int word = ix->word;
  const uint64_t W = (uint64_t)word;
  ix->toc_hash.resize(n);
  std::vector<uint64_t> sp(n);
  for (uint64_t i = 0, o = meta.toc_at; i < n; i++, o += 2 * W) {
    uint64_t h = rd(b + o, word);
    if (h > 0x0FFFFFFFull) return fail(MHM_ERR_FORMAT, "hash wider than 28 bits");
    // the device directory needs the TOC ascending, as the builder writes it
    if (i && h <= ix->toc_hash[i - 1]) return fail(MHM_ERR_FORMAT, "TOC hashes not strictly ascending");
    ix->toc_hash[i] = (uint32_t)h;
    sp[i] = rd(b + o + W, word);
  }
  // posting records: BufferSize = next stream position - this one; the value computed for the
  // last TOC entry is written one past the array (Hashmap.cpp:552-553), so the last hash is
  // present in the lookup table with BufferSize 0 and its record is never decoded
  // (Analyser.cpp:1613).
  std::vector<uint64_t> cnt(n + 1, 0);
  std::atomic<int> bad(0);
  const uint8_t* end = b + L;
  parallel_for(n, nthreads, [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t i = lo; i < hi; i++) {
      if (i + 1 == n) continue;
      if (sp[i] >= L || sp[i + 1] <= sp[i]) { bad = 1; continue; }
      int64_t c = record_count(b + sp[i], end);
      if (c < 0) { bad = 1; continue; }
      cnt[i] = (uint64_t)c;
    }
  });
  if (bad) return fail(MHM_ERR_FORMAT, "malformed posting record");
  ix->bucket.assign(n + 1, 0);
  for (uint64_t i = 0; i < n; i++) ix->bucket[i + 1] = ix->bucket[i] + cnt[i];
  uint64_t total = ix->bucket[n];
  try {
    ix->postings.resize(total);
  } catch (...) {
    return fail(MHM_ERR_OOM, "out of host memory for postings");
  }
  parallel_for(n, nthreads, [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t i = lo; i < hi; i++) {
      if (cnt[i] == 0) continue;
      if (!decode_record(b + sp[i], end, word, ix->n_refs, ix->postings.data() + ix->bucket[i], cnt[i])) bad = 1;
    }
  });
  if (bad) return fail(MHM_ERR_FORMAT, "malformed posting record");
  ix->has_empty_last = n > 0;
  ix->empty_last_hash = n > 0 ? ix->toc_hash[n - 1] : 0;
  return MHM_OK;
}

int mhm_load(const std::string& path, int k, int nthreads, MhmIndex* out, std::string* err) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    if (err) *err = "cannot open " + path;
    return MHM_ERR_IO;
  }
  uint64_t len = (uint64_t)f.tellg();
  f.seekg(0);
  std::vector<uint8_t> buf;
  try {
    buf.resize(len);
  } catch (...) {
    return MHM_ERR_OOM;
  }
  if (!f.read((char*)buf.data(), (std::streamsize)len)) {
    if (err) *err = "read error on " + path;
    return MHM_ERR_IO;
  }
  return mhm_parse(buf.data(), len, k, nthreads, out, err);
}

// ------------------------------------------------------------------------------------ writer

// Byte width of a value as the writer computes it: ((countBits(v) - 1) / 8) + 1 with C
// integer division, so 0 takes one byte (Hashmap.cpp:1534-1546, 1641-1671).
static int width_of(uint64_t v) {
  int bits = 0;
  while (v) {
    bits++;
    v >>= 1;
  }
  return ((bits - 1) / 8) + 1;
}

struct Group {
  uint64_t first;  // into the sorted entry arrays
  uint32_t n;
  uint32_t hash;
};

int mhm_width_of(uint64_t v) { return width_of(v); }

int mhm_plan(const uint64_t* offs, uint32_t n_refs, const std::vector<std::string>& headers, int word,
             uint64_t ng, uint64_t rec_total, uint64_t last_rec, MhmPlan* plan, std::string* err) {
  uint64_t seq_chars = offs[n_refs] - offs[0], hdr_chars = 0;
  for (uint32_t r = 0; r < n_refs; r++) hdr_chars += headers[r].size() + 2;  // '>' + name + NUL
  const uint64_t ml = sizeof(kMagic) - 1;
  auto layout = [&](uint64_t W, uint64_t* toc_at) {
    uint64_t sp = ml + 8 + 4 + 4 + 4 + 4;
    *toc_at = sp;
    sp += ng * W * 2;
    sp += W + W + n_refs * W + W + n_refs * W + W;
    sp += W + n_refs * 4ull + n_refs * W + n_refs * W;
    sp += seq_chars + hdr_chars;
    return sp;  // the first record
  };
  uint64_t toc_at;
  if (word == 0) word = (layout(4, &toc_at) + rec_total > 0xFFFFFFFFull) ? 8 : 4;
  if (word != 4 && word != 8) {
    if (err) *err = "word must be 4 or 8";
    return MHM_ERR_LIMIT;
  }
  plan->W = (uint64_t)word;
  plan->first_rec = layout(plan->W, &plan->toc_at);
  plan->total = plan->first_rec + rec_total;
  // the 32-bit build refuses files whose positions pass 2^32-1 (Hashmap.cpp:2103-2109)
  if (plan->W == 4 && plan->total - last_rec > 0xFFFFFFFFull) {
    if (err) *err = "file too large for the 32-bit format; use word 8";
    return MHM_ERR_LIMIT;
  }
  return MHM_OK;
}

int mhm_write_head(uint8_t* b, const MhmPlan& plan, const uint8_t* bases, const uint64_t* offs, uint32_t n_refs,
                   const std::vector<std::string>& headers, const std::vector<int32_t>& taxids, int k, uint64_t ng,
                   uint32_t max_group, std::string* err) {
  const uint64_t W = plan.W;
  const int Wi = (int)W;
  uint64_t max_ref = 0, max_hdr = 0;
  for (uint32_t r = 0; r < n_refs; r++) {
    max_hdr = std::max<uint64_t>(max_hdr, headers[r].size() + 2);
    max_ref = std::max<uint64_t>(max_ref, offs[r + 1] - offs[r]);
  }
  const uint64_t ml = sizeof(kMagic) - 1;
  uint64_t o = 0;
  std::memcpy(b, kMagic, ml);
  o = ml;
  wr(b + o, ng, 8);
  o += 8;
  wr(b + o, kVersion, 4);
  wr(b + o + 4, W, 4);
  wr(b + o + 8, (uint64_t)(uint32_t)k, 4);
  o += 12;
  b[o] = (uint8_t)W;
  b[o + 1] = (uint8_t)width_of(max_group);
  b[o + 2] = (uint8_t)width_of(max_ref);
  b[o + 3] = (uint8_t)width_of(max_hdr);
  o += 4;
  if (o != plan.toc_at) {
    if (err) *err = "internal layout mismatch";
    return MHM_ERR_FORMAT;
  }
  o += ng * 2 * W;  // bucket TOC: written by the caller
  wr(b + o, n_refs, Wi);
  o += W;
  for (uint32_t r = 0; r < n_refs; r++) wr(b + o + 4ull * r, (uint32_t)(r < taxids.size() ? taxids[r] : -1), 4);
  o += 4ull * n_refs;
  // sequence TOC
  uint64_t seq_chars = offs[n_refs] - offs[0];
  uint64_t after = o + W + W + n_refs * W + n_refs * W;
  const uint64_t seq_start = after + W + W + n_refs * W + n_refs * W;
  wr(b + o, after, Wi);
  wr(b + o + W, n_refs, Wi);
  o += 2 * W;
  for (uint32_t r = 0; r < n_refs; r++) wr(b + o + W * r, offs[r + 1] - offs[r], Wi);
  o += W * n_refs;
  uint64_t spx = seq_start;
  for (uint32_t r = 0; r < n_refs; r++) {
    wr(b + o + W * r, spx, Wi);
    spx += offs[r + 1] - offs[r];
  }
  o += W * n_refs;
  // header TOC
  after = o + W + W + n_refs * W + n_refs * W;
  wr(b + o, after, Wi);
  wr(b + o + W, n_refs, Wi);
  o += 2 * W;
  for (uint32_t r = 0; r < n_refs; r++) wr(b + o + W * r, headers[r].size() + 2, Wi);
  o += W * n_refs;
  for (uint32_t r = 0; r < n_refs; r++) {
    wr(b + o + W * r, spx, Wi);
    spx += headers[r].size() + 2;
  }
  o += W * n_refs;
  if (o != seq_start) {
    if (err) *err = "internal layout mismatch";
    return MHM_ERR_FORMAT;
  }
  std::memcpy(b + o, bases + offs[0], seq_chars);
  o += seq_chars;
  for (uint32_t r = 0; r < n_refs; r++) {
    b[o++] = '>';
    std::memcpy(b + o, headers[r].data(), headers[r].size());
    o += headers[r].size();
    b[o++] = 0;
  }
  if (o != plan.first_rec) {
    if (err) *err = "internal layout mismatch";
    return MHM_ERR_FORMAT;
  }
  return MHM_OK;
}

int mhm_build(const uint8_t* bases, const uint64_t* offs, uint32_t n_refs,
              const std::vector<std::string>& headers, const std::vector<int32_t>& taxids, int k,
              int word, int nthreads, std::vector<uint8_t>* out, std::string* err) {
  auto fail = [&](int code, const std::string& msg) {
    if (err) *err = msg;
    return code;
  };
  if (k < 2) return fail(MHM_ERR_LIMIT, "k too small");
  if (headers.size() != n_refs) return fail(MHM_ERR_LIMIT, "one header per reference required");
  const uint32_t step = (uint32_t)k / 2;
  const int hlen = k - (int)step + 1;  // Hashmap.cpp:2790
  const bool trace = std::getenv("MG_BUILD_TRACE") != nullptr;
  auto t_start = std::chrono::steady_clock::now();
  auto phase = [&](const char* what) {
    if (trace)
      std::fprintf(stderr, "[mhm_build] %-12s %.3f s\n", what,
                   std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count());
  };
  std::string nn(hlen, 'N');
  const uint32_t h_nnn = hash28((const uint8_t*)nn.data(), hlen);
  // 1. hash every indexed position of every reference (TBuildHashmapForReference,
  // Hashmap.cpp:2771-2906): positions i < len - hlen; a window hashing to the all-N hash is
  // skipped and the read pointer is then NOT advanced, so later windows lag behind i.
  std::vector<uint64_t> ref_first(n_refs + 1, 0);
  for (uint32_t r = 0; r < n_refs; r++) {
    uint64_t len = offs[r + 1] - offs[r];
    if (len <= (uint64_t)hlen) return fail(MHM_ERR_LIMIT, "reference shorter than the hash window");
    if (len > 0xFFFFFFFFull) return fail(MHM_ERR_LIMIT, "reference longer than 2^32");
    ref_first[r + 1] = ref_first[r] + (len - hlen);
  }
  const uint64_t npos = ref_first[n_refs];
  std::vector<uint32_t> ph(npos), pref(npos), ppos(npos);
  std::vector<uint64_t> kept_per_ref(n_refs, 0);
  {
    std::atomic<uint32_t> next(0);
    std::vector<std::thread> th;
    int nt = std::max(1, nthreads);
    for (int t = 0; t < nt; t++)
      th.emplace_back([&] {
        for (;;) {
          uint32_t r = next.fetch_add(1);
          if (r >= n_refs) break;
          const uint8_t* s = bases + offs[r];
          uint64_t istop = (offs[r + 1] - offs[r]) - hlen;
          uint64_t w = ref_first[r];
          const uint8_t* p = s;
          for (uint64_t i = 0; i < istop; i++) {
            uint32_t h = hash28(p, hlen);
            if (h == h_nnn) continue;
            ph[w] = h;
            pref[w] = r;
            ppos[w] = (uint32_t)i;
            w++;
            p++;
          }
          kept_per_ref[r] = w - ref_first[r];
        }
      });
    for (auto& x : th) x.join();
  }
  // compact the per-reference ranges (all-N windows leave holes)
  uint64_t m = 0;
  for (uint32_t r = 0; r < n_refs; r++) {
    uint64_t a = ref_first[r], c = kept_per_ref[r];
    if (a != m) {
      std::memmove(&ph[m], &ph[a], c * 4);
      std::memmove(&pref[m], &pref[a], c * 4);
      std::memmove(&ppos[m], &ppos[a], c * 4);
    }
    m += c;
  }
  phase("hashed");
  // 2. group by hash: partition on the top 20 hash bits, then sort every partition by
  // (hash, position, refID). The reference sorts a bucket by position only with std::sort
  // (Hashmap.cpp:1566), leaving equal positions in an unspecified order; readers treat every
  // such order alike.
  struct Ent {
    uint64_t hp;   // hash << 32 | position
    uint32_t ref;
    bool operator<(const Ent& o) const { return hp != o.hp ? hp < o.hp : ref < o.ref; }
  };
  const int PB = 20;
  const uint64_t NP = 1ull << PB;
  std::vector<Ent> ent;
  std::vector<uint64_t> pstart(NP + 1, 0);
  {
    std::vector<std::atomic<uint64_t>> pc(NP);
    for (auto& x : pc) x.store(0, std::memory_order_relaxed);
    parallel_for(m, std::max(1, nthreads), [&](uint64_t lo, uint64_t hi, int) {
      for (uint64_t i = lo; i < hi; i++) pc[ph[i] >> (28 - PB)].fetch_add(1, std::memory_order_relaxed);
    });
    phase("histogram");
    for (uint64_t p = 0; p < NP; p++) pstart[p + 1] = pstart[p] + pc[p].load(std::memory_order_relaxed);
    for (uint64_t p = 0; p < NP; p++) pc[p].store(pstart[p], std::memory_order_relaxed);
    try {
      ent.resize(m);
    } catch (...) {
      return fail(MHM_ERR_OOM, "out of host memory for the build");
    }
    parallel_for(m, std::max(1, nthreads), [&](uint64_t lo, uint64_t hi, int) {
      for (uint64_t i = lo; i < hi; i++) {
        uint64_t at = pc[ph[i] >> (28 - PB)].fetch_add(1, std::memory_order_relaxed);
        ent[at] = Ent{((uint64_t)ph[i] << 32) | ppos[i], pref[i]};
      }
    });
  }
  phase("scattered");
  std::vector<uint32_t>().swap(ph);
  std::vector<uint32_t>().swap(pref);
  std::vector<uint32_t>().swap(ppos);
  parallel_for(NP, std::max(1, nthreads), [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t p = lo; p < hi; p++)
      if (pstart[p + 1] - pstart[p] > 1) std::sort(ent.begin() + pstart[p], ent.begin() + pstart[p + 1]);
  });
  phase("sorted");
  std::vector<Group> groups;
  uint32_t max_group = 0;
  for (uint64_t i = 0; i < m;) {
    uint64_t j = i + 1;
    const uint32_t h = (uint32_t)(ent[i].hp >> 32);
    while (j < m && (uint32_t)(ent[j].hp >> 32) == h) j++;
    groups.push_back(Group{i, (uint32_t)(j - i), h});
    max_group = std::max<uint32_t>(max_group, (uint32_t)(j - i));
    i = j;
  }
  // per-entry (position << 32 | refID) in group order, the form the encoder reads
  std::vector<uint64_t> sorted_rp(m);
  parallel_for(m, std::max(1, nthreads), [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t i = lo; i < hi; i++) sorted_rp[i] = ((ent[i].hp & 0xFFFFFFFFull) << 32) | ent[i].ref;
  });
  std::vector<Ent>().swap(ent);
  // EnableFragmentedDatabase (k < 20, Hashmap.cpp:1759-1840): drop the buckets larger than
  // min(20, the 30th-percentile bucket size).
  if (k < 20 && !groups.empty()) {
    std::vector<uint32_t> sz(groups.size());
    for (size_t g = 0; g < groups.size(); g++) sz[g] = groups[g].n;
    std::sort(sz.begin(), sz.end());
    size_t idx = (size_t)((sz.size() / 100.0) * 30);
    uint32_t thr = std::min<uint32_t>(20, sz[idx]);
    std::vector<Group> kept;
    max_group = 0;
    for (auto& g : groups)
      if (g.n <= thr) {
        kept.push_back(g);
        max_group = std::max(max_group, g.n);
      }
    groups.swap(kept);
  }
  const uint64_t ng = groups.size();
  phase("grouped");
  // 3. per-record widths and sizes (GetSaveHashmapPreCalculates, Hashmap.cpp:1619-1697)
  std::vector<uint64_t> rec_size(ng);
  std::atomic<int> too_wide(0);
  parallel_for(ng, std::max(1, nthreads), [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t g = lo; g < hi; g++) {
      const uint64_t* e = &sorted_rp[groups[g].first];
      uint32_t n = groups[g].n;
      uint32_t idmin = UINT32_MAX, idmax = 0;
      for (uint32_t i = 0; i < n; i++) {
        uint32_t id = (uint32_t)e[i];
        idmin = std::min(idmin, id);
        idmax = std::max(idmax, id);
      }
      uint32_t pmin = (uint32_t)(e[0] >> 32), pmax = (uint32_t)(e[n - 1] >> 32);
      int wid = width_of(idmax - idmin), wpos = width_of(pmax - pmin);
      int wo = width_of(std::max(idmin, pmin)), wnum = width_of(n), wrep = width_of(n);
      uint64_t nrep = 1;
      for (uint32_t i = 1; i < n; i++) nrep += (e[i] >> 32) != (e[i - 1] >> 32);
      // the writer stores the repeat count in w_pos bytes; a count that does not fit would be
      // truncated and make the record unreadable, so refuse to write it
      if (wpos < 8 && nrep > wmask(wpos)) too_wide = 1;
      rec_size[g] = 4 + 2ull * wo + wnum + (uint64_t)wid * n + 1 + wpos + nrep * (uint64_t)(wrep + wpos);
    }
  });
  if (too_wide) return fail(MHM_ERR_LIMIT, "a bucket has more distinct positions than its width can count");
  phase("sized");
  // 4. layout and stream positions (SaveHashmapTableV3, Hashmap.cpp:1868-2128)
  uint64_t rec_total = 0;
  for (uint64_t g = 0; g < ng; g++) rec_total += rec_size[g];
  MhmPlan plan;
  int prc = mhm_plan(offs, n_refs, headers, word, ng, rec_total, ng ? rec_size[ng - 1] : 0, &plan, err);
  if (prc) return prc;
  const uint64_t W = plan.W;
  phase("planned");
  try {
    out->assign(plan.total, 0);
  } catch (...) {
    return fail(MHM_ERR_OOM, "out of host memory for the image");
  }
  phase("allocated");
  uint8_t* b = out->data();
  prc = mhm_write_head(b, plan, bases, offs, n_refs, headers, taxids, k, ng, max_group, err);
  if (prc) return prc;
  std::vector<uint64_t> rec_sp(ng + 1);
  rec_sp[0] = plan.first_rec;
  for (uint64_t g = 0; g < ng; g++) rec_sp[g + 1] = rec_sp[g] + rec_size[g];
  for (uint64_t g = 0, o = plan.toc_at; g < ng; g++, o += 2 * W) {
    wr(b + o, groups[g].hash, (int)W);
    wr(b + o + W, rec_sp[g], (int)W);
  }
  phase("laid out");
  // 5. posting records (Hashmap.cpp:2303-2512)
  parallel_for(ng, std::max(1, nthreads), [&](uint64_t lo, uint64_t hi, int) {
    for (uint64_t g = lo; g < hi; g++) {
      const uint64_t* e = &sorted_rp[groups[g].first];
      uint32_t n = groups[g].n;
      uint32_t idmin = UINT32_MAX, idmax = 0;
      for (uint32_t i = 0; i < n; i++) {
        idmin = std::min(idmin, (uint32_t)e[i]);
        idmax = std::max(idmax, (uint32_t)e[i]);
      }
      uint32_t pmin = (uint32_t)(e[0] >> 32), pmax = (uint32_t)(e[n - 1] >> 32);
      int wid = width_of(idmax - idmin), wpos = width_of(pmax - pmin);
      int wo = width_of(std::max(idmin, pmin)), wnum = width_of(n), wrep = width_of(n);
      uint8_t* p = b + rec_sp[g];
      p[0] = (uint8_t)wo;
      p[1] = (uint8_t)wid;
      p[2] = (uint8_t)wpos;
      p[3] = (uint8_t)wnum;
      p += 4;
      wr(p, idmin, wo);
      wr(p + wo, pmin, wo);
      wr(p + 2 * wo, n, wnum);
      p += 2 * wo + wnum;
      for (uint32_t i = 0; i < n; i++) {
        wr(p, (uint32_t)e[i] - idmin, wid);
        p += wid;
      }
      uint64_t nrep = 1;
      for (uint32_t i = 1; i < n; i++) nrep += (e[i] >> 32) != (e[i - 1] >> 32);
      *p++ = (uint8_t)wrep;
      wr(p, nrep, wpos);
      p += wpos;
      uint32_t i0 = 0;
      for (uint32_t i = 1; i <= n; i++) {
        if (i == n || (e[i] >> 32) != (e[i - 1] >> 32)) {
          wr(p, i - i0, wrep);
          wr(p + wrep, (uint32_t)(e[i0] >> 32) - pmin, wpos);
          p += wrep + wpos;
          i0 = i;
        }
      }
    }
  });
  phase("encoded");
  return MHM_OK;
}

}  // namespace mg
