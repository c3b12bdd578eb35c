/*
 * TEST INFRASTRUCTURE ONLY -- CPU restatement of MirAge's classification hot path, written
 * from the reference's behaviour (cited per function below). It is the checker for the CUDA
 * path and the reported CPU baseline; the product never links it.
 *
 * Parity pin: the dumps under tests/golden/ were produced by the unmodified reference CPU path
 * (oracle/ref_harness.cpp over the reference's own objects) and tests/test_oracle_golden.py
 * checks this file against them field by field (candidates, runs, Score/percentageMatch/
 * relative-score float bits, merged result and top group).
 *
 * Single .mhm file, 32-bit build (HASH_t = SEQ_ID_t = SEQ_POS_t = uint32, Enum.h:10-15) or the
 * -D__Hash64__ build (all uint64, Enum.h:16-21; values here must still fit 32 bits),
 * memory mode "extreme", speed mode "Sensitive", reverse complements on.
 */
#define _GNU_SOURCE
#include "mg_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define E_IO (-1)
#define E_FMT (-2)
#define E_OOM (-3)
#define E_INPUT (-4)

static const char MHM_MAGIC[] =
    "MirAge - Maarten Pater - www.mirdesign.nl - mirage@mirdesign.nl - Hashmap";

struct mgo_index {
  int k;
  uint8_t* file;
  uint64_t file_len;
  uint64_t n_hash;
  int word;              /* LoadedBytes: 4, or 8 with -D__Hash64__ */
  uint32_t* toc_hash;    /* file order */
  uint64_t* toc_sp;      /* stream position of the posting record */
  uint64_t* toc_size;    /* BufferSize as the reader computes it (last entry 0) */
  uint32_t* sorted;      /* TOC indices sorted by hash, for lookup */
  uint32_t n_refs;
  uint32_t* ref_size;
  uint64_t* ref_off;     /* offset of each reference in seq[] */
  const uint8_t* seq;    /* sequence block (referenceSequences_Buffer) */
  const uint8_t* pos_data;
  uint64_t pos_first_sp;
};

/* ---------------------------------------------------------------- hashing (A1) */

/* CreateHash32 (Hashmap.cpp:3197-3210): FNV-1 style, multiply then xor, 32-bit wrap. */
static uint32_t hash32(const uint8_t* p, int len) {
  uint32_t h = 2166136261u;
  for (int i = 0; i < len; i++) h = (h * 16777619u) ^ p[i];
  return h;
}

/* CreateHash24 (Hashmap.cpp:3233-3268) with HashBits = 28 (Hashmap.h:111). */
uint32_t mgo_hash28(const uint8_t* p, int len) {
  uint32_t h = hash32(p, len);
  return ((h >> 28) ^ h) & 0x0FFFFFFFu;
}

/* ---------------------------------------------------------------- .mhm reader */

static uint64_t rd_le(const uint8_t* p, int w) {
  uint64_t v = 0;
  for (int i = 0; i < w; i++) v |= (uint64_t)p[i] << (8 * i);
  return v;
}

static const mgo_index* g_sort_ix;
static int cmp_toc(const void* a, const void* b) {
  uint32_t ha = g_sort_ix->toc_hash[*(const uint32_t*)a], hb = g_sort_ix->toc_hash[*(const uint32_t*)b];
  return ha < hb ? -1 : ha > hb ? 1 : 0;
}

void mgo_close(mgo_index* ix) {
  if (!ix) return;
  free(ix->file);
  free(ix->toc_hash);
  free(ix->toc_sp);
  free(ix->toc_size);
  free(ix->sorted);
  free(ix->ref_size);
  free(ix->ref_off);
  free(ix);
}

/* Hashmap::LoadHashMapFromHashmapDB (Hashmap.cpp:402-580), LoadReferenceDataFromHashmapDB_
 * SuperLazy (:629-660) and the extreme-mode slurps (:258-306). */
int mgo_open(const char* path, int k, mgo_index** out) {
  *out = NULL;
  FILE* f = fopen(path, "rb");
  if (!f) return E_IO;
  fseek(f, 0, SEEK_END);
  long len = ftell(f);
  fseek(f, 0, SEEK_SET);
  mgo_index* ix = (mgo_index*)calloc(1, sizeof(mgo_index));
  if (!ix) { fclose(f); return E_OOM; }
  ix->k = k;
  ix->file = (uint8_t*)malloc((size_t)len + 16);
  if (!ix->file || fread(ix->file, 1, (size_t)len, f) != (size_t)len) {
    fclose(f);
    mgo_close(ix);
    return E_IO;
  }
  fclose(f);
  ix->file_len = (uint64_t)len;
  const uint8_t* b = ix->file;
  uint64_t o = 0, L = ix->file_len;
  size_t ml = strlen(MHM_MAGIC);
#define NEED(n) do { if (o + (uint64_t)(n) > L) { mgo_close(ix); return E_FMT; } } while (0)
  NEED(ml + 8 + 12 + 4);
  if (memcmp(b, MHM_MAGIC, ml) != 0) { mgo_close(ix); return E_FMT; }
  o = ml;
  ix->n_hash = rd_le(b + o, 8); o += 8;
  int32_t version = (int32_t)rd_le(b + o, 4); o += 4;
  int32_t loaded_bytes = (int32_t)rd_le(b + o, 4); o += 4;
  int32_t threshold = (int32_t)rd_le(b + o, 4); o += 4;
  int bsp = b[o];
  o += 4;
  /* version 4 (Hashmap.h:252); LoadedBytes 4 (32-bit build) or 8 (-D__Hash64__ build); k not
   * below the build threshold (:457) */
  if (version != 4 || (loaded_bytes != 4 && loaded_bytes != 8) || bsp != loaded_bytes || k < threshold) {
    mgo_close(ix);
    return E_FMT;
  }
  const int W = loaded_bytes;
  ix->word = W;
  uint64_t n = ix->n_hash;
  NEED(n * 2 * W);
  ix->toc_hash = (uint32_t*)malloc(n * 4 + 4);
  ix->toc_sp = (uint64_t*)malloc(n * 8 + 8);
  ix->toc_size = (uint64_t*)malloc(n * 8 + 8);
  ix->sorted = (uint32_t*)malloc(n * 4 + 4);
  if (!ix->toc_hash || !ix->toc_sp || !ix->toc_size || !ix->sorted) { mgo_close(ix); return E_OOM; }
  for (uint64_t i = 0; i < n; i++) {
    ix->toc_hash[i] = (uint32_t)rd_le(b + o, W);
    ix->toc_sp[i] = rd_le(b + o + W, W);
    o += 2 * W;
  }
  /* BufferSize: next stream position minus this one; the entry written for the last hash
   * lands one past the array (Hashmap.cpp:552-553), so the last hash keeps 0 and is treated
   * as present with no postings. */
  for (uint64_t i = 0; i < n; i++) ix->toc_size[i] = (i + 1 < n) ? ix->toc_sp[i + 1] - ix->toc_sp[i] : 0;
  for (uint64_t i = 0; i < n; i++) ix->sorted[i] = (uint32_t)i;
  g_sort_ix = ix;
  qsort(ix->sorted, n, 4, cmp_toc);
  ix->pos_first_sp = n ? ix->toc_sp[0] : 0;
  /* NCBI TaxIDs */
  NEED(W);
  uint64_t ntax = rd_le(b + o, W); o += W;
  NEED(ntax * 4);
  o += ntax * 4;
  /* sequences TOC */
  NEED(2 * W);
  o += W; /* spGoto */
  ix->n_refs = (uint32_t)rd_le(b + o, W); o += W;
  uint32_t nr = ix->n_refs;
  NEED((uint64_t)nr * 2 * W);
  ix->ref_size = (uint32_t*)malloc((uint64_t)nr * 4 + 4);
  ix->ref_off = (uint64_t*)malloc((uint64_t)nr * 8 + 8);
  if (!ix->ref_size || !ix->ref_off) { mgo_close(ix); return E_OOM; }
  for (uint32_t r = 0; r < nr; r++) ix->ref_size[r] = (uint32_t)rd_le(b + o + (uint64_t)W * r, W);
  o += (uint64_t)W * nr;
  uint64_t first_sp = nr ? rd_le(b + o, W) : 0;
  for (uint32_t r = 0; r < nr; r++) ix->ref_off[r] = rd_le(b + o + (uint64_t)W * r, W) - first_sp;
  o += (uint64_t)W * nr;
  if (nr && first_sp + ix->ref_off[nr - 1] + ix->ref_size[nr - 1] > L) { mgo_close(ix); return E_FMT; }
  ix->seq = b + first_sp;
  if (ix->pos_first_sp > L) { mgo_close(ix); return E_FMT; }
  ix->pos_data = b + ix->pos_first_sp;
#undef NEED
  *out = ix;
  return 0;
}

uint32_t mgo_n_refs(const mgo_index* ix) { return ix->n_refs; }
uint32_t mgo_ref_size(const mgo_index* ix, uint32_t r) { return r < ix->n_refs ? ix->ref_size[r] : 0; }
uint64_t mgo_n_hashes(const mgo_index* ix) { return ix->n_hash; }
void mgo_free(void* p) { free(p); }

/* TOC lookup: index into the TOC, or -1 when the hash is absent (unordered_map::find,
 * Analyser.cpp:1504). */
static int64_t toc_find(const mgo_index* ix, uint32_t h) {
  uint64_t lo = 0, hi = ix->n_hash;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (ix->toc_hash[ix->sorted[mid]] < h) lo = mid + 1;
    else hi = mid;
  }
  if (lo < ix->n_hash && ix->toc_hash[ix->sorted[lo]] == h) return ix->sorted[lo];
  return -1;
}

/* ---------------------------------------------------------------- growable scratch */

typedef struct { uint32_t ref, pos; } post_t;
typedef struct { uint32_t ref, rpos, qpos; } trip_t;

typedef struct {
  post_t* post; uint64_t post_cap;
  uint32_t* found_p; uint32_t* found_off; uint32_t* found_cnt; uint64_t found_cap;
  int32_t* occ; int32_t* occmax; int32_t* last; uint64_t occ_cap;
  trip_t* trip; uint64_t trip_cap;
  uint8_t* hit; uint64_t hit_cap;
  uint32_t* rep_cnt; uint32_t* rep_pos; uint64_t rep_cap;
  /* outputs of one strand */
  mgo_cand* cand; uint64_t cand_n, cand_cap;
  mgo_run* run; uint64_t run_n, run_cap;
} ws_t;

#define GROW(ptr, cap, need, T)                                           \
  do {                                                                    \
    if ((uint64_t)(need) > (cap)) {                                       \
      uint64_t nc = (cap) ? (cap) : 64;                                   \
      while (nc < (uint64_t)(need)) nc *= 2;                              \
      void* np = realloc((ptr), nc * sizeof(T));                          \
      if (!np) return E_OOM;                                              \
      (ptr) = (T*)np;                                                     \
      (cap) = nc;                                                         \
    }                                                                     \
  } while (0)

/* Posting-record decode (Analyser.cpp:1613-1750, extreme/high mode): appends the bucket's
 * (refID, pos) pairs to ws->post. Returns the number of entries or a negative error. */
static int64_t decode(const mgo_index* ix, int64_t t, ws_t* ws, uint64_t at) {
  if (ix->toc_size[t] == 0) return 0; /* skipped, Analyser.cpp:1613 */
  uint64_t off = (uint64_t)ix->toc_sp[t] - ix->pos_first_sp;
  const uint8_t* p = ix->pos_data + off;
  const uint8_t* end = ix->file + ix->file_len;
  if (p + 4 > end) return E_FMT;
  int wo = p[0], wid = p[1], wpos = p[2], wnum = p[3];
  p += 4;
  const int W = ix->word;
  const uint64_t M = W >= 8 ? ~0ull : ((1ull << (8 * W)) - 1);
  if (wo > W || wid > W || wpos > W || wnum > 8 || p + 2 * wo + wnum > end) return E_FMT;
  uint64_t id_min = rd_le(p, wo);
  uint64_t pos_min = rd_le(p + wo, wo);
  uint64_t num = rd_le(p + 2 * wo, wnum);
  p += 2 * wo + wnum;
  if (p + (uint64_t)wid * num + 1 + wpos > end) return E_FMT;
  GROW(ws->post, ws->post_cap, at + num, post_t);
  uint64_t raise = id_min; /* + MultipleHashmaps_SequenceOffset[0] == 0 for one file */
  for (uint64_t j = 0; j < num; j++) {
    uint64_t id = (rd_le(p + (uint64_t)j * wid, wid) + raise) & M;
    if (id >= ix->n_refs) return E_FMT;
    ws->post[at + j].ref = (uint32_t)id;
  }
  p += (uint64_t)wid * num;
  int wrep = p[0];
  uint64_t nrep = rd_le(p + 1, wpos);
  p += 1 + wpos;
  if (wrep > W || p + nrep * (uint64_t)(wrep + wpos) > end) return E_FMT;
  uint64_t filled = 0;
  for (uint64_t r = 0; r < nrep; r++) {
    uint64_t c = rd_le(p, wrep);
    uint64_t v = (rd_le(p + wrep, wpos) + pos_min) & M;
    p += wrep + wpos;
    if (filled + c > num || v > 0xFFFFFFFFull) return E_FMT; /* run-lengths cover numIDs */
    for (uint64_t i = 0; i < c; i++) ws->post[at + filled + i].pos = (uint32_t)v;
    filled += c;
  }
  if (filled != num) return E_FMT;
  return (int64_t)num;
}

static int cmp_trip(const void* a, const void* b) {
  const trip_t* x = (const trip_t*)a;
  const trip_t* y = (const trip_t*)b;
  if (x->ref != y->ref) return x->ref < y->ref ? -1 : 1;
  if (x->rpos != y->rpos) return x->rpos < y->rpos ? -1 : 1;
  if (x->qpos != y->qpos) return x->qpos < y->qpos ? -1 : 1;
  return 0;
}

float mgo_relative_score(float query_len, float ref_len, float score) {
  /* MatrixResult::GetRelativeScore, MatrixResult.cpp:21-29 */
  const float len_max = (float)(query_len < ref_len ? query_len : ref_len);
  const float score_max = (float)((((double)len_max * ((double)len_max + 1.0)) / 2.0) / (double)len_max + 1);
  score += 1;
  return logf(score) / logf(score_max);
}

void mgo_logf_bits(uint32_t lo_bits, uint64_t n, float* out) {
  for (uint64_t i = 0; i < n; i++) {
    uint32_t b = lo_bits + (uint32_t)i;
    float x;
    memcpy(&x, &b, 4);
    out[i] = logf(x);
  }
}

/* CalculateScore (MatrixCPU.cpp:18-214) for one candidate with its runs. */
static void calculate_score(const mgo_index* ix, const uint8_t* q, uint32_t L, uint32_t ref,
                            const mgo_run* runs, uint32_t n_runs, uint8_t* hit, float* out_score,
                            float* out_pct) {
  const uint64_t k = (uint64_t)ix->k;
  *out_score = -2;
  *out_pct = 0;
  if (n_runs == 0) return;
  const uint8_t* rs = ix->seq + ix->ref_off[ref];
  const uint64_t rsize = ix->ref_size[ref];
  uint64_t sum_r = 0, sum_c = 0;
  memset(hit, 0, L);
  for (uint32_t i = 0; i < n_runs; i++) {
    const mgo_run* r = &runs[i];
    uint64_t row_start = r->start_q, row_end = r->last_q;
    if (row_start > row_end) continue;
    uint64_t mid = row_end - row_start;
    /* tail: walk right from Last while bases agree (MatrixCPU.cpp:93-112) */
    uint64_t tail_size = rsize - r->last_ref;      /* size_t arithmetic as in :83 */
    if (k < tail_size) tail_size = k;
    uint64_t tail = 0, row = row_end, cref = r->last_ref;
    while (!(row >= L || cref >= rsize || tail >= tail_size)) {
      if (q[row] != rs[r->last_ref + tail]) break;
      tail++; row++; cref++;
    }
    /* head: walk left from Start; the reference byte paired with query row Start.Q-1-j is
     * Start.Ref-j, one to the right of the diagonal (MatrixCPU.cpp:116-171) */
    uint64_t head = 0;
    if (row_start > 0) {
      uint64_t head_size = r->start_ref < k ? r->start_ref : k;
      if (head_size > 0) {
        uint64_t j = 0;
        for (;;) {
          if (q[row_start - 1 - j] != rs[r->start_ref - j]) { head = j; break; }
          if (row_start - 1 - j == 0 || r->start_ref - j == 0 || head_size - 1 - j == 0) { head = j; break; }
          j++;
        }
      }
    }
    uint64_t total = tail + head + mid;
    if (total >= k) {
      sum_c += total;
      memset(hit + (row_start - head), 1, total);
      sum_r += (total * (total + 1)) / 2;
    }
  }
  if (sum_c > 0) {
    uint32_t hits = 0;
    for (uint32_t i = 0; i < L; i++) hits += hit[i] ? 1 : 0;
    float score = (float)sum_r / (float)sum_c;
    float pct = (float)((100.0 / (double)(float)L) * (double)(float)hits);
    *out_pct = pct;
    *out_score = (float)(((double)score / 100.0) * (double)pct);
  }
}

/* Uppercase (Sequences.cpp:43-55: bytes above 96 lose 32, char is signed). */
static uint8_t upper(uint8_t c) { return ((int8_t)c > 96) ? (uint8_t)(c - 32) : c; }

/* reverseComplementDNA's table (Sequences.cpp:795-841); 0 = not a nucleotide. */
static uint8_t complement(uint8_t c) {
  switch (c) {
    case 'A': return 'T'; case 'T': return 'A'; case 'U': return 'A';
    case 'G': return 'C'; case 'C': return 'G'; case 'Y': return 'R'; case 'R': return 'Y';
    case 'S': return 'S'; case 'W': return 'W'; case 'K': return 'M'; case 'M': return 'K';
    case 'B': return 'V'; case 'D': return 'H'; case 'H': return 'D'; case 'V': return 'B';
    case 'N': return 'N'; case '-': return '-'; case '~': return '~';
    default: return 0;
  }
}

/* TPrepareGPUAnalysis for one strand (Analyser.cpp:1453-2490) followed by the per-candidate
 * scoring of TGetScore / CreateResultsScores (MatrixCPU.cpp:248-370). Appends candidates and
 * runs to ws and returns the strand's HighestScore through *highest. */
static int classify_strand(const mgo_index* ix, const uint8_t* q, uint32_t L, ws_t* ws,
                           uint64_t* cand_first, uint32_t* n_cand, float* highest) {
  const uint32_t k = (uint32_t)ix->k;
  const uint32_t step = k / 2;             /* Analyser.cpp:1387-1388 */
  const int hlen = (int)(k - step + 1);    /* Analyser.cpp:1389 */
  *cand_first = ws->cand_n;
  *n_cand = 0;
  *highest = -1;
  /* Reads not longer than k make the reference hash past the end of the read (undefined
   * there); such reads can never reach a diagonal of k bases and get no seeds here. */
  if (L <= k) return 0;
  uint32_t istop = L - k;                  /* Analyser.cpp:1459-1463 */
  /* seeds and TOC lookups (A1, A2) */
  uint64_t nf = 0, ne = 0;
  uint64_t n_seeds = (istop + step - 1) / step;
  GROW(ws->found_p, ws->found_cap, n_seeds, uint32_t);
  ws->found_off = (uint32_t*)realloc(ws->found_off, ws->found_cap * 4);
  ws->found_cnt = (uint32_t*)realloc(ws->found_cnt, ws->found_cap * 4);
  if (!ws->found_off || !ws->found_cnt) return E_OOM;
  for (uint32_t p = 0; p < istop; p += step) {
    int64_t t = toc_find(ix, mgo_hash28(q + p, hlen));
    if (t < 0) continue;
    int64_t c = decode(ix, t, ws, ne);
    if (c < 0) return (int)c;
    ws->found_p[nf] = p;
    ws->found_off[nf] = (uint32_t)ne;
    ws->found_cnt[nf] = (uint32_t)c;
    nf++;
    ne += (uint64_t)c;
  }
  if (nf == 0) return 0;
  /* occurrence filter (A4, Analyser.cpp:2004-2196) */
  uint32_t lowest = ix->n_refs, highest_ref = 0;
  for (uint64_t e = 0; e < ne; e++) {
    if (ws->post[e].ref < lowest) lowest = ws->post[e].ref;
    if (ws->post[e].ref > highest_ref) highest_ref = ws->post[e].ref;
  }
  if (lowest > highest_ref) return 0;
  uint64_t span = (uint64_t)(highest_ref - lowest) + 1;
  GROW(ws->occ, ws->occ_cap, span, int32_t);
  ws->occmax = (int32_t*)realloc(ws->occmax, ws->occ_cap * 4);
  ws->last = (int32_t*)realloc(ws->last, ws->occ_cap * 4);
  if (!ws->occmax || !ws->last) return E_OOM;
  memset(ws->occ, 0, span * 4);
  memset(ws->occmax, 0, span * 4);
  memset(ws->last, 0xff, span * 4);
  uint64_t hs = 0;
  for (uint64_t i = 0; i < nf; i++) {
    for (uint32_t j = 0; j < ws->found_cnt[i]; j++) {
      uint32_t r = ws->post[ws->found_off[i] + j].ref - lowest;
      if (i == 0) {
        ws->occ[r] = 1;
        ws->occmax[r] = 1;
        ws->last[r] = 0;
        continue;
      }
      if ((int64_t)ws->last[r] == (int64_t)i) continue;
      if ((int64_t)ws->last[r] == (int64_t)i - 1) {
        ws->occ[r]++;
        if (ws->occ[r] > ws->occmax[r]) ws->occmax[r] = ws->occ[r];
        if ((uint64_t)ws->occmax[r] > hs) hs = (uint64_t)ws->occmax[r];
      } else {
        ws->occ[r] = 1;
        if (ws->occmax[r] < 1) ws->occmax[r] = 1;
      }
      ws->last[r] = (int32_t)i;
    }
  }
  uint64_t keep_min = hs != 0 ? hs - 1 : 0;   /* Analyser.cpp:2115 */
  if (keep_min < 1) keep_min = 1;
  uint64_t nt = 0;
  GROW(ws->trip, ws->trip_cap, ne, trip_t);
  for (uint64_t i = 0; i < nf; i++)
    for (uint32_t j = 0; j < ws->found_cnt[i]; j++) {
      post_t e = ws->post[ws->found_off[i] + j];
      if ((uint64_t)ws->occmax[e.ref - lowest] >= keep_min) {
        ws->trip[nt].ref = e.ref;
        ws->trip[nt].rpos = e.pos;
        ws->trip[nt].qpos = ws->found_p[i];
        nt++;
      }
    }
  if (nt == 0) return 0;
  /* sort by (ref, Reference, Query) (A5, Analyser.cpp:1024-1036) */
  qsort(ws->trip, nt, sizeof(trip_t), cmp_trip);
  /* distinct references and their longest diagonal run (A6, Analyser.cpp:2337-2395) */
  uint32_t n_refs_hit = 0;
  uint64_t best = 0;
  for (uint64_t a = 0; a < nt;) {
    uint64_t b = a + 1;
    while (b < nt && ws->trip[b].ref == ws->trip[a].ref) b++;
    uint64_t cur = 1, hi = 0;
    for (uint64_t i = a + 1; i < b; i++) {
      const trip_t* pv = &ws->trip[i - 1];
      const trip_t* cu = &ws->trip[i];
      if (!((uint64_t)pv->rpos + step == cu->rpos && (uint64_t)pv->qpos + step == cu->qpos)) {
        if (cur > hi) hi = cur;
        cur = 0;
      }
      cur++;
    }
    if (cur > hi) hi = cur;
    if (hi > best) best = hi;
    n_refs_hit++;
    a = b;
  }
  GROW(ws->cand, ws->cand_cap, ws->cand_n + n_refs_hit, mgo_cand);
  uint64_t c0 = ws->cand_n;
  for (uint64_t a = 0; a < nt;) {
    uint64_t b = a + 1;
    while (b < nt && ws->trip[b].ref == ws->trip[a].ref) b++;
    mgo_cand* cd = &ws->cand[ws->cand_n++];
    cd->ref = ws->trip[a].ref;
    cd->n_runs = 0;
    cd->run_off = (uint32_t)ws->run_n;
    cd->score = -2;
    cd->pct = 0;
    cd->rel = -1;
    if (best >= 2) {
      uint64_t cur = 1, hi = 0;
      for (uint64_t i = a + 1; i < b; i++) {
        const trip_t* pv = &ws->trip[i - 1];
        const trip_t* cu = &ws->trip[i];
        if (!((uint64_t)pv->rpos + step == cu->rpos && (uint64_t)pv->qpos + step == cu->qpos)) {
          if (cur > hi) hi = cur;
          cur = 0;
        }
        cur++;
      }
      if (cur > hi) hi = cur;
      /* keep rule: only references whose longest run equals the read's longest (:2428-2436) */
      if (hi >= best && hi >= 2) {
        uint64_t s = a;
        for (uint64_t i = a + 1; i <= b; i++) {
          int brk = (i == b);
          if (!brk) {
            const trip_t* pv = &ws->trip[i - 1];
            const trip_t* cu = &ws->trip[i];
            brk = !((uint64_t)pv->rpos + step == cu->rpos && (uint64_t)pv->qpos + step == cu->qpos);
          }
          if (brk) {
            GROW(ws->run, ws->run_cap, ws->run_n + 1, mgo_run);
            mgo_run* rr = &ws->run[ws->run_n++];
            rr->start_ref = ws->trip[s].rpos;
            rr->start_q = ws->trip[s].qpos;
            rr->last_ref = ws->trip[i - 1].rpos + step;
            rr->last_q = ws->trip[i - 1].qpos + step;
            cd->n_runs++;
            s = i;
          }
        }
      }
    }
    a = b;
  }
  /* scoring (A8) and relative scores (A10) */
  GROW(ws->hit, ws->hit_cap, L, uint8_t);
  float hi_rel = -1;
  for (uint64_t c = c0; c < ws->cand_n; c++) {
    mgo_cand* cd = &ws->cand[c];
    calculate_score(ix, q, L, cd->ref, ws->run + cd->run_off, cd->n_runs, ws->hit, &cd->score, &cd->pct);
    if (cd->score > -1) {
      cd->rel = mgo_relative_score((float)L, (float)ix->ref_size[cd->ref], cd->score);
      if (cd->rel > hi_rel) hi_rel = cd->rel;
    }
  }
  *n_cand = (uint32_t)(ws->cand_n - c0);
  *highest = hi_rel;
  return 0;
}

typedef struct {
  const mgo_index* ix;
  const uint8_t* bases;
  const uint64_t* offs;
  uint64_t lo, hi;
  mgo_strand* strands; /* local: 2 per read of [lo, hi) */
  mgo_read* reads;
  ws_t ws;
  int rc;
  int keep;            /* keep candidate / run arrays */
} job_t;

static void* run_job(void* arg) {
  job_t* jb = (job_t*)arg;
  ws_t* ws = &jb->ws;
  uint8_t* fwd = NULL;
  uint8_t* rev = NULL;
  uint64_t cap = 0;
  for (uint64_t i = jb->lo; i < jb->hi; i++) {
    uint64_t L64 = jb->offs[i + 1] - jb->offs[i];
    if (L64 > 0xFFFFFFFFull) { jb->rc = E_INPUT; break; }
    uint32_t L = (uint32_t)L64;
    if (L + 1 > cap) {
      cap = L + 1;
      fwd = (uint8_t*)realloc(fwd, cap);
      rev = (uint8_t*)realloc(rev, cap);
      if (!fwd || !rev) { jb->rc = E_OOM; break; }
    }
    const uint8_t* raw = jb->bases + jb->offs[i];
    for (uint32_t j = 0; j < L; j++) fwd[j] = upper(raw[j]);
    for (uint32_t j = 0; j < L; j++) {
      uint8_t c = complement(fwd[L - 1 - j]);
      if (!c) { jb->rc = E_INPUT; break; }
      rev[j] = c;
    }
    if (jb->rc) break;
    if (!jb->keep) { ws->cand_n = 0; ws->run_n = 0; }
    mgo_strand* s = &jb->strands[2 * (i - jb->lo)];
    uint64_t c0;
    int rc = classify_strand(jb->ix, fwd, L, ws, &c0, &s[0].n_cand, &s[0].highest);
    s[0].cand_off = (uint32_t)c0;
    if (!rc) rc = classify_strand(jb->ix, rev, L, ws, &c0, &s[1].n_cand, &s[1].highest);
    s[1].cand_off = (uint32_t)c0;
    if (rc) { jb->rc = rc; break; }
    /* strand merge (Analyser.cpp:592-611) and the log skip rule (:388) */
    mgo_read* rd = &jb->reads[i - jb->lo];
    int from_rc = s[0].highest < s[1].highest;
    const mgo_strand* ch = &s[from_rc];
    uint32_t n_scored = 0;
    for (uint32_t c = 0; c < ch->n_cand; c++) n_scored += ws->cand[ch->cand_off + c].score > -1;
    rd->highest = ch->highest;
    rd->strand = from_rc;
    rd->reported = (n_scored > 0 && ch->highest != 0);
    rd->n_top = 0;
    if (rd->reported)
      for (uint32_t c = 0; c < ch->n_cand; c++) {
        const mgo_cand* cd = &ws->cand[ch->cand_off + c];
        if (cd->score > -1 && cd->rel == ch->highest) rd->n_top++;
      }
  }
  free(fwd);
  free(rev);
  return NULL;
}

static void ws_free(ws_t* w) {
  free(w->post); free(w->found_p); free(w->found_off); free(w->found_cnt); free(w->occ);
  free(w->occmax); free(w->last); free(w->trip); free(w->hit); free(w->rep_cnt); free(w->rep_pos);
  free(w->cand); free(w->run);
}

static int run_all(const mgo_index* ix, const uint8_t* bases, const uint64_t* offs, uint64_t n,
                   int nthreads, int keep, job_t** jobs_out, int* nj_out, mgo_strand* strands,
                   mgo_read* reads) {
  if (nthreads < 1) nthreads = 1;
  if ((uint64_t)nthreads > n) nthreads = n ? (int)n : 1;
  job_t* jobs = (job_t*)calloc((size_t)nthreads, sizeof(job_t));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  if (!jobs || !th) { free(jobs); free(th); return E_OOM; }
  uint64_t per = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; t++) {
    jobs[t].ix = ix; jobs[t].bases = bases; jobs[t].offs = offs; jobs[t].keep = keep;
    jobs[t].lo = (uint64_t)t * per < n ? (uint64_t)t * per : n;
    jobs[t].hi = jobs[t].lo + per < n ? jobs[t].lo + per : n;
    uint64_t cnt = jobs[t].hi - jobs[t].lo;
    jobs[t].strands = strands ? strands + 2 * jobs[t].lo : (mgo_strand*)calloc(2 * cnt + 2, sizeof(mgo_strand));
    jobs[t].reads = reads ? reads + jobs[t].lo : (mgo_read*)calloc(cnt + 1, sizeof(mgo_read));
    pthread_create(&th[t], NULL, run_job, &jobs[t]);
  }
  int rc = 0;
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    if (jobs[t].rc && !rc) rc = jobs[t].rc;
  }
  free(th);
  if (!strands) for (int t = 0; t < nthreads; t++) { free(jobs[t].strands); free(jobs[t].reads); }
  *jobs_out = jobs;
  *nj_out = nthreads;
  return rc;
}

static int cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : x > y;
}

int mgo_classify(const mgo_index* ix, const uint8_t* bases, const uint64_t* offs, uint64_t n,
                 int nthreads, mgo_strand* strands, mgo_read* reads, mgo_cand** cands,
                 uint64_t* n_cands, mgo_run** runs, uint64_t* n_runs, uint32_t* top_refs,
                 uint64_t* top_off, uint64_t top_cap) {
  job_t* jobs = NULL;
  int nj = 0;
  int rc = run_all(ix, bases, offs, n, nthreads, 1, &jobs, &nj, strands, reads);
  if (rc) {
    for (int t = 0; t < nj; t++) ws_free(&jobs[t].ws);
    free(jobs);
    return rc;
  }
  /* concatenate per-thread candidate / run arrays, rebasing offsets */
  uint64_t tc = 0, tr = 0;
  for (int t = 0; t < nj; t++) { tc += jobs[t].ws.cand_n; tr += jobs[t].ws.run_n; }
  mgo_cand* C = (mgo_cand*)malloc((tc + 1) * sizeof(mgo_cand));
  mgo_run* R = (mgo_run*)malloc((tr + 1) * sizeof(mgo_run));
  if (!C || !R) { free(C); free(R); rc = E_OOM; }
  uint64_t cb = 0, rb = 0, tp = 0;
  for (int t = 0; t < nj && !rc; t++) {
    job_t* jb = &jobs[t];
    for (uint64_t c = 0; c < jb->ws.cand_n; c++) {
      C[cb + c] = jb->ws.cand[c];
      C[cb + c].run_off += (uint32_t)rb;
    }
    memcpy(R + rb, jb->ws.run, jb->ws.run_n * sizeof(mgo_run));
    for (uint64_t i = jb->lo; i < jb->hi; i++) {
      strands[2 * i].cand_off += (uint32_t)cb;
      strands[2 * i + 1].cand_off += (uint32_t)cb;
      if (top_off) {
        top_off[i] = tp;
        if (reads[i].reported) {
          const mgo_strand* ch = &strands[2 * i + reads[i].strand];
          uint64_t t0 = tp;
          for (uint32_t c = 0; c < ch->n_cand; c++) {
            const mgo_cand* cd = &C[ch->cand_off + c];
            if (cd->score > -1 && cd->rel == ch->highest) {
              if (tp >= top_cap) { rc = E_OOM; break; }
              top_refs[tp++] = cd->ref;
            }
          }
          qsort(top_refs + t0, tp - t0, 4, cmp_u32);
        }
      }
    }
    cb += jb->ws.cand_n;
    rb += jb->ws.run_n;
  }
  for (int t = 0; t < nj; t++) ws_free(&jobs[t].ws);
  free(jobs);
  if (rc) { free(C); free(R); return rc; }
  *cands = C; *n_cands = tc; *runs = R; *n_runs = tr;
  return 0;
}

int64_t mgo_classify_count(const mgo_index* ix, const uint8_t* bases, const uint64_t* offs,
                           uint64_t n, int nthreads) {
  job_t* jobs = NULL;
  int nj = 0;
  int rc = run_all(ix, bases, offs, n, nthreads, 0, &jobs, &nj, NULL, NULL);
  for (int t = 0; t < nj; t++) ws_free(&jobs[t].ws);
  free(jobs);
  return rc ? rc : (int64_t)n;
}
