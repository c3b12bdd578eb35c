/*
 * TEST INFRASTRUCTURE ONLY -- the CPU restatement of MirAge's classification hot path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load this library,
 * and only as the checker / reported CPU baseline. The product (mirage_b200) never links it.
 *
 * Parity of this restatement is pinned against the reference itself: oracle/ref_harness.cpp
 * drives the unmodified reference CPU path (compiled out of tree by oracle/Makefile) and the
 * golden dumps under tests/golden/ were produced by it; tests/test_oracle_golden.py checks
 * this restatement against them.
 */
#ifndef MG_ORACLE_H
#define MG_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mgo_index mgo_index;

/* One diagonal run of a candidate: Start and Last positions (Analyser.cpp:2453-2481). */
typedef struct {
  uint32_t start_ref, start_q, last_ref, last_q;
} mgo_run;

/* One candidate reference of one strand (the reference's matchedReferencesPerQuery entry). */
typedef struct {
  uint32_t ref;      /* global reference ID */
  uint32_t n_runs;   /* 0 for references dropped by the keep rule */
  uint32_t run_off;  /* index into the run array */
  float score;       /* CalculateScore's Score (-2 = no score) */
  float pct;         /* percentageMatch (0 when score == -2) */
  float rel;         /* GetRelativeScore (only when score > -1, else -1) */
} mgo_cand;

typedef struct {
  uint32_t cand_off, n_cand;  /* into the candidate array */
  float highest;              /* MatrixResult::HighestScore of the strand (-1 = none) */
} mgo_strand;

typedef struct {
  float highest;       /* after the strand merge */
  int32_t strand;      /* 0 forward, 1 reverse complement */
  int32_t reported;    /* 1 when LogMatrixResults would log the read */
  uint32_t n_top;      /* size of the top-scoring reference group */
} mgo_read;

/* Open a single-file .mhm (hashmap format version 4, 32-bit build). k = considerthreshold. */
int mgo_open(const char* path, int k, mgo_index** out);
void mgo_close(mgo_index* ix);
uint32_t mgo_n_refs(const mgo_index* ix);
uint32_t mgo_ref_size(const mgo_index* ix, uint32_t ref);
uint64_t mgo_n_hashes(const mgo_index* ix);

/* CreateHash24 (Hashmap.cpp:3233) over len bytes. */
uint32_t mgo_hash28(const uint8_t* p, int len);

/* Classify n reads (raw FASTA sequence bytes, CSR by offs[n+1]) with nthreads host threads.
 * Writes per read 2 strands (forward, reverse complement) into strands[2n], merged results
 * into reads[n]. Candidates and runs are allocated internally and returned through *cands,
 * *runs (free with mgo_free); counts in *n_cands, *n_runs. top_refs receives the top group
 * refIDs (ascending) of every reported read at top_off[i] (size n_top), capacity top_cap.
 * Returns 0, or a negative error code. */
int mgo_classify(const mgo_index* ix, const uint8_t* bases, const uint64_t* offs, uint64_t n,
                 int nthreads, mgo_strand* strands, mgo_read* reads, mgo_cand** cands,
                 uint64_t* n_cands, mgo_run** runs, uint64_t* n_runs, uint32_t* top_refs,
                 uint64_t* top_off, uint64_t top_cap);

/* Same work, results discarded: the timed CPU baseline. Returns reads classified. */
int64_t mgo_classify_count(const mgo_index* ix, const uint8_t* bases, const uint64_t* offs,
                           uint64_t n, int nthreads);

void mgo_free(void* p);

/* The relative score of GetRelativeScore (MatrixResult.cpp:21) for a query length, reference
 * length and Score, exactly as the reference computes it (float logf). */
float mgo_relative_score(float query_len, float ref_len, float score);

/* Host libm logf at n consecutive float bit patterns starting at lo_bits (the function
 * GetRelativeScore calls: MatrixResult.cpp:28 resolves log(float) to logf). */
void mgo_logf_bits(uint32_t lo_bits, uint64_t n, float* out);

#ifdef __cplusplus
}
#endif
#endif
