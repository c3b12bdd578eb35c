/*
 * mirage_b200 -- B200-native MirAge classification hot path, C ABI.
 *
 * The reference binds this path through C++ calls with STL types (no C ABI exists there):
 *   - index load:   Hashmap::ReadHashmapFile            (MirAge/Hashmap.cpp:329, Hashmap.h:175)
 *   - seed lookup:  Analyser::TPrepareGPUAnalysis        (MirAge/Analyser.cpp:1317, Analyser.h:175)
 *   - scoring:      MatrixCPU::CPUGetHighestScore        (MirAge/MatrixCPU.cpp:417, MatrixCPU.h:41)
 *                   CUDAGetHighestScore                  (MirAge/MatrixGPUCU.cu:571, Analyser.h:228)
 *   - strand merge: Analyser::TGetHighestScoreUsingCPU   (MirAge/Analyser.cpp:592-611)
 * The entry points below replace those calls one for one (each declaration names the call it
 * replaces). Plain pointers and sizes only; no exceptions cross this boundary; every function
 * returns MG_OK (0) or a negative MG_ERR_* code, with a message from mg_last_error().
 *
 * Semantics are the reference's CPU path (MatrixCPU), bit-exact: the same candidate
 * references, the same Score / percentageMatch / relative-score float bits and the same
 * top-scoring reference set per read, for a single .mhm file in memory mode "extreme",
 * speed mode "Sensitive", reverse complements on.
 *
 * Threading: an mg_index is immutable after mg_open and may be shared by threads; each call
 * that takes an mg_index serialises on the index's internal stream lock. mg_server is
 * internally synchronised.
 */
#ifndef MIRAGE_B200_H
#define MIRAGE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MG_OK 0
#define MG_ERR_IO (-1)        /* file cannot be opened or read */
#define MG_ERR_BADFMT (-2)    /* not a readable .mhm (or k below its build threshold) */
#define MG_ERR_OOM (-3)       /* host or device allocation failed; output buffer too small */
#define MG_ERR_LIMIT (-4)     /* a size outside what this build supports */
#define MG_ERR_CUDA (-5)      /* CUDA runtime error */
#define MG_ERR_BADINPUT (-6)  /* a read holds a byte with no reverse complement */
#define MG_ERR_TIMEOUT (-7)   /* a device-side wait exceeded its iteration bound */
#define MG_ERR_INVAL (-8)     /* bad argument */
#define MG_ERR_BUSY (-9)      /* served form: not enough free slots / memory right now */

typedef struct mg_index mg_index;
typedef struct mg_server mg_server;

/* Sequences parsed from a FASTA text (mg_parse_fasta_device). Sequence i is
 * bases[offsets[i] .. offsets[i+1]); its header line is text[header_at[i] .. + header_len[i])
 * of the caller's text (starting with '>', without a trailing '\r'). Free with mg_seqs_free. */
typedef struct {
  uint64_t n_seqs;
  uint64_t* offsets;      /* n_seqs + 1 */
  uint8_t* bases;
  uint64_t* header_at;    /* n_seqs */
  uint32_t* header_len;   /* n_seqs */
} mg_seqs;

/* A batch of reads as CSR: read i is bases[offsets[i] .. offsets[i+1]), raw sequence bytes
 * as they appear in the FASTA/FASTQ file (the library applies the reference's normalisation:
 * bytes 97..127 lose 32, Sequences.cpp:43-55, and builds the reverse complement of every read,
 * Sequences.cpp:795-889). */
typedef struct {
  uint64_t n_reads;
  const uint64_t* offsets; /* n_reads + 1 entries, offsets[0] == 0 */
  const uint8_t* bases;
} mg_batch;

/* Result of one read after the strand merge (Analyser.cpp:592-611). */
typedef struct {
  float highest;       /* MatrixResult::HighestScore of the kept strand (-1: no candidate) */
  uint32_t cand_off;   /* first scored candidate of this read in mg_result.cands */
  uint16_t n_fwd;      /* scored candidates of the forward strand (they come first) */
  uint16_t n_rc;       /* scored candidates of the reverse-complement strand */
  uint8_t strand;      /* 0: forward kept, 1: reverse complement kept; a rejected read holds
                        * MG_READ_BAD_BYTE or MG_READ_TOO_LARGE (and the call fails) */
  uint8_t reported;    /* 1 when the reference logs this read (Analyser.cpp:388) */
  uint16_t n_top;      /* size of the top-scoring reference group */
} mg_read_result;

#define MG_READ_BAD_BYTE 0xFF   /* the read holds a byte without a reverse complement */
#define MG_READ_TOO_LARGE 0xFE  /* the read exceeds the oversize tier's limits */

/* One scored candidate (a MatrixResult::ResultsScores entry with its raw score). Candidates
 * of a strand are in ascending refID order, as CreateResultsScores emits them. */
typedef struct {
  uint32_t ref;        /* global reference ID (.mhm order) */
  float rel;           /* relative score, MatrixResult::GetRelativeScore */
  float score;         /* CalculateScore's Score */
  float pct;           /* CalculateScore's percentageMatch */
} mg_candidate;

/* Caller-owned output buffers. */
typedef struct {
  mg_read_result* reads;   /* n_reads entries */
  mg_candidate* cands;     /* cand_cap entries */
  uint64_t cand_cap;
  uint64_t n_cands;        /* written: candidates used (or needed, with MG_ERR_OOM) */
} mg_result;

/* Index statistics. */
typedef struct {
  uint64_t n_hashes, n_postings, n_refs, ref_bases;
  uint64_t device_bytes;   /* HBM held by the index */
  int32_t k, word;         /* k and the .mhm word width (4 or 8) */
  double load_seconds, upload_seconds;
  int32_t probe_slots;     /* 1 while the hash-slot table is built (mg_set_probe_slots) */
} mg_index_info;

/* Replaces Hashmap::ReadHashmapFile (Hashmap.cpp:329) for one file: parses the .mhm, decodes
 * every posting record (Analyser.cpp:1602-1752) and builds the HBM-resident lookup tables on
 * `device`. k is considerthreshold (MirAge.cpp:208); it may not be below the index's own. */
int mg_open(const char* mhm_path, int k, int device, mg_index** out);

/* Same from an in-memory .mhm image. */
int mg_open_image(const uint8_t* image, uint64_t len, int k, int device, mg_index** out);

void mg_close(mg_index* ix);
int mg_index_get_info(const mg_index* ix, mg_index_info* info);

/* Host-only validation of a .mhm image (no GPU needed): parses the file the way mg_open does,
 * decodes every posting record, and fills the counts of *info (device fields zero). Same
 * error codes as mg_open_image. */
int mg_inspect_image(const uint8_t* image, uint64_t len, int k, mg_index_info* info);

/* The logarithm the relative score uses, evaluated on the index's device at n points
 * (device results for x in [1, 2^20), which match the host libm's logf bit for bit). Exposed
 * so callers can verify that agreement. Host buffers. */
int mg_eval_logf(mg_index* ix, const float* x, float* out, uint64_t n);

/* Diagnostics (no counterpart in the reference). mg_set_timing(ix, 1) records CUDA events
 * around every kernel of each following classification call; mg_last_kernel_times writes the
 * last call's device times in milliseconds, 5 entries: [dual-strand warp tier with its finishing
 * pass (or the plain form's kernel), general warp tier, block tier, global-memory tier, output
 * compaction]; in the batched and served forms the second to fourth run on a second stream,
 * beside the finishing pass. mg_bucket_sizes returns the number of postings stored under each
 * of n 28-bit hashes (the index directory, read on the device). */
int mg_set_timing(mg_index* ix, int on);
/* Layout of the seed probe (no counterpart in the reference, whose probe is an unordered_map
 * find, Analyser.cpp:1483-1519). With on = 1 the index holds a hash-slot table: 64 bytes per
 * 28-bit hash (17.2 GB of HBM) with the bucket's posting count, its first posting's offset and its
 * first 7 postings, so the dual-strand tiers read most seeds' postings from one 64-byte block;
 * with on = 0 they read the 4-byte directory and then the postings. mg_open builds the table for
 * indexes of at least 2^25 postings. Results are the same either way. Waits for the device to be
 * idle; MG_ERR_BUSY while a server (mg_server_create) is attached to the index. */
int mg_set_probe_slots(mg_index* ix, int on);

/* Launch shapes of the batched and served forms. They replace the reference's work balancing
 * (Hardware::TryAutoIncreaseBlocksize and HardwareAutoConfigure, Hardware.cpp:138-228, which
 * size its CPU and GPU batches at run time); results do not depend on them. A zero field keeps
 * the library's default. mg_open sets them from the tuning file of the GPU model (written by
 * python -m mirage_b200.tune) when one holds an entry for the index's density class
 * (postings per 28-bit hash: sparse below 0.25, dense below 4, saturated from 4 on). */
typedef struct {
  uint32_t dual_blocks_per_sm;   /* resident 8-warp blocks per SM of the first dual-strand tier (1-5) */
  uint32_t steal_chunk;          /* reads a warp of that tier takes per work-stealing step (1-64) */
  uint32_t first_tier;           /* dual-strand tier reads start at: 1 the 64-posting tier (default),
                                  * 2 the 128-posting one, 3 the 256-posting one (for indexes whose
                                  * strands mostly exceed the smaller tiers) */
  uint32_t second_blocks_per_sm; /* 4-warp blocks per SM of the 128-posting tier (1-6) */
  uint32_t finish_blocks_per_sm; /* 256-thread blocks per SM of the dual tiers' finishing pass (1-8) */
  uint32_t long_blocks_per_sm;   /* blocks per SM of the long-read tier (1-2) */
  uint32_t chunks;               /* pieces of a large host-buffer batch in mg_classify (1-8) */
  uint32_t weighted_chunks;      /* 1: 8 chunks weighted 1-2-3-3-3-3-2-1; 2: equal chunks */
  uint32_t third_blocks_per_sm;  /* 2-warp blocks per SM of the 256-posting tier (1-6) */
  uint32_t pack_bases;           /* mg_classify's upload of the bases: 1 as given (default); 2 packed 2 bits
                                  * per base on host threads (other bytes as a list of exceptions) and
                                  * unpacked on the device, a quarter of the bytes over the link */
} mg_tuning;
int mg_set_tuning(mg_index* ix, const mg_tuning* t);
/* The launch shapes in effect (defaults filled in) and the density class used to pick them. */
int mg_get_tuning(const mg_index* ix, mg_tuning* t, char* density_class, uint64_t class_len);
/* Diagnostic (no counterpart in the reference): the roofline of the lookup path. Times 2^26
 * gathers of whole 32-byte sectors (8 lanes per sector) at pseudo-random positions of a device
 * buffer of the largest power of two <= buffer_bytes (use several times the L2 size) on
 * `device`, best of three after a warm-up, and writes the achieved GB/s. Allocates and frees
 * the buffer itself. */
int mg_gather_bandwidth(int device, uint64_t buffer_bytes, double* gbs);
int mg_last_kernel_times(mg_index* ix, float* ms5);
/* Diagnostic: how many reads each tier of the last batched call run in one piece (the device
 * form, or host buffers too few to chunk) handed on: [the 64-, 128- and 256-posting dual-strand
 * tiers, the general warp tier, the smaller and the larger long-read size, the block tier] (the
 * last goes to the global-memory tier). With first_tier 2 or 3 the tiers before it count 0. */
int mg_last_tier_counts(mg_index* ix, uint32_t* counts7);
int mg_bucket_sizes(mg_index* ix, const uint32_t* hashes, uint32_t* counts, uint64_t n);

/* Replaces Hashmap::BuildHashmapTable + SaveHashmapTableV3 (Hashmap.cpp:967, :1701): builds a
 * .mhm image from references. names: n_refs NUL-terminated header names (without '>');
 * taxids may be NULL (-1 each); word 0 chooses 4 unless the file needs 8. On success
 * *image / *len receive a malloc'd buffer (free with mg_free). */
int mg_build_image(const uint8_t* bases, const uint64_t* offsets, uint32_t n_refs,
                   const char* const* names, const int32_t* taxids, int k, int word,
                   uint8_t** image, uint64_t* len);
void mg_free(void* p);

/* Replaces Sequences::LoadInputFiles' FASTA read (GetNumberOfHeaders, TReadFastaSequencesFromMem,
 * SequenceToUpperCase; Sequences.cpp:283-320, 57-214, 43-55) for a query or reference file held in
 * memory, parsed by kernels on `device`: the text must start with '>'; each '>' line starts a
 * sequence; other lines are appended without a trailing '\r'; uppercase != 0 uppercases the
 * bases as the reference does. A line starting with '@' is refused (MG_ERR_BADINPUT): the
 * reference reads FASTA only. */
int mg_parse_fasta_device(int device, const uint8_t* text, uint64_t len, int uppercase, mg_seqs* out);
void mg_seqs_free(mg_seqs* seqs);

/* mg_build_image on `device`: the same image, byte for byte, built by GPU kernels (window
 * hashing, one radix sort by (hash, position), bucket sizing and record encoding; the host lays
 * out the header, the reference tables and the sequence block). Needs about 64 bytes of device
 * memory per indexed position. */
int mg_build_image_device(int device, const uint8_t* bases, const uint64_t* offsets, uint32_t n_refs,
                          const char* const* names, const int32_t* taxids, int k, int word,
                          uint8_t** image, uint64_t* len);

/* Plain form. Replaces the reference's per-batch sequence TPrepareGPUAnalysis (Analyser.cpp:
 * 1317) -> CPUGetHighestScore (MatrixCPU.cpp:417) -> strand merge (Analyser.cpp:592-611):
 * one block per read in one launch per batch (the global-memory tier takes reads beyond its
 * shared memory), host buffers in and out with synchronous copies.
 * Read lengths: like the reference's CPU path, no cap below 2,000,000 bases (the batched forms
 * too; the served form takes up to 65,535). Reads past 65,535 bases, 4,400 seeds or 65,536
 * postings per strand go to the oversize tier, whose device workspace is sized by the first
 * batch that needs it: that batch runs a second time once it has grown (up to 1 GiB, a strand
 * of at most 2^24 postings); a read beyond those limits fails the call with MG_ERR_LIMIT and is
 * marked MG_READ_TOO_LARGE. */
int mg_score_batch(mg_index* ix, const mg_batch* batch, mg_result* out);

/* Batched form: the same results from the tiered persistent kernels (a warp per read with work
 * stealing first, larger tiers for the reads it hands on), copies of one chunk overlapped with
 * the classification of the one before on streams. Host buffers in and out. */
int mg_classify(mg_index* ix, const mg_batch* batch, mg_result* out);

/* Batched form on device-resident buffers (no host copies): d_offsets / d_bases / outputs are
 * device pointers; stream is a cudaStream_t (NULL = the index's stream). Part of the work runs
 * on a second, internal stream that waits for `stream` and that `stream` waits for again before
 * the results are written, so work queued on `stream` before and after sees the usual order. */
int mg_classify_device(mg_index* ix, uint64_t n_reads, const uint64_t* d_offsets,
                       const uint8_t* d_bases, mg_read_result* d_reads, mg_candidate* d_cands,
                       uint64_t cand_cap, uint64_t* d_n_cands, void* stream);
/* Waits for work queued by mg_classify_device on `stream` and reports its errors; *n_cands
 * receives the number of candidates written. It completes the index's last mg_classify_device
 * launch, whose device buffers must stay valid until it returns: a batch whose reads have more
 * candidates than the internal staging area held, or that holds reads for the oversize tier
 * beyond its current workspace (see mg_score_batch), is run again here once that has grown. */
int mg_classify_device_sync(mg_index* ix, void* stream, uint64_t* n_cands);

/* Scoring-only drop-in for MatrixCPU::CPUGetHighestScore (MatrixCPU.cpp:417) when the
 * candidate lists come from the reference's own TPrepareGPUAnalysis: per strand s (query
 * bytes bases[q_off[s]..q_off[s+1]), already normalised), candidates cand_ref[c_off[s] ..
 * c_off[s+1]) with runs run[r_off[c] .. r_off[c+1]) given as 4 uint32 (Start.Reference,
 * Start.Query, Last.Reference, Last.Query). Outputs Score, percentageMatch and relative score
 * per candidate (score -2 and rel -1 for unscored candidates) and HighestScore per strand.
 * A candidate reference beyond the index, or a walked run (Start.Query <= Last.Query) whose
 * Last.Query exceeds its query length or whose Start.Reference lies beyond its reference, is
 * refused with MG_ERR_INVAL before anything is copied to the device. */
int mg_score_candidates(mg_index* ix, uint64_t n_strands, const uint64_t* q_off,
                        const uint8_t* bases, const uint64_t* c_off, const uint32_t* cand_ref,
                        const uint64_t* r_off, const uint32_t* runs, float* score, float* pct,
                        float* rel, float* highest);

/* mg_score_candidates for callers that may not allocate device memory (their device memory is
 * held by another allocator, or a cudaFree's device-wide synchronisation would stall other
 * work). No counterpart in the reference. Same arguments and outputs, all of them DEVICE
 * pointers on ix's device, plus a stream (NULL = the index's stream); it calls no cudaMalloc or
 * cudaFree. Its working memory is a fixed 4,849,920-byte array that the library holds on every
 * GPU that loads it, until exit; that caps a query strand at 2048 bases (longer ones: MG_ERR_LIMIT,
 * and their candidates are left unscored). Every call, the first included, ends by waiting for
 * its own GPU work on `stream` (it reads the array's error word back). The first call on each
 * device also looks up the array's device address, a set-up step that has to come before any
 * stream capture begins on that device. Every call on a device uses the same array: calls whose
 * GPU work overlapped would race on it, so the library serialises the calls on each device
 * (calls on different devices do not wait for each other). A candidate reference or run outside
 * its reference or query returns MG_ERR_INVAL, as it does in mg_score_candidates. */
int mg_score_candidates_noalloc(mg_index* ix, uint64_t n_strands, const uint64_t* d_q_off,
                                const uint8_t* d_bases, const uint64_t* d_c_off,
                                const uint32_t* d_cand_ref, const uint64_t* d_r_off,
                                const uint32_t* d_runs, float* d_score, float* d_pct,
                                float* d_rel, float* d_highest, void* stream);

/* Served form: continuous batching against the HBM-resident index (no counterpart in the
 * reference). A request is admitted while it fits the pinned request ring, the tracked-request
 * limit and the device-memory budget (its bases, offsets, read results and 8 candidates per read
 * are booked until it completes; the budget follows the device's free memory as steps finish).
 * Queued reads are coalesced into steps of the fused pipeline and requests complete
 * independently. */
typedef struct {
  uint32_t max_inflight_reads;  /* reads on the device at once (0: default) */
  uint32_t max_requests;        /* concurrently tracked requests (0: default) */
  uint64_t device_budget;       /* bytes of device memory for request buffers (0: a quarter of the free memory) */
  uint32_t step_slots;          /* steps in flight at once, each with its own device buffers and stream
                                 * (2-4; 0: 3) */
} mg_server_config;

int mg_server_create(mg_index* ix, const mg_server_config* cfg, mg_server** out);
/* Copies the batch; returns MG_ERR_BUSY when it cannot be admitted now (retry later). */
int mg_server_submit(mg_server* s, const mg_batch* batch, uint64_t* ticket);
/* mg_server_submit with the caller's result buffers: the server writes the request's read
 * results into out->reads (n_reads entries, cand_off counted from out->cands[0]) and its
 * candidates into out->cands as its steps finish, so completion copies nothing; the buffers must
 * stay valid until mg_server_poll / mg_server_wait has returned the request (out may be NULL
 * there; out->n_cands of the submitted struct receives the count). When the candidates exceed
 * out->cand_cap the request completes with MG_ERR_OOM and n_cands holds the number needed. */
int mg_server_submit_into(mg_server* s, const mg_batch* batch, mg_result* out, uint64_t* ticket);
/* Page-locks the host range [ptr, ptr + len) for the server (cudaHostRegister). A request
 * submitted afterwards whose bases lie inside a registered range is copied to the device
 * straight from the caller's memory rather than through the request ring (its offsets are
 * still copied), so the caller keeps those bases unchanged until the request is complete.
 * Memory that is page-locked already (cudaMallocHost, cudaHostRegister) is refused with
 * MG_ERR_INVAL: the server reads directly only from ranges that it registered itself. Ranges
 * stay registered, and must stay allocated, until mg_server_destroy. */
int mg_server_register_host(mg_server* s, const void* ptr, uint64_t len);
/* Where the server's time went since mg_server_create (seconds; the server thread's launch,
 * device and idle times sum to its lifetime; the delivery thread's time is apart). */
typedef struct {
  uint64_t steps, reads, requests;
  uint64_t ring_bytes;    /* bases that submit copied into the request ring */
  uint64_t direct_bytes;  /* bases copied to the device from registered caller memory */
  double submit_copy_s;   /* submit: copying requests into the ring, summed over the callers */
  double launch_s;        /* server thread: forming steps, host-to-device copies, launches */
  double device_s;        /* server thread: draining finished steps (counters, candidate copies) */
  double deliver_s;       /* delivery thread: handing results to requests */
  double idle_s;          /* server thread: waiting for requests, a free step slot or a step to finish */
  double step_s;          /* summed over steps: from launch to the end of the step's device work */
} mg_server_stats;
int mg_server_get_stats(mg_server* s, mg_server_stats* out);
/* Non-blocking: returns 1 and fills out when the request is complete, 0 when not yet. */
int mg_server_poll(mg_server* s, uint64_t ticket, mg_result* out);
/* Blocking variant of mg_server_poll with a timeout in milliseconds (MG_ERR_TIMEOUT). */
int mg_server_wait(mg_server* s, uint64_t ticket, mg_result* out, uint32_t timeout_ms);
void mg_server_destroy(mg_server* s);

/* Result logs in the reference's format (host only). Replaces LogManager::Open +
 * WriteOutputHeaders (LogManager.cpp:319-404) and Analyser::LogMatrixResults /
 * LogMatrixResult / LogResultsToFileManager (Analyser.cpp:378-491, 228-376): the four files
 * results_{HighSensitivity,HighPrecision,Balanced,Raw}.log in out_dir with their headers;
 * thresholds are the LogThreshold_* settings. mg_logs_write logs n merged results: the
 * caller's input IDs (InputID column), input headers (with '>', no line end), and per
 * reference its header (with '>') and TaxID; first_group_only = output_firstresults_only. */
typedef struct mg_logs mg_logs;
int mg_logs_open(const char* out_dir, int high_precision_enabled, float th_sensitivity, float th_balanced,
                 float th_precision, mg_logs** out);
int mg_logs_write(mg_logs* logs, const mg_read_result* reads, const mg_candidate* cands, uint64_t n,
                  const uint64_t* input_ids, const char* const* input_headers, const char* const* ref_headers,
                  const int32_t* taxids, int first_group_only);
void mg_logs_close(mg_logs* logs);
/* LogManager::CreateUniqueOutputFolders (LogManager.cpp:288): creates
 * <output_path>/results_<seconds since epoch> and returns its path in out. */
int mg_make_results_dir(const char* output_path, char* out, uint64_t out_len);
/* Header (with '>'), NCBI TaxID and length of reference `ref` of an open index. */
int mg_index_reference(const mg_index* ix, uint32_t ref, const char** header, int32_t* taxid, uint32_t* length);

const char* mg_strerror(int code);
const char* mg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
