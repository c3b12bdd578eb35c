// MirAge hashmap database (.mhm, format version 4): reader and writer.
//
// Layout (Hashmap::SaveHashmapTableV3, Hashmap.cpp:1701-2533; reader Hashmap.cpp:402-660):
//   magic text | n_hash (8 B) | version=4 (i32) | W (i32, 4 for the 32-bit build, 8 with
//   -D__Hash64__) | threshold k (i32) | bytes_streampos, bytes_numRefIDsPerHash,
//   writeSequenceBitsSize, writeHeaderBitsSize (1 B each)
//   TOC: n_hash x (hash W B, stream position W B), ascending hash
//   TaxIDs: count (W B), count x i32
//   sequence TOC: end-of-TOC position (W), count (W), sizes (count x W), positions (count x W)
//   header TOC: same shape
//   reference bases, headers (each header stored with its trailing NUL)
//   one posting record per TOC hash (see decode_record in mhm.cpp)
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mg {

struct Posting {
  uint32_t ref;
  uint32_t pos;
};

// A loaded index, decoded into flat arrays (the device upload works from these).
struct MhmIndex {
  int word = 4;                    // W: 4 (32-bit build) or 8 (64-bit build)
  int32_t threshold = 0;           // k the index was built with
  uint64_t n_hash = 0;
  std::vector<uint32_t> toc_hash;  // file order (ascending when written by the builder)
  std::vector<uint64_t> bucket;    // n_hash + 1 offsets into postings, file order
  std::vector<Posting> postings;   // decoded (refID, position) pairs, record order
  bool has_empty_last = false;     // the last TOC hash is present with no postings (reader quirk)
  uint32_t empty_last_hash = 0;
  uint32_t n_refs = 0;
  std::vector<uint32_t> ref_len;
  std::vector<uint64_t> ref_off;   // offset of each reference in bases
  std::vector<uint8_t> bases;      // the sequence block as stored
  std::vector<int32_t> taxids;
  std::vector<std::string> headers;  // as stored, including '>' and without the trailing NUL
};

// Error codes shared with the C ABI.
enum : int {
  MHM_OK = 0,
  MHM_ERR_IO = -1,
  MHM_ERR_FORMAT = -2,
  MHM_ERR_OOM = -3,
  MHM_ERR_LIMIT = -4,
};

// Where the parts of a .mhm image lie (byte offsets into the image).
struct MhmMeta {
  uint64_t toc_at = 0;     // bucket TOC: n_hash x (hash, record stream position), word bytes each
  uint64_t bases_at = 0;   // reference sequence block
  uint64_t bases_len = 0;
};

// Everything but the bucket TOC and the posting records: header, TaxIDs, reference lengths and
// offsets, headers, and (copy_bases) the sequence block into out->bases. toc_hash, bucket and
// postings stay empty.
int mhm_parse_meta(const uint8_t* data, uint64_t len, int k, MhmIndex* out, MhmMeta* meta, bool copy_bases,
                   std::string* err);

// Parse an in-memory .mhm image. nthreads host threads decode the posting records.
int mhm_parse(const uint8_t* data, uint64_t len, int k, int nthreads, MhmIndex* out, std::string* err);
int mhm_load(const std::string& path, int k, int nthreads, MhmIndex* out, std::string* err);

// Build a .mhm image from references (the index build of Hashmap.cpp:967-1292 / 2771-2976 and
// the writer of :1701-2533). bases/offs: sequence bytes as the reference parser stores them
// (uppercased); headers without '>'; taxids may be empty (-1 each). word 0 picks 4 unless the
// file needs 64-bit positions.
int mhm_build(const uint8_t* bases, const uint64_t* offs, uint32_t n_refs,
              const std::vector<std::string>& headers, const std::vector<int32_t>& taxids, int k,
              int word, int nthreads, std::vector<uint8_t>* out, std::string* err);

uint32_t hash28(const uint8_t* p, int len);

// Byte width of a value in the writer's rule ((bits - 1) / 8) + 1 (Hashmap.cpp:1641-1671).
int mhm_width_of(uint64_t v);

// Word width and section offsets of a .mhm image with ng buckets whose records take rec_total
// bytes, the last bucket's last_rec of them (the layout of SaveHashmapTableV3,
// Hashmap.cpp:1868-2128). word 0 picks 4 unless the file needs 64-bit positions.
struct MhmPlan {
  uint64_t W = 0;          // word width, 4 or 8
  uint64_t toc_at = 0;     // bucket TOC: ng x (hash, record stream position), W bytes each
  uint64_t first_rec = 0;  // first posting record
  uint64_t total = 0;      // image size
};
int mhm_plan(const uint64_t* offs, uint32_t n_refs, const std::vector<std::string>& headers, int word,
             uint64_t ng, uint64_t rec_total, uint64_t last_rec, MhmPlan* plan, std::string* err);
// Everything of the image but the bucket TOC and the records, into out[0, plan.first_rec).
int mhm_write_head(uint8_t* out, const MhmPlan& plan, const uint8_t* bases, const uint64_t* offs, uint32_t n_refs,
                   const std::vector<std::string>& headers, const std::vector<int32_t>& taxids, int k, uint64_t ng,
                   uint32_t max_group, std::string* err);

}  // namespace mg
