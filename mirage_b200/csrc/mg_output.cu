// Result logs in the reference's format (Analyser::LogMatrixResult, Analyser.cpp:401-491;
// Analyser::LogResultsToFileManager, :228-376; LogManager, LogManager.cpp:286-412):
//   <OutputPath>/results_<epoch>/results_{HighSensitivity,HighPrecision,Balanced,Raw}.log
//   header "InputID;InputSequence;Confident;TaxIDs;Occurence_Per_TaxID;Headers"
//   one line per logged group: InputID;input header;to_string(score);TaxIDs;occurrences;headers
// The line order inside a group follows the reference's own standard-library calls: the scores
// are ordered with std::sort (descending score) and each group with std::stable_sort under the
// reference's TaxID comparator. That comparator is not a strict weak order (TaxID -1 compares
// below everything, itself included), so the order it leaves depends on the algorithm; calling
// the same algorithms on the same sequences reproduces the reference's lines byte for byte.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <string>
#include <sys/stat.h>
#include <unordered_map>
#include <vector>

#include "../../include/mirage_b200.h"
#include "mg_internal.h"

struct mg_logs {
  std::ofstream out[4];  // HighSensitivity, HighPrecision, Balanced, Raw
  bool enabled[4] = {true, true, true, true};
  float th_sensitivity = 0.4f, th_precision = 1.0f, th_balanced = 0.7f;
  std::string dir;
};

namespace {

struct Scored {
  float score;
  uint32_t ref;
};

const char* kKinds[4] = {"HighSensitivity", "HighPrecision", "Balanced", "Raw"};
const char* kHeader = "InputID;InputSequence;Confident;TaxIDs;Occurence_Per_TaxID;Headers";

// One logged line (LogResultsToFileManager).
std::string format_line(uint64_t input_id, const char* input_header, float score, std::vector<uint32_t> results,
                        const char* const* ref_headers, const int32_t* taxids) {
  std::string s;
  s.reserve(3000);
  s += std::to_string((int)input_id);
  s += ";";
  s += input_header;
  s += ";";
  s += std::to_string(score);
  s += ";";
  if (results.empty()) {
    s += "?;";
    return s;
  }
  std::unordered_map<uint32_t, size_t> occ;
  for (uint32_t r : results) occ[(uint32_t)taxids[r]]++;
  std::stable_sort(results.begin(), results.end(), [&](uint32_t const& a, uint32_t const& b) {
    const uint32_t ta = (uint32_t)taxids[a], tb = (uint32_t)taxids[b];
    if (ta == (uint32_t)-1) return true;
    if (tb == (uint32_t)-1) return false;
    if (ta == tb) return false;
    if (occ[ta] == occ[tb]) return false;
    if (occ[ta] > occ[tb]) return true;
    if (occ[ta] < occ[tb]) return false;
    return ta < tb;
  });
  int32_t current = taxids[results[0]];
  const size_t max_occ = occ[(uint32_t)current];
  for (size_t h = 0; h < results.size(); h++) {
    const int32_t t = taxids[results[h]];
    if (h > 0 && t == current) continue;
    if (occ[(uint32_t)t] != max_occ) break;
    current = t;
    if (h != 0) s += ",";
    s += std::to_string(current);
  }
  s += ";";
  for (size_t h = 0; h < results.size(); h++) {
    const int32_t t = taxids[results[h]];
    if (h > 0 && t == current) continue;
    const size_t n = occ[(uint32_t)t];
    if (n != max_occ) break;
    current = t;
    if (h != 0) s += ",";
    s += std::to_string(n);
  }
  s += ";";
  for (size_t h = 0; h < results.size(); h++) {
    const int32_t t = taxids[results[h]];
    if (occ[(uint32_t)t] != max_occ) break;
    if (h != 0) s += ",";
    s += ref_headers[results[h]];
  }
  return s;
}

}  // namespace

extern "C" {

int mg_logs_open(const char* out_dir, int high_precision_enabled, float th_sensitivity, float th_balanced,
                 float th_precision, mg_logs** out) {
  if (!out_dir || !out) return mg::set_error(MG_ERR_INVAL, "null argument");
  mg_logs* L = new mg_logs();
  L->dir = out_dir;
  L->th_sensitivity = th_sensitivity;
  L->th_balanced = th_balanced;
  L->th_precision = th_precision;
  for (int i = 0; i < 4; i++) {
    std::string p = L->dir + "/results_" + kKinds[i] + ".log";
    L->out[i].open(p, std::ios::app);
    if (!L->out[i].is_open()) {
      delete L;
      return mg::set_error(MG_ERR_IO, "cannot open " + p);
    }
  }
  // LogManager::WriteOutputHeaders; the HighPrecision file carries a notice instead of the
  // header when the hashmap was loaded partially (MirAge.cpp:425-434)
  for (int i = 0; i < 4; i++) {
    if (i == 1 && !high_precision_enabled) {
      L->out[i] << "Hashmap loading is <100% and therefore high precision is not possible. Set loading to 100% to "
                   "enable high precision (Use Hashmap_Load_Hashmap_Percentage in configuration file)."
                << std::endl;
      L->enabled[i] = false;
    } else {
      L->out[i] << kHeader << std::endl;
    }
  }
  *out = L;
  return MG_OK;
}

int mg_logs_write(mg_logs* L, const mg_read_result* reads, const mg_candidate* cands, uint64_t n,
                  const uint64_t* input_ids, const char* const* input_headers, const char* const* ref_headers,
                  const int32_t* taxids, int first_group_only) {
  if (!L || (n && (!reads || !input_ids || !input_headers || !ref_headers || !taxids)))
    return mg::set_error(MG_ERR_INVAL, "null argument");
  std::vector<Scored> scores;
  for (uint64_t i = 0; i < n; i++) {
    const mg_read_result& r = reads[i];
    // Analyser.cpp:388: skip when no scores or the highest score is 0
    const uint32_t nk = r.strand == 0 ? r.n_fwd : r.n_rc;
    if (nk == 0 || r.highest == 0.0f) continue;
    const mg_candidate* c = cands + r.cand_off + (r.strand == 0 ? 0 : r.n_fwd);
    scores.clear();
    for (uint32_t j = 0; j < nk; j++) scores.push_back(Scored{c[j].rel, c[j].ref});
    std::sort(scores.begin(), scores.end(), [](const Scored& a, const Scored& b) { return a.score > b.score; });
    size_t at = 0;
    while (at < scores.size()) {
      const float g = scores[at].score;
      std::vector<uint32_t> group;
      while (at < scores.size() && scores[at].score == g) group.push_back(scores[at++].ref);
      const std::string line = format_line(input_ids[i], input_headers[i], g, group, ref_headers, taxids);
      if (g >= L->th_sensitivity && L->enabled[0]) L->out[0] << line << std::endl;
      if (g >= L->th_precision && L->enabled[1]) L->out[1] << line << std::endl;
      if (g >= L->th_balanced && L->enabled[2]) L->out[2] << line << std::endl;
      L->out[3] << line << std::endl;
      if (first_group_only) break;
    }
  }
  for (auto& o : L->out)
    if (!o.good()) return mg::set_error(MG_ERR_IO, "write error on a result log");
  return MG_OK;
}

void mg_logs_close(mg_logs* L) {
  if (!L) return;
  for (auto& o : L->out) o.close();
  delete L;
}

int mg_make_results_dir(const char* output_path, char* out, uint64_t out_len) {
  if (!output_path || !out) return mg::set_error(MG_ERR_INVAL, "null argument");
  // LogManager::CreateUniqueOutputFolders (LogManager.cpp:288-313)
  std::string p = std::string(output_path) + "/results_" + std::to_string((size_t)time(0));
  mkdir(p.c_str(), S_IRWXU | S_IRGRP | S_IXGRP);
  if (p.size() + 1 > out_len) return mg::set_error(MG_ERR_INVAL, "path buffer too small");
  std::memcpy(out, p.c_str(), p.size() + 1);
  return MG_OK;
}

int mg_index_reference(const mg_index* ix, uint32_t ref, const char** header, int32_t* taxid, uint32_t* length) {
  if (!ix) return mg::set_error(MG_ERR_INVAL, "null argument");
  if (ref >= ix->host.n_refs) return mg::set_error(MG_ERR_INVAL, "reference out of range");
  if (header) *header = ref < ix->host.headers.size() ? ix->host.headers[ref].c_str() : "";
  if (taxid) *taxid = ref < ix->host.taxids.size() ? ix->host.taxids[ref] : -1;
  if (length) *length = ix->host.ref_len[ref];
  return MG_OK;
}

}  // extern "C"
