// mirage_gpu: the MirAge program's classification run with the hot path on the GPU.
//
// Keeps the reference's interfaces: the configuration file (`name:value # comment`, keys case
// insensitive, Configuration.cpp:96-150) at ./../mirage/data/mirage.identifier.cfg or the path
// given by -cfg, every setting overridable as `-<name> <value>` (Configuration.cpp:7-15,
// 165-181), -input <query file> (MirAge.cpp:131), a FASTA reference (indexed on the fly and
// saved as results_<epoch>/hashmap_<name>.mhm when output_save_hashmap_database is 1) or a
// .mhm index, and the four result logs in <OutputPath>/results_<epoch>/.
//
// The classification itself (seed lookup, diagonal scoring, best reference pick, strand merge)
// runs through the library's batched form (mg_classify) on the GPU given by -gpu (default 0).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "mirage_b200.h"

namespace {

std::string trim(std::string s) {
  const char* ws = " \t\n\r\f\v";
  s.erase(s.find_last_not_of(ws) + 1);
  s.erase(0, s.find_first_not_of(ws));
  return s;
}

std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::tolower);
  return s;
}

struct Config {
  std::unordered_map<std::string, std::vector<std::string>> kv;
  std::vector<std::string> args;  // CLI, names lowercased

  bool load(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    int no = 0;
    while (std::getline(f, line)) {
      no++;
      line = trim(line.substr(0, line.find('#')));
      if (line.empty()) continue;
      size_t c = line.find(':');
      if (c == std::string::npos) {
        std::fprintf(stderr, "ERROR in configuration file, setting or value not found at line %d: [%s]\n", no,
                     line.c_str());
        std::exit(1);
      }
      kv[lower(trim(line.substr(0, c)))].push_back(trim(line.substr(c + 1)));
    }
    return true;
  }
  // CLI `-name value` first, then the file (Configuration::GetConfigurationSettingArray)
  std::string get(const std::string& name, const std::string& def = "", bool required = false) const {
    const std::string key = "-" + lower(name);
    for (size_t i = 0; i + 1 < args.size(); i++)
      if (args[i] == key && !args[i + 1].empty()) return args[i + 1];
    auto it = kv.find(lower(name));
    if (it != kv.end() && !it->second.empty()) return it->second.front();
    if (required) {
      std::fprintf(stderr, "Configuration setting '%s' not found.\n", name.c_str());
      std::exit(1);
    }
    return def;
  }
  size_t count(const std::string& name) const {
    auto it = kv.find(lower(name));
    return it == kv.end() ? 0 : it->second.size();
  }
};

struct Seqs {
  std::vector<uint8_t> bases;
  std::vector<uint64_t> offs{0};
  std::vector<std::string> headers;  // header line with '>' / '@'
};

// A FASTA file as the reference's loader reads it (Sequences.cpp:283-320, 57-214), parsed on the
// GPU (mg_parse_fasta_device); uppercase as the loader does for references. Returns false when the
// file cannot be read; a file the reference would not load either (not starting with '>', or
// FASTQ) stops the program with the library's message.
bool read_fasta(const std::string& path, int gpu, Seqs* out, bool uppercase) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return false;
  const uint64_t len = (uint64_t)f.tellg();
  f.seekg(0);
  std::vector<uint8_t> text(len);
  if (len && !f.read((char*)text.data(), (std::streamsize)len)) return false;
  mg_seqs s{};
  const int rc = mg_parse_fasta_device(gpu, text.data(), len, uppercase ? 1 : 0, &s);
  if (rc) {
    std::fprintf(stderr, "mirage_gpu: reading %s failed: %s (%s)\n", path.c_str(), mg_strerror(rc), mg_last_error());
    std::exit(1);
  }
  out->offs.assign(s.offsets, s.offsets + s.n_seqs + 1);
  out->bases.assign(s.bases, s.bases + s.offsets[s.n_seqs]);
  out->headers.resize(s.n_seqs);
  for (uint64_t i = 0; i < s.n_seqs; i++)
    out->headers[i].assign((const char*)text.data() + s.header_at[i], s.header_len[i]);
  mg_seqs_free(&s);
  return true;
}

std::string base_name_no_ext(const std::string& p) {
  std::string f = p.substr(p.find_last_of('/') == std::string::npos ? 0 : p.find_last_of('/') + 1);
  size_t dot = f.find_last_of('.');
  return dot == std::string::npos ? f : f.substr(0, dot);
}

bool ends_with(const std::string& s, const std::string& x) {
  return s.size() >= x.size() && s.compare(s.size() - x.size(), x.size(), x) == 0;
}

[[noreturn]] void die(const char* what, int rc) {
  std::fprintf(stderr, "mirage_gpu: %s failed: %s (%s)\n", what, mg_strerror(rc), mg_last_error());
  std::exit(1);
}

}  // namespace

int main(int argc, char** argv) {
  Config cfg;
  std::string cfg_path = "./../mirage/data/mirage.identifier.cfg";  // Configuration.h:22
  std::string query_override;
  int gpu = 0;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "-h" || a == "--help" || a == "-help" || a == "--h") {
      std::printf("mirage_gpu [-cfg file] [-input query.fasta] [-gpu N] [-<setting> <value> ...]\n");
      return 0;
    }
    if (a == "-cfg" && i + 1 < argc) {
      cfg_path = argv[++i];
      continue;
    }
    if (a == "-input" && i + 1 < argc) {
      query_override = argv[++i];
      continue;
    }
    if (a == "-gpu" && i + 1 < argc) {
      gpu = std::atoi(argv[++i]);
      continue;
    }
    cfg.args.push_back(a[0] == '-' ? lower(a) : a);
  }
  if (!cfg.load(cfg_path)) {
    std::fprintf(stderr, "Could not read configuration file: %s\n", cfg_path.c_str());
    return 1;
  }
  const int k = std::atoi(cfg.get("considerthreshold", "31").c_str());
  const bool first_only = cfg.get("output_firstresults_only", "1") != "0";
  const std::string reference = cfg.get("Reference", "", true);
  const std::string query = query_override.empty() ? cfg.get("Query", "", true) : query_override;
  const std::string out_path = cfg.get("OutputPath", ".");
  const float th_s = std::strtof(cfg.get("LogThreshold_HighSensitivity", "0.4").c_str(), nullptr);
  const float th_p = std::strtof(cfg.get("LogThreshold_HighPrecision", "1").c_str(), nullptr);
  const float th_b = std::strtof(cfg.get("LogThreshold_Balanced", "0.7").c_str(), nullptr);
  const int pct = std::atoi(cfg.get("Hashmap_Load_Hashmap_Percentage", "100").c_str());
  const std::string speed = lower(cfg.get("UltraFastMode", "sensitive"));
  const std::string mem = lower(cfg.get("Hashmap_Load_Reference_Memory_UsageMode", "extreme"));
  const bool save_db = cfg.get("output_save_hashmap_database", "1") != "0";
  // reads per mg_classify call: GPU_BatchReads (this program's own key) when given, else the
  // reference's GPU block size raised to at least 1,000,000 (the batched form's efficient size)
  const std::string gb = cfg.get("GPU_BatchReads", "");
  const uint64_t batch =
      gb.empty() ? std::max<uint64_t>(1000000, std::strtoull(cfg.get("Hardware_BlockSize_Default_GPU", "20000").c_str(), nullptr, 10))
                 : std::max<uint64_t>(1, std::strtoull(gb.c_str(), nullptr, 10));
  if (speed != "sensitive") {
    std::fprintf(stderr, "mirage_gpu: UltraFastMode '%s' is not supported (only Sensitive).\n", speed.c_str());
    return 1;
  }
  if (pct != 100) {
    std::fprintf(stderr, "mirage_gpu: Hashmap_Load_Hashmap_Percentage must be 100 (partial loading is random).\n");
    return 1;
  }
  if (mem != "extreme" && mem != "high")
    std::fprintf(stderr, "mirage_gpu: memory mode '%s' is served with the 'extreme' semantics.\n", mem.c_str());
  if (cfg.count("Reference") > 1) {
    std::fprintf(stderr, "mirage_gpu: one reference file or .mhm index is supported.\n");
    return 1;
  }
  auto t0 = std::chrono::steady_clock::now();
  char dir[4096];
  int rc = mg_make_results_dir(out_path.c_str(), dir, sizeof dir);
  if (rc) die("creating the results folder", rc);

  mg_index* ix = nullptr;
  if (ends_with(reference, ".mhm")) {
    rc = mg_open(reference.c_str(), k, gpu, &ix);
    if (rc) die("loading the hashmap", rc);
  } else {
    Seqs refs;
    if (!read_fasta(reference, gpu, &refs, true)) {
      std::fprintf(stderr, "Could not find or read fasta file: %s\n", reference.c_str());
      return 1;
    }
    std::vector<std::string> names;
    std::vector<const char*> np;
    for (auto& h : refs.headers) names.push_back(h.substr(1));
    for (auto& n : names) np.push_back(n.c_str());
    uint8_t* img = nullptr;
    uint64_t len = 0;
    // on the GPU; the host builder writes the same bytes when the device lacks the memory
    rc = mg_build_image_device(gpu, refs.bases.data(), refs.offs.data(), (uint32_t)names.size(), np.data(), nullptr, k,
                               0, &img, &len);
    if (rc == MG_ERR_OOM)
      rc = mg_build_image(refs.bases.data(), refs.offs.data(), (uint32_t)names.size(), np.data(), nullptr, k, 0, &img,
                          &len);
    if (rc) die("building the hashmap", rc);
    if (save_db) {
      std::string p = std::string(dir) + "/hashmap_" + base_name_no_ext(reference) + ".mhm";
      std::ofstream o(p, std::ios::binary);
      o.write((const char*)img, (std::streamsize)len);
    }
    rc = mg_open_image(img, len, k, gpu, &ix);
    mg_free(img);
    if (rc) die("loading the hashmap", rc);
  }
  mg_index_info info{};
  mg_index_get_info(ix, &info);
  std::vector<const char*> ref_headers(info.n_refs);
  std::vector<int32_t> taxids(info.n_refs);
  for (uint32_t r = 0; r < info.n_refs; r++) mg_index_reference(ix, r, &ref_headers[r], &taxids[r], nullptr);

  Seqs q;
  if (!read_fasta(query, gpu, &q, false)) {
    std::fprintf(stderr, "Could not find or read fasta file: %s\n", query.c_str());
    return 1;
  }
  mg_logs* logs = nullptr;
  rc = mg_logs_open(dir, pct == 100, th_s, th_b, th_p, &logs);
  if (rc) die("opening the result logs", rc);
  const uint64_t n = q.headers.size();
  auto t1 = std::chrono::steady_clock::now();
  uint64_t reported = 0;
  // Two result buffers: batch i+1 is classified into one while a writer thread logs batch i from
  // the other (LogMatrixResults / LogResultsToFileManager, Analyser.cpp:228-491, run off the
  // GPU's critical path). Batches are logged in order, one at a time.
  struct Buf {
    std::vector<mg_read_result> reads;
    std::vector<mg_candidate> cands;
    std::vector<uint64_t> offs, ids;
    std::vector<const char*> in_headers;
    uint64_t m = 0;
  } buf[2];
  std::thread writer;
  int write_rc = 0;
  uint64_t bi = 0;
  for (uint64_t b0 = 0; b0 < n; b0 += batch, bi++) {
    Buf& B = buf[bi & 1];  // last logged two batches ago; that writer was joined one batch ago
    const uint64_t b1 = std::min(n, b0 + batch), m = b1 - b0;
    B.m = m;
    B.offs.assign(m + 1, 0);
    for (uint64_t i = 0; i <= m; i++) B.offs[i] = q.offs[b0 + i] - q.offs[b0];
    B.reads.assign(m, mg_read_result{});
    B.cands.resize(std::max<uint64_t>(B.cands.size(), 8 * m + 1024));
    mg_batch bt{m, B.offs.data(), q.bases.data() + q.offs[b0]};
    mg_result res{B.reads.data(), B.cands.data(), B.cands.size(), 0};
    rc = mg_classify(ix, &bt, &res);
    if (rc == MG_ERR_OOM && res.n_cands > B.cands.size()) {
      B.cands.resize(res.n_cands);
      res = mg_result{B.reads.data(), B.cands.data(), B.cands.size(), 0};
      rc = mg_classify(ix, &bt, &res);
    }
    if (rc) die("classifying", rc);
    B.ids.resize(m);
    B.in_headers.resize(m);
    for (uint64_t i = 0; i < m; i++) {
      B.ids[i] = b0 + i;
      B.in_headers[i] = q.headers[b0 + i].c_str();
      reported += B.reads[i].reported;
    }
    if (writer.joinable()) writer.join();
    if (write_rc) die("writing the result logs", write_rc);
    writer = std::thread([&, bp = &B] {
      write_rc = mg_logs_write(logs, bp->reads.data(), bp->cands.data(), bp->m, bp->ids.data(), bp->in_headers.data(),
                               ref_headers.data(), taxids.data(), first_only ? 1 : 0);
    });
  }
  if (writer.joinable()) writer.join();
  if (write_rc) die("writing the result logs", write_rc);
  mg_logs_close(logs);
  auto t2 = std::chrono::steady_clock::now();
  const double a = std::chrono::duration<double>(t2 - t1).count(), all = std::chrono::duration<double>(t2 - t0).count();
  std::printf("Reads: %llu  assigned: %llu  analysis %.3f s (%.0f reads/s)  total %.3f s\nLogfile: %s/results_Raw.log\n",
              (unsigned long long)n, (unsigned long long)reported, a, a > 0 ? n / a : 0.0, all, dir);
  mg_close(ix);
  return 0;
}
