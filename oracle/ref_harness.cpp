// Test infrastructure only: a driver around the UNMODIFIED MirAge CPU path.
//
// This program links the reference's own object files (compiled out of tree by
// oracle/Makefile from the reference sources; nothing is copied) and calls its
// hot-path entry points directly instead of going through
// Analyser::ExecuteAnalysis_MultiHardware:
//
//   Sequences::LoadInputFiles            Sequences.cpp:893   (FASTA query parse, uppercase,
//                                                             reverse complements, .mhm load)
//   Analyser::TPrepareGPUAnalysis        Analyser.cpp:1317   (seed lookup, occurrence filter,
//                                                             diagonal runs, keep rule)
//   MatrixCPU::CPUGetHighestScore        MatrixCPU.cpp:417   (dot-matrix scoring + relative score)
//   strand merge                         Analyser.cpp:592-611 (restated here, 12 lines)
//   Analyser::LogMatrixResults           Analyser.cpp:378    (the reference's own result logs)
//
// It dumps every intermediate the parity tests compare: per (read, strand) the kept candidate
// references with their diagonal runs, every candidate's Score / percentageMatch float bits,
// the relative scores and the merged per-read result.
//
// Job partitioning. TPrepareGPUAnalysis reuses one boolean flag array across all reads of a
// job and clears only its first n_found_seeds entries (Analyser.cpp:2135), so an entry of a
// later read can inherit a stale "keep" flag from an earlier read of the same job, and a
// freshly allocated array holds heap garbage. `--job 1` runs every strand as its own job and
// the operator new[] of oracle/ref_alloc.cpp hands out zeroed memory, which gives the per-read
// semantics that the restatement and the GPU path implement. `--job N` reproduces the stock
// program's grouping (N strands per job, forward/reverse pairs adjacent) so the size of that
// defect can be measured.
//
// `--scheme stock` times the stock program's own scheduling instead: numCores x 4 prepare
// workers (Analyser.cpp:3500-3503) over jobs of numQIDs_PerThread strands, where
// numQIDs_PerThread = 2 * max(1, n_reads / (numCores x 40 + 1)), made even (Analyser.cpp:
// 3712-3724), with the sample taken as one batch; numCores = std::thread::hardware_concurrency.
// Its candidate lists carry the stale-flag defect above, so it is a timing mode, not a dump mode.
//
// Usage:
//   mg_ref_harness --mhm X.mhm --reads R.fasta [--out dump.txt] [--job N] [--threads T]
//                  [--scheme stock] [--logdir DIR] [--time] [--limit NREADS]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <string>
#include <vector>
#include <map>
#include <set>
#include <unordered_map>
#include <unordered_set>
#include <iostream>
#include <fstream>
#include <sstream>
#include <algorithm>
#include <mutex>
#include <thread>
#include <future>
#include <atomic>
#include <chrono>
#include <memory>
#include <random>
#include <cmath>
#include <new>
#include <functional>
#include <iomanip>
#include <numeric>
#include <stdexcept>
#include <sys/stat.h>
#include <unistd.h>

// MatrixCPU keeps the per-candidate scores in private members; expose them for the dump.
#define private public
#define protected public
#include "Sequences.h"
#include "LogToScreen.h"
#include "Display.h"
#include "LogManager.h"
#include "Configuration.h"
#include "MultiNodePlatform.h"
#include "Files.h"
#include "Hardware.h"
#include "MultiThreading.h"
#include "Hashmap.h"
#include "SignalHandler.h"
#include "Screen.h"
#include "Analyser.h"
#include "MatrixCPU.h"
#undef private
#undef protected

// Array allocations are padded and zero-filled by oracle/ref_alloc.cpp (linked in).

// The objects the reference's own main() constructs (MirAge.cpp:70-98), wired the same way.
string Output_Path;
MultiThreading multiThreading;
LogToScreen lts;
LogToScreen logResultsToScreen;
LogManager logFileManagerHighSensitivity;
LogManager logFileManagerHighPrecision;
LogManager logFileManagerBalanced;
LogManager logFileManagerRaw;
Configuration configuration;
Display display(&lts, &configuration.Output_Mode);
Files files(&display);
Hardware hardware(&display, &multiThreading);
MultiNodePlatform multiNodePlatform(&display, &logFileManagerRaw, &files);
SignalHandler signalHandler(&display, &multiThreading);
Sequences sequences(&files, &display, &multiThreading, &multiNodePlatform,
                    &multiNodePlatform.combineResult_AllNodes);
Analyser analyser(&logResultsToScreen, &sequences, &multiThreading, &logFileManagerHighSensitivity,
                  &logFileManagerHighPrecision, &logFileManagerBalanced, &logFileManagerRaw,
                  &display, &hardware, &multiNodePlatform, &signalHandler, &configuration);
Hashmap hashmap(&display, &multiThreading, &multiNodePlatform, &sequences,
                &analyser.ConsiderThreshold, &logFileManagerRaw, &files, &configuration);

static uint32_t fbits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

struct Opts {
  std::string mhm, reads, out, logdir;
  size_t job = 1;
  int threads = 1;
  bool time_only = false;
  long limit = -1;
  int repeat = 1;
  int k = 31;
  bool first_only = true;
  bool parse_only = false;
  bool stock = false;
};

static void usage() {
  std::fprintf(stderr,
               "mg_ref_harness --mhm X.mhm --reads R.fasta [--out dump.txt] [--job N] "
               "[--threads T] [--logdir DIR] [--time] [--k 31] [--all-groups]\n");
  std::exit(2);
}

int main(int argc, char** argv) {
  Opts o;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) usage();
      return argv[++i];
    };
    if (a == "--mhm") o.mhm = next();
    else if (a == "--reads") o.reads = next();
    else if (a == "--out") o.out = next();
    else if (a == "--logdir") o.logdir = next();
    else if (a == "--job") o.job = std::stoul(next());
    else if (a == "--threads") o.threads = std::stoi(next());
    else if (a == "--time") o.time_only = true;
    else if (a == "--limit") o.limit = std::stol(next());
    else if (a == "--repeat") o.repeat = std::stoi(next());
    else if (a == "--k") o.k = std::stoi(next());
    else if (a == "--all-groups") o.first_only = false;
    else if (a == "--parse-only") o.parse_only = true;
    else if (a == "--scheme") {
      const std::string v = next();
      if (v == "stock") o.stock = true;
      else if (v != "job") usage();
    }
    else usage();
  }
  if (o.mhm.empty() || o.reads.empty()) usage();

  // Settings of data/mirage.identifier.cfg that touch the hot path (values set directly
  // instead of parsing the configuration file; MirAge.cpp:203-300 reads the same keys).
  configuration.Output_Mode = Output_Modes::Silent;
  analyser.ConsiderThreshold = o.k;
  analyser.Output_HighestScoredResultsOnly = o.first_only;
  Analyser::SpeedMode = Enum::Analysis_Modes::Sensitive;
  Hashmap::Hashmap_Load_Reference_Memory_UsageMode = Enum::Hashmap_MemoryUsageMode::Extreme;
  Hashmap::Use_Experimental_LazyLoading = true;
  Hashmap::Hashmap_Load_Hashmap_Percentage = 100;
  Hashmap::Hashmap_Load_Hashmap_Skip_On_Failure = false;
  sequences.SortQuerySequencesOnLoad = false;
  multiThreading.maxCPUThreads = 200000;
  multiThreading.SetGPUActive_NumberOfGPUs(0);  // AllGPUsActive() is then trivially true
  hardware.Type.push_back(Hardware::HardwareTypes::CPU);
  hardware.DeviceID.push_back(0);
  files.queryFilePath = o.reads;
  files.referenceFilePath = {o.mhm};
  LogManager::LogThreshold_HighSensitivity = 0.4f;
  LogManager::LogThreshold_HighPrecision = 1.0f;
  LogManager::LogThreshold_Balanced = 0.7f;

  bool logs = !o.logdir.empty() && !o.time_only;
  if (logs) {
    mkdir(o.logdir.c_str(), 0755);
    Output_Path = o.logdir;
    logFileManagerHighSensitivity.Open(&Output_Path[0], NULL, NULL, (char*)"HighSensitivity");
    logFileManagerBalanced.Open(&Output_Path[0], NULL, NULL, (char*)"Balanced");
    logFileManagerRaw.Open(&Output_Path[0], NULL, NULL, (char*)"Raw");
    logFileManagerHighPrecision.Open(&Output_Path[0], NULL, NULL, (char*)"HighPrecision");
    logFileManagerHighSensitivity.WriteOutputHeaders();
    logFileManagerBalanced.WriteOutputHeaders();
    logFileManagerRaw.WriteOutputHeaders();
    logFileManagerHighPrecision.WriteOutputHeaders();
  }

  auto t_load0 = std::chrono::steady_clock::now();
  sequences.LoadInputFiles(o.logdir.empty() ? std::string("/tmp") : o.logdir, &hashmap, false);
  analyser.ConsiderThreshold_HashmapLoaded = hashmap.GetLoadedThreshold();
  int32_t k = analyser.ConsiderThreshold_HashmapLoaded != -1 ? analyser.ConsiderThreshold_HashmapLoaded
                                                             : analyser.ConsiderThreshold;
  auto t_load1 = std::chrono::steady_clock::now();

  // --parse-only: the query file as the reference's loader parsed it (forward sequences, then
  // the headers), one "Q <length> <hex bytes>" / "H <hex bytes>" line each
  if (o.parse_only) {
    FILE* f = o.out.empty() ? stdout : std::fopen(o.out.c_str(), "w");
    const size_t nf = sequences.inputSequences->size() / 2;
    std::fprintf(f, "N %zu %zu\n", nf, sequences.inputHeaders.size());
    auto hex = [&](const char* p, size_t n) {
      for (size_t i = 0; i < n; i++) std::fprintf(f, "%02x", (unsigned char)p[i]);
    };
    for (size_t i = 0; i < nf; i++) {
      const std::vector<char>& q = (*sequences.inputSequences)[i];
      std::fprintf(f, "Q %zu ", q.size());
      hex(q.data(), q.size());
      std::fprintf(f, "\n");
    }
    for (auto* h : sequences.inputHeaders) {
      std::fprintf(f, "H ");
      hex(h->data(), h->size());
      std::fprintf(f, "\n");
    }
    if (f != stdout) std::fclose(f);
    return 0;
  }
  size_t n_reads = sequences.inputSequences->size() / 2;
  if (o.limit >= 0 && (size_t)o.limit < n_reads) n_reads = (size_t)o.limit;

  // Batch order of the stock program: read i then its reverse complement i + N
  // (Analyser.cpp:3736-3752), so batch slot 2j is forward and 2j+1 reverse.
  size_t n_total = sequences.inputSequences->size() / 2;
  std::vector<SEQ_ID_t> qids;
  qids.reserve(2 * n_reads);
  for (size_t i = 0; i < n_reads; i++) {
    qids.push_back((SEQ_ID_t)i);
    qids.push_back((SEQ_ID_t)(i + n_total));
  }
  size_t nq = qids.size();
  if (o.stock) {
    // Analyser.cpp:3500-3503 (workers) and 3712-3724 (strands per job)
    const size_t cores = std::max(1u, std::thread::hardware_concurrency());
    const size_t total_prepare = cores * 40 + 1;
    size_t per = std::max<size_t>(1, n_reads / total_prepare) * 2;
    per -= per % 2;
    o.job = per;
    o.threads = (int)(cores * 4);
  }

  // --time --repeat R: the hot path R times over the same reads (the index stays loaded);
  // one JSON line per repetition.
  const int reps = o.time_only ? std::max(1, o.repeat) : 1;
  for (int rep = 0; rep < reps; rep++) {
  Analyser::Analysis_Arguments* args = new Analyser::Analysis_Arguments();
  args->matchedReferencesPerQuery_CombiPositions_LastPositionInRange.resize(nq);
  args->matchedReferencesPerQuery_HeadTailSequences.resize(nq);
  args->matchedReferencesPerQuery_CombiPositions.resize(nq);
  args->matchedReferencesPerQuery_RefPositions.resize(nq);
  args->matchedReferencesPerQuery_QueryPositions.resize(nq);
  args->matchedReferencesPerQuery.resize(nq);
  args->querySequences.resize(nq);
  args->queryIDs.resize(nq);
  args->runningThreadsGPUPreAnalysis = 0;

  size_t job = std::max<size_t>(1, o.job);
  size_t n_jobs = (nq + job - 1) / job;
  std::vector<Analyser::PrepareGPU_Arguments*> jobs(n_jobs);
  for (size_t j = 0; j < n_jobs; j++) {
    auto* pg = new Analyser::PrepareGPU_Arguments();
    pg->AnalysisArguments = args;
    for (size_t q = j * job; q < std::min(nq, (j + 1) * job); q++) pg->QueryIDs.push_back(qids[q]);
    pg->ThreadResultID = j;
    pg->NumQIDs_PerThread = job;
    pg->ThreadID = 0;
    pg->sequences = &sequences;
    pg->DeviceID = 0;
    pg->ConsiderThreshold = k;
    pg->multiThreading = &multiThreading;
    pg->hardware = &hardware;
    pg->display = &display;
    jobs[j] = pg;
  }
  args->runningThreadsGPUPreAnalysis = (int)n_jobs;

  // Per-worker lookup caches, cleared after every job as TPrepareGPUAnalysis_Worker does
  // (Analyser.cpp:3391-3440).
  size_t n_files = Hashmap::HashmapFileLocations.size();
  std::atomic<size_t> next_job(0);
  auto t0 = std::chrono::steady_clock::now();
  auto worker = [&]() {
    std::vector<hashmap_MatchedHashStreamPos*> mhsp(n_files);
    for (size_t f = 0; f < n_files; f++) mhsp[f] = new hashmap_MatchedHashStreamPos();
    std::vector<hashmap_streams*> lazy;
    for (;;) {
      size_t j = next_job.fetch_add(1);
      if (j >= n_jobs) break;
      jobs[j]->MatchedHashStreamPos = &mhsp;
      jobs[j]->ReferenceHashMap_Lazy = &lazy;
      Analyser::TPrepareGPUAnalysis(jobs[j]);
      for (size_t f = 0; f < n_files; f++) mhsp[f]->clear();
      delete jobs[j];
    }
    for (auto* p : mhsp) delete p;
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < std::max(1, o.threads); t++) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  auto t1 = std::chrono::steady_clock::now();

  MatrixCPU mc(&display, &multiThreading);
  std::vector<MatrixResult> results = mc.CPUGetHighestScore(
      &args->querySequences, &sequences, true, 0, k, &args->matchedReferencesPerQuery,
      &args->matchedReferencesPerQuery_CombiPositions,
      &args->matchedReferencesPerQuery_CombiPositions_LastPositionInRange,
      &args->matchedReferencesPerQuery_HeadTailSequences, -1);
  auto t2 = std::chrono::steady_clock::now();

  // Per-strand results before the merge, for the dump.
  std::vector<MatrixResult> per_strand;
  if (!o.time_only) per_strand = results;

  // Strand merge, Analyser.cpp:592-611.
  std::sort(results.begin(), results.end(),
            [](const MatrixResult& a, const MatrixResult& b) { return a.QueryID < b.QueryID; });
  for (size_t i = 0; i + 1 < results.size(); i += 2) {
    MatrixResult* f = &results[i];
    MatrixResult* r = &results[i + 1];
    if (f->HighestScore < r->HighestScore) {
      *f = *r;
      f->QueryID = i;
    }
    r->HighestScore = 0;
  }
  // Top group per read, the selection LogMatrixResult makes (Analyser.cpp:404-425).
  std::vector<std::vector<SEQ_ID_t>> top(results.size());
  for (size_t i = 0; i < results.size(); i += 2) {
    MatrixResult& mr = results[i];
    if (mr.Scores.empty() || mr.HighestScore == 0) continue;
    for (auto& s : mr.Scores)
      if (s.score == mr.HighestScore) top[i].push_back(s.referenceID);
  }
  auto t3 = std::chrono::steady_clock::now();

  double prep_s = std::chrono::duration<double>(t1 - t0).count();
  double score_s = std::chrono::duration<double>(t2 - t1).count();
  double pick_s = std::chrono::duration<double>(t3 - t2).count();
  double load_s = std::chrono::duration<double>(t_load1 - t_load0).count();
  double total = prep_s + score_s + pick_s;
  std::fprintf(stderr,
               "{\"rep\": %d, \"reads\": %zu, \"job\": %zu, \"threads\": %d, \"load_s\": %.4f, \"prep_s\": %.4f, "
               "\"score_s\": %.4f, \"pick_s\": %.4f, \"hot_s\": %.4f, \"reads_per_s\": %.2f}\n",
               rep, n_reads, job, o.threads, load_s, prep_s, score_s, pick_s, total,
               total > 0 ? n_reads / total : 0.0);
  if (o.time_only) {
    delete args;
    continue;
  }

  if (logs) {
    // The reference's own log writer (Analyser.cpp:378-491).
    Output_Modes mode = Output_Modes::Silent;
    Analyser::LogMatrixResults(&results, -1, &args->queryIDs, &multiThreading, &sequences, &mode,
                               &logResultsToScreen, &logFileManagerHighSensitivity,
                               &logFileManagerHighPrecision, &logFileManagerBalanced,
                               &logFileManagerRaw, o.first_only);
    logFileManagerHighSensitivity.Flush();
    logFileManagerHighPrecision.Flush();
    logFileManagerBalanced.Flush();
    logFileManagerRaw.Flush();
  }

  if (!o.out.empty()) {
    FILE* f = std::fopen(o.out.c_str(), "w");
    if (!f) {
      std::perror("open dump");
      return 1;
    }
    std::fprintf(f, "# mgdump 1 k=%d reads=%zu job=%zu\n", k, n_reads, job);
    // Per strand: S <slot> <queryID> <len> <n_cand>
    //   C <refID> <n_runs> <score_bits> <pct_bits|-> then R <start.ref> <start.q> <last.ref> <last.q> per run
    //   H <highest_bits> <n_scores> then P <rel_bits> <refID> per scored candidate (refID order)
    size_t flat = 0;
    for (size_t s = 0; s < nq; s++) {
      auto& cands = args->matchedReferencesPerQuery[s];
      size_t L = args->querySequences[s]->size();
      std::fprintf(f, "S %zu %u %zu %zu\n", s, (unsigned)args->queryIDs[s], L, cands.size());
      for (size_t c = 0; c < cands.size(); c++) {
        float sc = mc.scoresFromThreads[flat + c];
        auto& st = args->matchedReferencesPerQuery_CombiPositions[s][c];
        auto& la = args->matchedReferencesPerQuery_CombiPositions_LastPositionInRange[s][c];
        if (sc > -1)
          std::fprintf(f, "C %u %zu %08x %08x\n", (unsigned)cands[c], st.size(), fbits(sc),
                       fbits(mc.percentageMatchFromThreads[flat + c]));
        else
          std::fprintf(f, "C %u %zu %08x -\n", (unsigned)cands[c], st.size(), fbits(sc));
        for (size_t r = 0; r < st.size(); r++)
          std::fprintf(f, "R %u %u %u %u\n", (unsigned)st[r].Reference, (unsigned)st[r].Query,
                       (unsigned)la[r].Reference, (unsigned)la[r].Query);
      }
      flat += cands.size();
      MatrixResult& mr = per_strand[s];
      std::fprintf(f, "H %08x %zu\n", fbits(mr.HighestScore), mr.Scores.size());
      for (auto& p : mr.Scores) std::fprintf(f, "P %08x %u\n", fbits(p.score), (unsigned)p.referenceID);
    }
    // Merged per read: M <read> <strand 0|1> <highest_bits> <n_top> <top refIDs...>
    for (size_t i = 0; i < results.size(); i += 2) {
      MatrixResult& mr = results[i];
      bool from_rc = per_strand[i].HighestScore < per_strand[i + 1].HighestScore;
      std::fprintf(f, "M %zu %d %08x %zu", i / 2, from_rc ? 1 : 0, fbits(mr.HighestScore),
                   top[i].size());
      for (auto r : top[i]) std::fprintf(f, " %u", (unsigned)r);
      std::fprintf(f, "\n");
    }
    std::fclose(f);
  }
  }  // repetitions
  return 0;
}
