// Shared pieces of the register/ballot form of the per-strand steps (mg_dual.cuh), which replace
// the sorts and scans over shared arrays of process_strand (mg_kernels.cuh) for reads of up to
// kLeanQ bases:
//
//   seeds / probe          one lane per seed; found index = popc of the found ballot below it
//   occurrence filter      per posting, the bitmask of found indices where its reference occurs;
//                          the longest run of set bits is that reference's occMax
//                          (Analyser.cpp:2057-2115)
//   sort (ref, pos, q)     rank sort of the kept postings (keys are distinct)
//   diagonal runs          run starts as a bit mask; run length = i - last start + 1
//                          (Analyser.cpp:2337-2490)
//   scoring                head/tail walks, coverage and scores in k_finish_dual (mg_lib.cu), from
//                          one record per run end (MatrixCPU.cpp:18-214)
#pragma once
#include "mg_kernels.cuh"

namespace mg {

constexpr int kLeanQ = 320;  // longest read of the register/ballot form

__device__ __forceinline__ int longest_run(uint32_t m) {
  int r = 0;
  while (m) {
    m &= m >> 1;
    r++;
  }
  return r;
}

}  // namespace mg
