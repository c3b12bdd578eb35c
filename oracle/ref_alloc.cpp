// Test infrastructure: array allocation functions linked into the reference binaries built by
// oracle/Makefile (the reference sources are not changed).
//
// 1. Padding. Hashmap::LoadHashMapFromHashmapDB writes the last TOC entry's BufferSize one
//    element past its `new pair<...>[n]` array (Hashmap.cpp:509, 552-553); with a plain heap
//    that write corrupts the next chunk and the stock program crashes at random during index
//    load. 64 spare bytes per array absorb it without changing any value the program reads.
// 2. Zero fill. TPrepareGPUAnalysis reads flags of a freshly allocated `new bool[n]` that it
//    only partly clears (Analyser.cpp:2124-2135); zero-filled memory gives that read a defined
//    value (false), the value a fresh mapping would hold.
#include <cstdlib>
#include <new>

void* operator new[](std::size_t n) {
  void* p = std::calloc(n + 64, 1);
  if (!p) throw std::bad_alloc();
  return p;
}
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete[](void* p, std::size_t) noexcept { std::free(p); }
