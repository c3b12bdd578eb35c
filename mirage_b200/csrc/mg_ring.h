// Host-side FIFO ring allocator for the served form's pinned request memory.
#pragma once
#include <cstdint>
#include <deque>

namespace mg {

// FIFO ring of pinned host memory: allocations at the head, releases in any order, space
// reclaimed in allocation order. Non-empty and head > tail: live bytes are [tail, head);
// head <= tail: they wrap, [tail, cap) + [0, head) (head == tail is full).
struct Ring {
  struct Entry {
    uint64_t at;
    bool freed;
  };
  uint8_t* base = nullptr;
  uint64_t cap = 0, head = 0, tail = 0;
  std::deque<Entry> live;
  bool alloc(uint64_t len, uint64_t* at) {
    len = (len + 15) & ~15ull;
    if (len > cap) return false;
    uint64_t pos;
    if (live.empty()) {
      head = tail = 0;
      pos = 0;
    } else if (head > tail) {
      if (cap - head >= len) pos = head;
      else if (tail >= len) pos = 0;  // wrap; [head, cap) stays unused until then
      else return false;
    } else {
      if (tail - head >= len) pos = head;
      else return false;
    }
    live.push_back(Entry{pos, false});
    head = pos + len;
    *at = pos;
    return true;
  }
  void release(uint64_t at) {
    for (Entry& e : live)
      if (e.at == at && !e.freed) {
        e.freed = true;
        break;
      }
    while (!live.empty() && live.front().freed) live.pop_front();
    tail = live.empty() ? head : live.front().at;
  }
};

}  // namespace mg
