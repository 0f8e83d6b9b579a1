// Randomised check of otm::RingOffsets: live allocations never overlap and stay inside the
// region; releases in any order reclaim the space; a region drained of allocations takes a
// full-size allocation again. Exit status 0 on success.
#include <cstdio>
#include <map>
#include <random>
#include <vector>

#include "otm_host_ring.h"

struct Live {
  size_t off, len;
  int64_t seq;
};

int main() {
  for (int trial = 0; trial < 200; trial++) {
    std::mt19937_64 rng(1234 + trial);
    const size_t cap = 64 * (1 + rng() % 400), align = 64;
    otm::RingOffsets ring(cap, align);
    std::vector<Live> live;
    size_t allocs = 0;
    for (int op = 0; op < 4000; op++) {
      const bool do_alloc = live.empty() || rng() % 100 < 55;
      if (do_alloc) {
        const size_t n = 1 + rng() % (cap / 3 + 1);
        size_t off = 0;
        int64_t seq = 0;
        if (!ring.alloc(n, &off, &seq)) continue;
        const size_t len = (n + align - 1) / align * align;
        if (off % align || off + len > cap) {
          std::printf("trial %d: allocation [%zu,+%zu) outside the region %zu\n", trial, off, len, cap);
          return 1;
        }
        for (const Live& l : live)
          if (off < l.off + l.len && l.off < off + len) {
            std::printf("trial %d: [%zu,+%zu) overlaps live [%zu,+%zu)\n", trial, off, len, l.off, l.len);
            return 1;
          }
        live.push_back(Live{off, len, seq});
        allocs++;
      } else {
        // mostly the oldest few (first come, first served), sometimes any
        const size_t k = rng() % 4 == 0 ? rng() % live.size() : rng() % std::min<size_t>(live.size(), 3);
        ring.release(live[k].seq);
        live.erase(live.begin() + k);
      }
    }
    for (const Live& l : live) ring.release(l.seq);
    size_t off = 0;
    int64_t seq = 0;
    if (ring.live() != 0 || !ring.alloc(cap, &off, &seq) || off != 0 || allocs == 0) {
      std::printf("trial %d: drained ring does not take a full-size allocation\n", trial);
      return 1;
    }
  }
  std::printf("ok\n");
  return 0;
}
