// CPU check of the cluster V-cycle's host-side plan (cl_plan in otm_cluster.cuh) for the
// cluster size the library is built with: for many level stacks, every shared-memory region of a
// CTA lies inside the planned bytes and no two overlap, the z-slabs cover every plane once, the
// plane tables fit, and the ghost-copy rule of the kernel (a plane is the lower ghost of the CTA
// whose slab starts after it and the upper ghost of the CTA whose slab ends before it; at most two
// pushes per plane) feeds every ghost copy a CTA with planes reads. Host code only; prints "ok".
#include <algorithm>
#include <cstdio>
#include <utility>
#include <vector>

#include "otm_cluster.cuh"

using namespace otm;

static int fails = 0;
#define CHECK(c, ...)                  \
  do {                                 \
    if (!(c)) {                        \
      std::printf(__VA_ARGS__);        \
      std::printf("\n");               \
      fails++;                         \
    }                                  \
  } while (0)

static int wrapz(int z, int n) { return ((z % n) + n) % n; }

static void check_stack(Dims d0) {
  // the levels of the cluster part: halve while every axis is even, >= 8 and above 64 unknowns
  std::vector<Dims> dims;
  Dims d = d0;
  while (true) {
    dims.push_back(d);
    const bool can = d.nx % 2 == 0 && d.ny % 2 == 0 && d.nz % 2 == 0 && d.nx >= 8 && d.ny >= 8 && d.nz >= 8 &&
                     d.nv() > 64;
    if (!can) break;
    d = Dims{d.nx / 2, d.ny / 2, d.nz / 2};
  }
  if (dims.size() < 2) return;
  ClDesc cd{};
  const size_t bytes = cl_plan(dims.data(), int(dims.size()), &cd);
  if (bytes == 0) return;  // no plan: the per-level kernels run instead
  CHECK(bytes <= size_t(kMaxDynSmem), "%dx%dx%d: %zu bytes over the limit", d0.nx, d0.ny, d0.nz, bytes);
  const long words = long(bytes / sizeof(float));
  std::vector<std::pair<long, long>> regions;  // [begin, end) in floats
  auto add = [&](long off, long n, const char* what, int l) {
    if (off < 0) return;
    CHECK(off + n <= words, "%dx%dx%d level %d: %s ends past the plan", d0.nx, d0.ny, d0.nz, l, what);
    regions.push_back({off, off + n});
  };
  int tab_total = 0;
  for (int l = 0; l < cd.nlev; l++) {
    const ClLevel& V = cd.lv[l];
    const int nz = V.d.nz;
    CHECK(V.zstart[0] == 0 && V.zstart[kCl] == nz, "level %d: slabs do not cover [0, %d)", l, nz);
    int maxpl = 0;
    for (int c = 0; c < kCl; c++) {
      CHECK(V.zstart[c] <= V.zstart[c + 1], "level %d: slabs out of order", l);
      maxpl = std::max(maxpl, V.zstart[c + 1] - V.zstart[c]);
    }
    CHECK(V.cs >= maxpl * V.d.nx * V.d.ny, "level %d: case stride too small", l);
    CHECK(V.urs >= V.d.nx && V.ups >= V.urs * V.d.ny && V.ucs >= (maxpl + 2) * V.ups, "level %d: u strides", l);
    add(V.u_off, 3L * V.ucs, "u", l);
    add(V.f_off, 3L * V.cs, "f", l);
    add(V.r_off, 3L * V.cs, "r", l);
    add(V.st_off, 27L * V.cs, "stencils", l);
    add(V.inv_off, long(V.cs), "inverse diagonal", l);
    CHECK(V.tab_off == tab_total, "level %d: plane table offset", l);
    tab_total += 3 * nz;
    // ghost copies: pushes per plane (the kernel keeps at most two) and every read ghost fed
    for (int z = 0; z < nz; z++) {
      int k = 0;
      for (int q = 0; q < kCl; q++) {
        const int a = V.zstart[q], b = V.zstart[q + 1];
        if (a == b) continue;
        k += wrapz(a - 1, nz) == z;
        k += wrapz(b, nz) == z;
      }
      CHECK(k <= 2, "level %d plane %d feeds %d ghost copies", l, z, k);
    }
  }
  // the host-built plane tables (cl_tables): every plane's owner and local plane, and the ghost
  // copies it feeds, as restated here
  std::vector<int> tab;
  cl_tables(&cd, tab);
  CHECK(cd.ntab == tab_total && int(tab.size()) == tab_total, "plane tables: %d entries, %d expected", cd.ntab,
        tab_total);
  for (int l = 0; l < cd.nlev && int(tab.size()) == tab_total; l++) {
    const ClLevel& V = cd.lv[l];
    const int nz = V.d.nz;
    for (int z = 0; z < nz; z++) {
      int c = 0;
      while (V.zstart[c + 1] <= z) c++;
      CHECK(tab[V.tab_off + z] == ((c << 16) | (z - V.zstart[c])), "level %d plane %d: owner entry", l, z);
      std::vector<int> want;
      for (int q = 0; q < kCl; q++) {
        const int a = V.zstart[q], b = V.zstart[q + 1];
        if (a == b) continue;
        if (wrapz(a - 1, nz) == z) want.push_back((q << 16) | 0);
        if (wrapz(b, nz) == z) want.push_back((q << 16) | (b - a + 1));
      }
      while (want.size() < 2) want.push_back(-1);
      const int* push = tab.data() + V.tab_off + nz + 2 * z;
      CHECK(push[0] == want[0] && push[1] == want[1], "level %d plane %d: ghost pushes", l, z);
    }
  }
  add(cd.gather_off, 3L * cd.nc, "coarsest gather", -1);
  add(cd.tab_base, long(tab_total), "plane tables", -1);
  CHECK(tab_total <= kClMaxTab, "plane tables: %d entries", tab_total);
  std::sort(regions.begin(), regions.end());
  for (size_t i = 1; i < regions.size(); i++)
    CHECK(regions[i].first >= regions[i - 1].second, "%dx%dx%d: shared-memory regions overlap", d0.nx, d0.ny,
          d0.nz);
}

int main() {
  for (int nx = 4; nx <= 32; nx += 2)
    for (int ny = 4; ny <= 32; ny += 2)
      for (int nz = 4; nz <= 32; nz += 2)
        if (size_t(nx) * ny * nz <= size_t(kClMaxNv)) check_stack(Dims{nx, ny, nz});
  if (fails) {
    std::printf("%d failures\n", fails);
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
