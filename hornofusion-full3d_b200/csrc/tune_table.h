// Launch shapes measured on B200 by hornofusion-full3d_b200/autotune.py
// (tune_table.json beside it holds every measurement). Meshes that are not
// in a table fall back to the rules below.
#pragma once

namespace eaf {

struct TunedWidth {
  int nr, nth, nz, width;
};

// Lane width (blocks of 512 threads) of batched and served solves.
static constexpr TunedWidth kTunedWidths[] = {
    {12, 24, 16, 1},
    {18, 36, 24, 4},
    {35, 70, 50, 32},
    {60, 120, 84, 48},
};

inline int tuned_lane_width(int nr, int nth, int nz) {
  for (const TunedWidth& t : kTunedWidths)
    if (t.nr == nr && t.nth == nth && t.nz == nz) return t.width;
  const long long n = (long long)nr * nth * nz;
  long long w = (n + 16383) / 16384;  // about 32 cells per thread
  return (int)(w < 1 ? 1 : (w > 64 ? 64 : w));
}

struct TunedLaunch {
  int nr, nth, nz, block, grid, cluster, stream;
};

// (block, grid, blocks per cluster (1 = no clusters), flat-grid kernel:
// per-thread loads (0), bulk-copy streaming (1) or own cells kept in shared
// memory (2)) of the single-system persistent solver.
static constexpr TunedLaunch kTunedLaunches[] = {
    {12, 24, 16, 288, 16, 16, 0},
    {18, 36, 24, 512, 16, 16, 0},
    {35, 70, 50, 512, 148, 1, 2},
    {60, 120, 84, 512, 148, 1, 2},
    {120, 240, 168, 1024, 148, 1, 0},
};

// Most blocks a tuned launch of a mesh of at most `max_cells` cells can run
// (a grid is raised to one whole cluster at least); 0 if there is none.
constexpr int max_tuned_grid_up_to(long long max_cells) {
  int g = 0;
  for (const TunedLaunch& t : kTunedLaunches) {
    const int blocks = t.grid > t.cluster ? t.grid : t.cluster;
    if ((long long)t.nr * t.nth * t.nz <= max_cells && blocks > g) g = blocks;
  }
  return g;
}

inline bool tuned_single_launch(int nr, int nth, int nz, int* block, int* grid,
                                int* cluster = nullptr, int* stream = nullptr) {
  for (const TunedLaunch& t : kTunedLaunches)
    if (t.nr == nr && t.nth == nth && t.nz == nz) {
      *block = t.block;
      *grid = t.grid;
      if (cluster) *cluster = t.cluster;
      if (stream) *stream = t.stream;
      return true;
    }
  return false;
}

}  // namespace eaf
