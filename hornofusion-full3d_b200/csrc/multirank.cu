// Multi-rank drop-in: host-side index work that lets an MPI-decomposed run
// (m%is_parallel) use the single-GPU solvers. Every rank packs its block of
// the CG inputs, one rank assembles the global halo-layout arrays, solves on
// its GPU and returns each rank its block of the solution with the halos the
// reference's final exchange would have filled. No MPI here: the caller
// moves the buffers (MPI_Gatherv / MPI_Scatterv, or torch.distributed).
//
// Reference: the process grid (factorize_3d, src/mod_mpi_topology.f90:157-204),
// the block of each rank (decompose_domain, :209-250), the 26-neighbour halo
// exchange that closes cg_3d_mpi (:567; physical-boundary neighbours are
// MPI_PROC_NULL, theta periodic), and the gather-to-global pattern of
// gather_global_field (src/mod_parallel_utils.f90:92-111).
//
// Local arrays are Fortran (-1:iloc+2, -1:jloc+2, -1:kloc+2), column-major;
// global arrays (-1:nr+2, -1:nth+2, -1:nz+2), the CG's halo layout. Buffers
// hold one box each, r fastest.
#include <math.h>
#include <string.h>

#include "eafcg.h"

namespace {

struct Box {
  int i0, i1, j0, j1, k0, k1;  // inclusive local bounds
  long long count() const {
    return (long long)(i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1);
  }
};

inline long long lidx(const int loc[3], int i, int j, int k) {
  const long long sx = loc[0] + 4, sxy = sx * (loc[1] + 4);
  return (i + 1) + sx * (j + 1) + sxy * (k + 1);
}

bool valid_block(const int grid[3], const int coords[3], const int loc[3]) {
  for (int d = 0; d < 3; ++d) {
    if (grid[d] < 1 || coords[d] < 0 || coords[d] >= grid[d] || loc[d] < 1) return false;
  }
  return true;
}

// Box a rank sends: its interior, plus the two halo layers beyond a physical
// r or z boundary it touches (theta halos are rebuilt by the solve).
Box pack_box(const int grid[3], const int coords[3], const int loc[3]) {
  Box b;
  b.i0 = coords[0] == 0 ? -1 : 1;
  b.i1 = coords[0] == grid[0] - 1 ? loc[0] + 2 : loc[0];
  b.j0 = 1;
  b.j1 = loc[1];
  b.k0 = coords[2] == 0 ? -1 : 1;
  b.k1 = coords[2] == grid[2] - 1 ? loc[2] + 2 : loc[2];
  return b;
}

// Box a rank receives: every local cell whose global r and z index lies in
// the domain (theta is periodic, so all of -1..jloc+2), i.e. the interior and
// every halo cell the reference's final exchange fills from a neighbour;
// cells beyond a physical boundary keep their values.
Box unpack_box(int nr, int nz, const int start[3], const int loc[3]) {
  auto lo = [](int s) { return s >= 3 ? -1 : 2 - s; };            // global index >= 1
  auto hi = [](int s, int l, int n) { return n - s + 1 < l + 2 ? n - s + 1 : l + 2; };
  Box b;
  b.i0 = lo(start[0]);
  b.i1 = hi(start[0], loc[0], nr);
  b.j0 = -1;
  b.j1 = loc[1] + 2;
  b.k0 = lo(start[2]);
  b.k1 = hi(start[2], loc[2], nz);
  return b;
}

}  // namespace

extern "C" {

int eaf_mr_grid(int nprocs, int nr, int nth, int nz, int grid[3]) {
  if (nprocs < 1 || nr < 1 || nth < 1 || nz < 1 || !grid) return EAF_EINVAL;
  double best = 1.0e20;
  int bp = 1, bt = 1, bz = nprocs;
  for (int tp = 1; tp <= nprocs; ++tp) {
    if (nprocs % tp != 0) continue;
    for (int tt = 1; tt <= nprocs / tp; ++tt) {
      if ((nprocs / tp) % tt != 0) continue;
      if (nth % tt != 0) continue;
      const int tz = nprocs / (tp * tt);
      const double cr = (double)nr / tp, ct = (double)nth / tt, cz = (double)nz / tz;
      const double asp = fmax(cr / ct, ct / cr) * fmax(cr / cz, cz / cr) * fmax(ct / cz, cz / ct);
      if (asp < best) {
        best = asp;
        bp = tp;
        bt = tt;
        bz = tz;
      }
    }
  }
  grid[0] = bp;
  grid[1] = bt;
  grid[2] = bz;
  return EAF_OK;
}

int eaf_mr_block(int nr, int nth, int nz, const int grid[3], const int coords[3], int loc[3],
                 int start[3]) {
  if (!grid || !coords || !loc || !start) return EAF_EINVAL;
  const int n[3] = {nr, nth, nz};
  for (int d = 0; d < 3; ++d) {
    if (grid[d] < 1 || coords[d] < 0 || coords[d] >= grid[d] || n[d] < grid[d])
      return EAF_EINVAL;
    loc[d] = n[d] / grid[d];
    if (coords[d] == grid[d] - 1) loc[d] += n[d] % grid[d];
    start[d] = coords[d] * (n[d] / grid[d]) + 1;
  }
  return EAF_OK;
}

long long eaf_mr_pack_count(const int grid[3], const int coords[3], const int loc[3]) {
  if (!grid || !coords || !loc || !valid_block(grid, coords, loc)) return -1;
  return pack_box(grid, coords, loc).count();
}

long long eaf_mr_unpack_count(int nr, int nz, const int start[3], const int loc[3]) {
  if (!start || !loc || loc[0] < 1 || loc[1] < 1 || loc[2] < 1) return -1;
  return unpack_box(nr, nz, start, loc).count();
}

int eaf_mr_pack(const double* local, const int grid[3], const int coords[3],
                const int loc[3], double* buf) {
  if (!local || !buf || !grid || !coords || !loc || !valid_block(grid, coords, loc))
    return EAF_EINVAL;
  const Box b = pack_box(grid, coords, loc);
  long long o = 0;
  for (int k = b.k0; k <= b.k1; ++k)
    for (int j = b.j0; j <= b.j1; ++j)
      for (int i = b.i0; i <= b.i1; ++i) buf[o++] = local[lidx(loc, i, j, k)];
  return EAF_OK;
}

int eaf_mr_place(double* global, int nr, int nth, int nz, const int grid[3],
                 const int coords[3], const int loc[3], const int start[3],
                 const double* buf) {
  if (!global || !buf || !grid || !coords || !loc || !start || !valid_block(grid, coords, loc))
    return EAF_EINVAL;
  if (start[0] + loc[0] - 1 > nr || start[1] + loc[1] - 1 > nth || start[2] + loc[2] - 1 > nz)
    return EAF_EINVAL;
  const int gl[3] = {nr, nth, nz};
  const Box b = pack_box(grid, coords, loc);
  long long o = 0;
  for (int k = b.k0; k <= b.k1; ++k)
    for (int j = b.j0; j <= b.j1; ++j)
      for (int i = b.i0; i <= b.i1; ++i)
        global[lidx(gl, start[0] + i - 1, start[1] + j - 1, start[2] + k - 1)] = buf[o++];
  return EAF_OK;
}

int eaf_mr_extract(const double* global, int nr, int nth, int nz, const int loc[3],
                   const int start[3], double* buf) {
  if (!global || !buf || !loc || !start || loc[0] < 1 || loc[1] < 1 || loc[2] < 1)
    return EAF_EINVAL;
  if (start[0] < 1 || start[1] < 1 || start[2] < 1 || start[0] + loc[0] - 1 > nr ||
      start[1] + loc[1] - 1 > nth || start[2] + loc[2] - 1 > nz)
    return EAF_EINVAL;
  const int gl[3] = {nr, nth, nz};
  const Box b = unpack_box(nr, nz, start, loc);
  long long o = 0;
  for (int k = b.k0; k <= b.k1; ++k)
    for (int j = b.j0; j <= b.j1; ++j) {
      const int jg = ((start[1] + j - 2) % nth + nth) % nth + 1;  // periodic
      for (int i = b.i0; i <= b.i1; ++i)
        buf[o++] = global[lidx(gl, start[0] + i - 1, jg, start[2] + k - 1)];
    }
  return EAF_OK;
}

int eaf_mr_unpack(double* local, int nr, int nz, const int loc[3], const int start[3],
                  const double* buf) {
  if (!local || !buf || !loc || !start || loc[0] < 1 || loc[1] < 1 || loc[2] < 1)
    return EAF_EINVAL;
  const Box b = unpack_box(nr, nz, start, loc);
  long long o = 0;
  for (int k = b.k0; k <= b.k1; ++k)
    for (int j = b.j0; j <= b.j1; ++j)
      for (int i = b.i0; i <= b.i1; ++i) local[lidx(loc, i, j, k)] = buf[o++];
  return EAF_OK;
}

}  // extern "C"
