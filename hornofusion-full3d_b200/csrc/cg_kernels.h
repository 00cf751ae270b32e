// Internal launch interface between the C-ABI shim (api.cu) and the kernel
// translation units. Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "cg_common.cuh"
#include "eafcg.h"

namespace eaf {

// Held around "set a kernel's dynamic shared memory size, then launch it or
// query its occupancy": the size is an attribute of the function, so two
// host threads (a server's worker and a caller's solve) that launch one
// kernel with different sizes must not interleave the two steps.
std::mutex& launch_attr_mutex();


// Written by the solver kernel (block 0, thread 0) at the end of a solve.
struct SolveResult {
  int status;      // EAF_OK, EAF_ENONFINITE or EAF_ETIMEOUT
  int n_iter;      // CG iterations (mixed form: total inner iterations)
  int n_outer;     // refinement steps (mixed form), 0 for the plain form
  int sym;         // 1 = symmetric 4-array operator, 0 = general 7-array
  double residual; // final relative residual
  double bnorm;    // ||Su||
};

// Halo-layout inputs of one solve (the reference workspace arrays).
struct HaloInputs {
  const double* aW;
  const double* aE;
  const double* aS;
  const double* aN;
  const double* aB;
  const double* aT;
  const double* aP;
  const double* Su;
  const double* phi;
};

// Compact-layout device state of one system (interior cells only).
struct SysF64 {
  double *aP, *aE, *aN, *aT;  // symmetric form: aW, aS, aB are implied
  double *aW, *aS, *aB;       // general form only
  double *b, *x, *r, *q;
  double *p, *p2;             // search direction, double-buffered by iteration
  double *z;                  // preconditioned residual r / max(|aP|, SMALL)
  double *s0, *s1;            // single-reduction form: s = A p, double-buffered
  double *dinv;               // single-reduction form: 1 / max(|aP|, SMALL)
  int* asym;                  // pack: number of link pairs that disagree
};

// FP32 shadow of a system for the mixed-precision inner solve.
struct SysF32 {
  float *aP, *aE, *aN, *aT, *aW, *aS, *aB;
  float *r, *z, *q, *e;  // inner residual, r / max(|aP|, SMALL), A p, correction
  float *p, *p2;         // direction, double-buffered by inner iteration
};

struct GroupWs {
  double* part;                 // block partials, [slots][blocks]
  unsigned long long* counter;  // barrier arrival counter (zeroed per launch)
  int* err;                     // shared error word (zeroed per launch)
  SolveResult* result;
};

MeshDims make_dims(int nr, int nth, int nz);


// pack: halo layout -> compact layout, symmetry check, FP64 initial
// residual r = Su - A phi with the reference stencil (phi's theta halo
// wrapped, its r/z halo cells read as given).
cudaError_t launch_pack_f64(const MeshDims& d, const HaloInputs& in,
                            const SysF64& s, cudaStream_t st);
// unpack: compact x -> phi interior + theta-halo columns over the full i, k
// halo ranges (phi's r/z halo cells are left as they are).
cudaError_t launch_unpack_f64(const MeshDims& d, const double* x, double* phi,
                              cudaStream_t st);
// Persistent cooperative plain-FP64 Jacobi-PCG.
cudaError_t launch_cg_f64(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                          int max_iter, double tol, uint64_t timeout_ns,
                          int grid, int block, cudaStream_t st);
// The single-system kernel variant that runs blocks of `block` threads on
// an n-cell mesh. The 1024-thread variant prefetches into L2 ahead of its
// load rounds when the mesh's working set (128 B a cell) is larger than the
// L2 can hold alongside it (l2_prefetch_pays): at 64 registers it has too
// few loads in flight to keep HBM busy on its own. All variants give the
// same bits for one launch shape.
bool l2_prefetch_pays(long long n);
const void* cg_f64_kernel_ptr(int block, long long n);
// The same solver with each phase's operands staged in shared memory by
// bulk copies a few tiles ahead (symmetric operators; the 7-array form runs
// per-thread loads in the same kernel); bit-identical to cg_f64_kernel on
// the same launch. Blocks a multiple of 32 threads; stream_stages() says
// how many tiles are in flight (0: the mesh's rows are too long for it).
cudaError_t launch_cg_f64_stream(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                                 int max_iter, double tol, uint64_t timeout_ns, int grid,
                                 int block, cudaStream_t st);
int stream_stages(int block, int nr);
int stream_max_coresident(int block, int nr, int sms);
// The same solver with each block's own cells' x, r, aP and q kept in its
// shared memory for the whole solve (4 doubles a cell, dynamic shared
// memory of keep_smem_bytes); bit-identical to cg_f64_kernel on the same
// launch. keep_max_coresident: blocks of that launch the device can hold at
// once (0: the slice does not fit).
cudaError_t launch_cg_f64_keep(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                               int max_iter, double tol, uint64_t timeout_ns, int grid,
                               int block, cudaStream_t st);
size_t keep_smem_bytes(long long n, int grid);
int keep_max_coresident(int block, long long n, int grid, int sms);
// The same solver on a grid of thread-block clusters of `cluster` blocks
// (2..16; grid a multiple of it, at most 128 clusters): its all-reduces fold
// through the leader block's shared memory in each cluster and a global
// stage among the leaders only (cluster_red.cuh). `slots` holds at least
// cluster_slot_doubles(grid / cluster) doubles (the handle's partial table
// serves). Returns cudaErrorInvalidValue for a shape it cannot run.
cudaError_t launch_cg_f64_cluster(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                                  double* slots, size_t slot_doubles, int max_iter,
                                  double tol, uint64_t timeout_ns, int grid, int block,
                                  int cluster, cudaStream_t st);
// Clusters of `cluster` blocks of `block` threads that can be resident at
// once (0 if the size cannot be launched).
int max_active_clusters(int block, long long n, int cluster);
// The same solve on ONE cluster of `cluster` blocks whose shared memory holds
// the whole system for the whole solve (cg_dsm.cu); bit-identical to the
// cluster kernel on the launch (cluster, block, cluster). Meshes of at most
// dsm_max_cells(cluster) cells (about 28,000 at 16 blocks on B200).
// `signal` picks how a block signals its partials: kDsmSignalClusterBarrier
// (a full cluster barrier, default: measured faster) or kDsmSignalMbarrier
// (remote mbarrier arrivals).
constexpr int kDsmSignalClusterBarrier = 1;
constexpr int kDsmSignalMbarrier = 2;
cudaError_t launch_cg_f64_dsm(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                              int max_iter, double tol, int block, int cluster,
                              cudaStream_t st, int signal = kDsmSignalClusterBarrier,
                              uint64_t timeout_ns = 2000000000ull);
int dsm_max_cells(int cluster);
// Whether one cluster of `cluster` blocks of `block` threads holding an
// n-cell system can be resident on the current device.
bool dsm_can_launch(long long n, int block, int cluster);

// Launch of a persistent single-system solver: blocks, threads per block,
// blocks per thread-block cluster (1 = none).
struct SolverLaunch {
  int grid, block, cluster;
  int stream = 0;  // 1: the bulk-copy streaming kernel (flat grids only)
  int slots = 0;   // 1: flat grid, slot-polling all-reduce (clusters of one)
  int keep = 0;    // 1: flat grid, own cells kept in shared memory
};
// The launch a handle with the requested shape (0 = automatic) uses on an
// nr x nth x nz mesh (api.cu): the tuned shape, else the fallback rules,
// with the cluster size and grid clamped to what the device can run.
SolverLaunch choose_launch(int nr, int nth, int nz, int sms, int req_block, int req_grid,
                           int req_cluster, int form, bool f64, int req_kernel = 0);
// Whether the plain FP64 solve on launch L runs the cluster-resident kernel.
bool runs_resident(const SolverLaunch& L, long long n, bool allowed);
// Enqueues the plain FP64 solver (reference form) on launch L: the flat,
// cluster or cluster-resident kernel; `slot_doubles` is the size of ws.part.
// `resident`: 0 never the cluster-resident kernel, 1 it with cluster-barrier
// signalling, 2 it with mbarrier signalling.
cudaError_t launch_f64_solver(const SolverLaunch& L, int resident, const MeshDims& d,
                              const SysF64& s, const GroupWs& ws, size_t slot_doubles,
                              int max_iter, double tol, uint64_t timeout_ns, cudaStream_t st);
// Single-reduction (Chronopoulos-Gear) form of the same PCG: one group
// all-reduce per iteration; uses s0/s1 and reuses r, z, q, p2 as the
// double-buffered r and w = A M^-1 r.
cudaError_t launch_cg1_f64(const MeshDims& d, const SysF64& s, const GroupWs& ws,
                           int max_iter, double tol, uint64_t timeout_ns, int grid, int block,
                           cudaStream_t st);
const void* cg1_f64_kernel_ptr(int block);




// Mixed precision (cg_mixed.cu).
// `trace` (nullable, 3 * max_outer doubles) receives per refinement step the
// inner iterations, the inner CG's residual reduction and the outer residual.
cudaError_t launch_cg_mixed(const MeshDims& d, const SysF64& s, const SysF32& f,
                            const GroupWs& ws, int max_outer, int max_inner,
                            double tol, double inner_tol, uint64_t timeout_ns,
                            int grid, int block, cudaStream_t st, double* trace = nullptr);
const void* cg_mixed_kernel_ptr();

// ---------------------------------------------------------------------------
// Batched launch: independent systems, one persistent cooperative launch.
// Blocks are split into lanes of consecutive blocks; a lane solves the
// systems of its queue one after another with a lane-local group barrier.
// A system's reduction order depends only on its lane width and the block
// size, never on the rest of the batch.
// ---------------------------------------------------------------------------
struct BatchSys {
  MeshDims d;
  SysF64 s;
  SysF32 f;
  SolveResult* result;
};

struct BatchTables {
  const BatchSys* sys;          // [nsys]
  const int* lane_of_block;     // [grid]
  const int* lane_first_block;  // [nlanes]
  const int* lane_width;        // [nlanes]
  const int* lane_q_begin;      // [nlanes + 1], offsets into queue
  const int* queue;             // system ids, lane by lane
  unsigned long long* counters; // [nlanes * kCounterStride]
  double* parts;                // [8 * grid]: lane L uses [8*first, 8*(first+width))
  int* err;                     // shared error word
};
constexpr int kCounterStride = 16;  // 128 bytes between lane counters

cudaError_t launch_batch_f64(const BatchTables& t, int grid, int block, int max_iter,
                             double tol, uint64_t timeout_ns, cudaStream_t st);
cudaError_t launch_batch_mixed(const BatchTables& t, int grid, int block,
                               int max_outer, int max_inner, double tol,
                               double inner_tol, uint64_t timeout_ns, cudaStream_t st);
const void* batch_f64_kernel_ptr();
// Line-by-line TDMA sweeps (tdma_3d_mpi, serial) on halo-layout arrays, in
// place on phi; `mbox` holds tdma_mailbox_doubles() doubles of line
// hand-over slots. One cooperative launch of tdma_grid() warps; every mesh
// extent at most 1024.
// `fac` holds tdma_factor_doubles() doubles of line factors (computed by the
// launch from the coefficients).
size_t tdma_mailbox_doubles(int nr, int nth, int nz);
size_t tdma_factor_doubles(int nr, int nth, int nz);
int tdma_grid(int nr, int nth, int nz);
cudaError_t launch_tdma_f64(const HaloInputs& in, double* phi, int nr, int nth, int nz,
                            int n_sweep, double* mbox, double* fac, const GroupWs& ws,
                            uint64_t timeout_ns, cudaStream_t st);
const void* tdma_kernel_ptr();
// compute_residual_3d_mpi (serial) into ws.result->residual.
cudaError_t launch_residual_f64(const HaloInputs& in, const double* phi, const MeshDims& d,
                                const GroupWs& ws, uint64_t timeout_ns, int grid, int block,
                                cudaStream_t st);
const void* residual_kernel_ptr();
// Counts[0] = pairs where the TDMA's reciprocal-corrected division differs
// from `/` in any bit, counts[1] = pairs that took its fast path.
cudaError_t run_div_check(long long n, unsigned long long seed, unsigned long long* counts,
                          cudaStream_t st);

// Post-CG corrections (solve_pressure_correction after the CG), three
// launches on `st`; every pointer of `f` is a device pointer.
cudaError_t launch_pcorr_f64(const eaf_pcorr_fields_t& f, int nr, int nth, int nz,
                             cudaStream_t st);

// Pressure-equation assembly (solve_pressure_correction before the CG), three
// launches on `st` into device pointers of `f`; `scratch` holds
// assembly_scratch_doubles() doubles (gradients, block partials, and the
// residual at assembly_result()).
size_t assembly_scratch_doubles(int nr, int nth, int nz);
cudaError_t launch_assemble_f64(const eaf_assembly_fields_t& f, int nr, int nth, int nz,
                                double* scratch, cudaStream_t st);
const double* assembly_result(double* scratch, int nr, int nth, int nz);

// Threads per block of the batched kernels (FP64 and mixed).
constexpr int kBatchBlock = 512;
const void* batch_mixed_kernel_ptr();

// Barrier self-test (api.cu).
cudaError_t launch_barrier_selftest(const GroupWs& ws, uint64_t timeout_ns,
                                    cudaStream_t st);
// Self-test of the release-free p.q all-reduce's waits (cg_f64.cu): ws.part
// holds at least 16 doubles.
cudaError_t launch_allreduce_selftest(const GroupWs& ws, uint64_t timeout_ns, int mode,
                                      cudaStream_t st);

}  // namespace eaf
