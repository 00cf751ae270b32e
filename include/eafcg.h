/*
 * eafcg.h -- C ABI of the B200 pressure-correction CG (libeafcg.so).
 *
 * Drop-in for the reference Jacobi-preconditioned CG
 *   subroutine cg_3d_mpi(aW, aE, aS, aN, aB, aT, aP, Su, phi, m,
 *                        max_iter, tol, residual, n_iter)
 *   (src/mod_solver_3d.f90:485-496), called once per SIMPLE outer iteration
 *   from solve_pressure_correction (src/mod_pressure_3d.f90:316-318).
 *
 * Array contract (every coefficient, Su and phi):
 *   Fortran real(dp) (-1:nr+2, -1:nth+2, -1:nz+2), column-major, r fastest;
 *   the pointer is element (-1,-1,-1); Fortran (i,j,k) sits at linear index
 *   (i+1) + (nr+4)*((j+1) + (nth+4)*(k+1)).  This is the reference
 *   workspace layout (src/mod_workspace.f90:24-27, src/mod_fields_3d.f90:265).
 * Reads the interior of the coefficients and Su, and phi's interior plus its
 * r/z halo cells that the 7-point stencil touches (the reference's first
 * matvec reads them); writes phi's interior and its four theta-halo columns
 * j = -1, 0, nth+1, nth+2 over the full i and k halo ranges, which is the
 * serial theta-periodic copy the reference applies before returning
 * (src/mod_solver_3d.f90:567, src/mod_mpi_topology.f90:303-311).
 *
 * Semantics follow cg_3d_mpi: relative residual ||r||/||Su|| with strict
 * `< tol` exit after the update; Jacobi z = r / max(|aP|, 1e-30);
 * breakdown exit when |p.q| < 1e-30; zero right-hand side (||Su|| < 1e-30)
 * returns residual 0 and n_iter 0 with phi's interior untouched. Not
 * reaching tol within max_iter is not an error. Scalar dots are reduced
 * on the device in a fixed order, so results are reproducible run to run
 * but not bit-identical to the reference's sequential sums.
 *
 * Every call is synchronous with respect to the host unless its name ends
 * in _async. One handle must not be used by two host threads at once.
 * The calling thread's current CUDA device is left as it was.
 */
#ifndef EAFCG_H
#define EAFCG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum eaf_status {
  EAF_OK = 0,
  EAF_ECUDA = 1,         /* a CUDA runtime call failed                     */
  EAF_EINVAL = 2,        /* bad argument (NULL pointer, size, tolerance)   */
  EAF_ENONFINITE = 3,    /* the residual came out NaN or Inf; it is still
                            returned (the caller propagates NaN, as
                            src/mod_pressure_3d.f90:322 does)              */
  EAF_ETIMEOUT = 4,      /* a bounded device or queue wait gave up         */
  EAF_EUNSUPPORTED = 5,  /* e.g. a decomposed (is_parallel) mesh           */
  EAF_ENOMEM = 6,        /* device or host allocation failed               */
  EAF_EADMIT = 7,        /* serving: run refused by the HBM budget         */
  EAF_EBUSY = 8,         /* serving: result not ready yet                  */
  EAF_ECLOSED = 9        /* serving: server shut down / run closed         */
};

/* Human-readable name of a status code (static storage). */
const char* eaf_status_string(int status);

/* Text of the last CUDA failure seen by this host thread. */
const char* eaf_last_error(void);

/* ---- single-system plain FP64 solver ----------------------------------- */
typedef struct eaf_cg* eaf_cg_t;

/* Creates a solver for one nr x nth x nz mesh on `device` (the whole theta x z
 * domain on one GPU). Allocates all device mirrors and Krylov workspace once;
 * replaces the per-call allocate/deallocate of r, z, pv, q
 * (src/mod_solver_3d.f90:505-507, 569). */
int eaf_cg_create(eaf_cg_t* out, int nr, int nth, int nz, int device);

/* Same, for a caller that still holds a decomposed mesh: is_parallel != 0
 * returns EAF_EUNSUPPORTED (there is no CPU fallback). Mirrors the
 * m%is_parallel switch of cg_3d_mpi's bounds() (src/mod_solver_3d.f90:574-586). */
int eaf_cg_create_mesh(eaf_cg_t* out, int nr, int nth, int nz, int is_parallel,
                       int device);

int eaf_cg_destroy(eaf_cg_t h);

/* The drop-in: host arrays in the reference layout (pinned memory is
 * faster but not required). Replaces the call at
 * src/mod_pressure_3d.f90:316-318; argument meaning as
 * src/mod_solver_3d.f90:485-496. */
int eaf_cg_solve_f64(eaf_cg_t h, const double* aW, const double* aE,
                     const double* aS, const double* aN, const double* aB,
                     const double* aT, const double* aP, const double* Su,
                     double* phi, int max_iter, double tol, double* residual,
                     int* n_iter);

/* Same contract with device pointers (same layout, on the handle's device).
 * Inputs are read and phi is written on the handle's stream. */
int eaf_cg_solve_f64_device(eaf_cg_t h, const double* aW, const double* aE,
                            const double* aS, const double* aN, const double* aB,
                            const double* aT, const double* aP, const double* Su,
                            double* phi, int max_iter, double tol,
                            double* residual, int* n_iter);

/* Mixed precision: FP32 Jacobi-PCG inner solves (FP32 coefficients, vectors
 * and dot accumulation) inside an FP64 iterative-refinement loop that keeps
 * Su, phi, the outer residual Su - A phi, the convergence norm and the pin
 * in FP64. Stops when ||Su - A phi|| / ||Su|| < tol or after max_outer
 * refinement steps; each inner solve stops at relative reduction inner_tol
 * or after max_inner iterations. n_iter returns the total inner iterations,
 * n_outer the refinement steps. No reference counterpart: this is a new
 * solver form behind the same array contract as eaf_cg_solve_f64. */
int eaf_cg_solve_mixed(eaf_cg_t h, const double* aW, const double* aE,
                       const double* aS, const double* aN, const double* aB,
                       const double* aT, const double* aP, const double* Su,
                       double* phi, int max_outer, int max_inner, double tol,
                       double inner_tol, double* residual, int* n_iter,
                       int* n_outer);
int eaf_cg_solve_mixed_device(eaf_cg_t h, const double* aW, const double* aE,
                              const double* aS, const double* aN,
                              const double* aB, const double* aT,
                              const double* aP, const double* Su, double* phi,
                              int max_outer, int max_inner, double tol,
                              double inner_tol, double* residual, int* n_iter,
                              int* n_outer);

/* Trace of the last mixed-precision solve: for each refinement step (at most
 * max_steps), three doubles -- the inner FP32 iterations of the step, the
 * reduction of the inner CG's recurred residual over the step, and the FP64
 * outer residual ||Su - A phi|| / ||Su|| after it. n_steps receives the
 * number of steps copied. No reference counterpart (diagnostics). */
int eaf_cg_mixed_trace(eaf_cg_t h, double* steps, int max_steps, int* n_steps);

/* Launch shape of the persistent kernel: threads per block and number of
 * co-resident blocks (0 = automatic). Used by the autotuner. */
int eaf_cg_set_launch(eaf_cg_t h, int block_threads, int grid_blocks);
int eaf_cg_get_launch(eaf_cg_t h, int* block_threads, int* grid_blocks);

/* Launch shape of the last solve (it fixes the association of the device
 * dot products; the oracle's kernel-order mode takes the same shape). */
int eaf_cg_last_launch(eaf_cg_t h, int* block_threads, int* grid_blocks);

/* Thread-block clusters for the plain FP64 solve (reference form): blocks
 * per cluster, 2..16, or 1 for none, or 0 for the tuned choice of the mesh.
 * On a cluster grid each all-reduce folds the blocks' partials through the
 * cluster leader's shared memory and only the leaders meet in global memory,
 * so the dot products are associated per cluster (the oracle's plan
 * (grid, block, cluster)); every other operation is unchanged. A size the
 * device cannot launch falls back to none. No reference counterpart: the
 * reference's dot is one sequential sum plus MPI_Allreduce
 * (src/mod_solver_3d.f90:607-618). eaf_cg_get_cluster reports the size the
 * next solve uses, eaf_cg_last_cluster the size the last one used. */
int eaf_cg_set_cluster(eaf_cg_t h, int cluster_blocks);
int eaf_cg_get_cluster(eaf_cg_t h, int* cluster_blocks);
int eaf_cg_last_cluster(eaf_cg_t h, int* cluster_blocks);

/* A launch that is ONE cluster (grid == cluster blocks) on a mesh that fits
 * the cluster's shared memory (about 28,000 cells at 16 blocks) runs, by
 * default, the cluster-resident kernel: the whole system lives in
 * distributed shared memory for the whole solve and an iteration touches no
 * global memory. resident = 1: its blocks signal their partials by a full
 * cluster barrier (default); 2: by remote mbarrier arrivals; 0: run the
 * global-memory cluster kernel instead. All give the same bits on one
 * launch. No reference counterpart. */
int eaf_cg_set_resident(eaf_cg_t h, int resident);

/* Kernel of the plain FP64 solve on a flat (cluster-free) grid: per-thread
 * loads (EAF_CG_KERNEL_LOADS), or each phase's operands staged in shared
 * memory by bulk copies a few tiles ahead of use (EAF_CG_KERNEL_STREAM),
 * or per-thread loads with a slot-polling all-reduce (EAF_CG_KERNEL_SLOTS),
 * or with the update operands kept in shared memory (EAF_CG_KERNEL_KEEP),
 * or the tuned choice of the mesh (EAF_CG_KERNEL_AUTO). All give the same
 * bits on the same launch shape. eaf_cg_last_kernel reports which ran. No
 * reference counterpart. */
#define EAF_CG_KERNEL_AUTO 0
#define EAF_CG_KERNEL_LOADS 1
#define EAF_CG_KERNEL_STREAM 2
/* per-thread loads, all-reduce by polling every block's partial in its slot
 * (the cluster all-reduce with clusters of one block) instead of an arrival
 * counter; same association, so the same bits as EAF_CG_KERNEL_LOADS */
#define EAF_CG_KERNEL_SLOTS 3
/* per-thread loads, with each block's own cells' x, r, aP and A p kept in
 * its shared memory for the whole solve, so the update phase reads only the
 * search direction from global memory; same arithmetic in the same order,
 * so the same bits as EAF_CG_KERNEL_LOADS. Runs where a block's slice fits
 * (4 doubles a cell, about 7,000 cells a block), else the per-thread-load
 * kernel does. */
#define EAF_CG_KERNEL_KEEP 4
int eaf_cg_set_kernel(eaf_cg_t h, int kernel);
int eaf_cg_last_kernel(eaf_cg_t h, int* kernel);

/* Line-by-line TDMA on the handle's mesh: replaces tdma_3d_mpi
 * (src/mod_solver_3d.f90:252-366, serial branch; callers in momentum,
 * energy, species, k-epsilon, DO radiation and continuity, e.g.
 * src/mod_momentum_3d.f90:329). n_sweep sweeps of Thomas line solves -- all r
 * lines, then all theta lines, then all z lines, theta halos refreshed
 * before each direction -- in the reference's Gauss-Seidel line order, so
 * phi comes out bit-identical to the sequential routine. The eight inputs
 * and phi are in the CG's halo layout; phi is updated in place (interior and
 * theta halos). Works on any linear operator (the transport equations are
 * not symmetric). n_sweep <= 0 leaves phi untouched. Returns EAF_OK,
 * EAF_ETIMEOUT (a bounded wait between lines gave up), EAF_EINVAL or
 * EAF_ECUDA. */
int eaf_tdma_3d_f64(eaf_cg_t h, const double* aW, const double* aE, const double* aS,
                    const double* aN, const double* aB, const double* aT,
                    const double* aP, const double* Su, double* phi, int n_sweep);
int eaf_tdma_3d_f64_device(eaf_cg_t h, const double* aW, const double* aE,
                           const double* aS, const double* aN, const double* aB,
                           const double* aT, const double* aP, const double* Su,
                           double* phi, int n_sweep);

/* Relative residual of a transport equation: replaces
 * compute_residual_3d_mpi (src/mod_solver_3d.f90:625-694, serial):
 * sqrt(sum r^2) / (sqrt(sum (|Su| + |aP phi| + SMALL)^2) + SMALL) over the
 * cells that are not identity rows, phi's halos read as stored. The two sums
 * are associated as the CG's dot products for the launch shape reported by
 * eaf_cg_last_launch (the reference sums sequentially). */
int eaf_residual_3d_f64(eaf_cg_t h, const double* aW, const double* aE, const double* aS,
                        const double* aN, const double* aB, const double* aT,
                        const double* aP, const double* Su, const double* phi,
                        double* residual);
int eaf_residual_3d_f64_device(eaf_cg_t h, const double* aW, const double* aE,
                               const double* aS, const double* aN, const double* aB,
                               const double* aT, const double* aP, const double* Su,
                               const double* phi, double* residual);

/* Post-CG corrections of the pressure-correction step: replaces the serial
 * code after the CG in solve_pressure_correction
 * (src/mod_pressure_3d.f90:333-397) with correct_velocities (:689-746):
 *   1. conservative face fluxes Fc = Fs + ac (pp_P - pp_nb) where linked
 *      (lk == 1) in non-solid cells; theta halos of Fc and lk refreshed;
 *   2. velocity corrections u -= (alpha V / aP_u) dpp/dx of the liquid in
 *      its active cells, then of the gas (has_gas) in its active cells;
 *   3. p = clamp(p + alpha_p pp, +-2e6) over the whole array;
 *   4. sealed cells (non-solid, neither phase active): p = mean of their
 *      active neighbours' p, 0 if none; theta halos of p refreshed.
 * Results are bit-identical to the serial Fortran (the clamp of a NaN p is
 * not pinned). Every 3-D array is in the CG's halo layout; r, theta and z
 * are the cell-centre coordinates with halo entries (n + 4 values from
 * index -1); int arrays are Fortran default integers/logicals (nonzero =
 * true). The gas fields may be NULL when has_gas is 0. */
typedef struct {
  const double* alpha;   /* volume fraction */
  const double* aP_ur;   /* momentum diagonals */
  const double* aP_uth;
  const double* aP_uz;
  double* ur;            /* velocities, corrected in place */
  double* uth;
  double* uz;
} eaf_phase_fields_t;

typedef struct {
  const double* pp;                       /* the CG solution */
  const double *Fs_r, *Fs_th, *Fs_z;      /* predicted face fluxes */
  const double *ac_r, *ac_th, *ac_z;      /* face links */
  double *Fc_r, *Fc_th, *Fc_z;            /* conservative fluxes, in/out */
  const double* vol;                      /* cell volumes */
  const double *r, *theta, *z;            /* cell centres, index -1..n+2 */
  double* p;                              /* pressure, in/out */
  eaf_phase_fields_t liq;
  eaf_phase_fields_t gas;
  int *lk_r, *lk_th, *lk_z;               /* face link flags (halos refreshed) */
  const int* cell_type;                   /* 0 = solid */
  const int *act_l, *act_g;               /* phase activity masks */
  int has_gas;                            /* gas phase in the pressure equation */
  double alpha_p;                         /* pressure under-relaxation */
} eaf_pcorr_fields_t;

/* Host arrays: uploads the fields to the handle's device mirror (allocated
 * on first use), corrects, downloads the in/out arrays. */
int eaf_pressure_correct_f64(eaf_cg_t h, const eaf_pcorr_fields_t* f);
/* Device arrays, corrected in place on the handle's stream (synchronised
 * before return). */
int eaf_pressure_correct_f64_device(eaf_cg_t h, const eaf_pcorr_fields_t* f);

/* Assembly of the pressure-correction equation: replaces the serial code of
 * solve_pressure_correction before the CG (src/mod_pressure_3d.f90:135-310):
 * cell pressure gradients of each phase (cell_gradients :621-651, the gas
 * one with the liquid-weight correction), the Rhie-Chow face contributions of
 * the liquid and, when it is in the equation, of the gas
 * (add_phase_contribution :469-619), the gas compressibility source, the
 * diagonal with compliance and acoustic terms, the boundary folding
 * (apply_pressure_bc, src/mod_boundary_3d.f90:180-277) and the continuity
 * residual sum|Su| / flux_ref. Outputs: aW..Su and pp (zeroed), the
 * liquid's exported face terms Fs_*, ac_* and link flags lk_* (Fc_* zeroed),
 * every array overwritten over the whole halo layout -- bit-identical to the
 * serial Fortran; the residual's two sums are associated per block (within
 * 1e-12 of the sequential sums). Activity masks and the liquid room are the
 * caller's (they come from the phase state). Fortran MAX/MIN on NaN are not
 * pinned. Layouts as eaf_pcorr_fields_t; `outlet` marks electrode holes on
 * the top layer (k = nz; out_mask of apply_pressure_bc). Arrays the switches
 * leave unread may be NULL: liq_room without liq_room_valid, liq_T and the
 * gas velocities and momentum diagonals without gas_in_poisson, gas alpha
 * and rho without either gas switch, gas_T_old without gas_compressibility.
 * Output arrays must not overlap input arrays. dt must be > 0; meshes up to
 * 2^31 halo elements (else EAF_EUNSUPPORTED). */
typedef struct {
  const double *alpha, *rho, *ur, *uth, *uz, *aP_ur, *aP_uth, *aP_uz;
} eaf_phase_state_t;

typedef struct {
  const int *cell_type, *outlet, *act_l, *act_g;
  const double *vol, *Ar, *Ath, *Az;
  const double *r, *theta, *z;            /* cell centres, index -1..n+2 */
  const double *p, *liq_room;
  eaf_phase_state_t liq, gas;
  const double *liq_T, *gas_T_old;
  int liq_room_valid;                     /* ws_liq_room_valid */
  int gas_in_poisson;                     /* gas_in_poisson .and. solve_multiphase */
  int gas_compressibility;                /* gas_compressibility .and. solve_multiphase */
  double dt, rho_gas, T_ambient, beta_expansion;
  double *aW, *aE, *aS, *aN, *aB, *aT, *aP, *Su, *pp;
  double *Fs_r, *Fs_th, *Fs_z, *ac_r, *ac_th, *ac_z, *Fc_r, *Fc_th, *Fc_z;
  int *lk_r, *lk_th, *lk_z;
} eaf_assembly_fields_t;

/* Host arrays (uploaded to the handle's mirror, outputs downloaded). */
int eaf_pressure_assemble_f64(eaf_cg_t h, const eaf_assembly_fields_t* f, double* residual);
/* Device arrays, assembled in place on the handle's stream. */
int eaf_pressure_assemble_f64_device(eaf_cg_t h, const eaf_assembly_fields_t* f,
                                     double* residual);

/* One whole pressure step: the serial numerics of solve_pressure_correction
 * (src/mod_pressure_3d.f90:135-397) -- this assembly, the CG of cg_3d_mpi
 * into f->pp with max_iter / tol (:316-318), then the post-CG corrections of
 * eaf_pressure_correct_f64 with under-relaxation alpha_p over the same
 * arrays (the gas is corrected when gas_in_poisson is set). Besides the
 * assembly's outputs it updates f->p and the velocities of the phases in the
 * equation IN PLACE (their pointers are written through). As the reference
 * (:320), the corrections run whatever the CG returns, and a NaN CG residual
 * replaces the continuity residual in *residual. *cg_res and *n_iter are the
 * CG's. Returns the CG's status (EAF_OK or EAF_ENONFINITE) or an error.
 * Every array is bit-identical to the serial Fortran when the CG's dot
 * products are associated as the kernel's (eaf_cg_last_launch). */
int eaf_pressure_step_f64(eaf_cg_t h, const eaf_assembly_fields_t* f, double alpha_p,
                          int max_iter, double tol, double* residual, double* cg_res,
                          int* n_iter);
int eaf_pressure_step_f64_device(eaf_cg_t h, const eaf_assembly_fields_t* f, double alpha_p,
                                 int max_iter, double tol, double* residual, double* cg_res,
                                 int* n_iter);

/* Multi-rank drop-in helpers (host-side index work, no device and no MPI):
 * an MPI-decomposed run (m%is_parallel) gathers its blocks onto one rank,
 * solves there on the GPU and scatters the solution back.
 *   eaf_mr_grid   the npr x npth x npz process grid for nprocs ranks
 *                 (factorize_3d, src/mod_mpi_topology.f90:157-204);
 *   eaf_mr_block  a block's extents and 1-based global start from its
 *                 Cartesian coordinates (decompose_domain, :209-250);
 *   eaf_mr_pack   (every rank) its interior, plus the two halo layers
 *                 beyond a physical r or z boundary it touches, of one local
 *                 array (-1:iloc+2, -1:jloc+2, -1:kloc+2) into a buffer of
 *                 eaf_mr_pack_count doubles;
 *   eaf_mr_place  (solving rank) that buffer into the global halo-layout
 *                 array (the gather_global_field pattern,
 *                 src/mod_parallel_utils.f90:92-111);
 *   eaf_mr_extract / eaf_mr_unpack  (solving rank / every rank) the block's
 *                 cells whose global r and z index lies in the domain (theta
 *                 periodic) -- interior and the halos that the final
 *                 26-neighbour exchange of cg_3d_mpi (:567) fills; halos beyond
 *                 a physical boundary keep their values -- eaf_mr_unpack_count
 *                 doubles.
 * grid, coords, loc and start are 3-vectors in (r, theta, z) order. */
int eaf_mr_grid(int nprocs, int nr, int nth, int nz, int grid[3]);
int eaf_mr_block(int nr, int nth, int nz, const int grid[3], const int coords[3], int loc[3],
                 int start[3]);
long long eaf_mr_pack_count(const int grid[3], const int coords[3], const int loc[3]);
long long eaf_mr_unpack_count(int nr, int nz, const int start[3], const int loc[3]);
int eaf_mr_pack(const double* local, const int grid[3], const int coords[3],
                const int loc[3], double* buf);
int eaf_mr_place(double* global, int nr, int nth, int nz, const int grid[3],
                 const int coords[3], const int loc[3], const int start[3],
                 const double* buf);
int eaf_mr_extract(const double* global, int nr, int nth, int nz, const int loc[3],
                   const int start[3], double* buf);
int eaf_mr_unpack(double* local, int nr, int nz, const int loc[3], const int start[3],
                  const double* buf);

/* Recurrences of the plain FP64 solve on this handle (eaf_cg_solve_f64 and
 * its _device form, and the CG inside eaf_pressure_step_f64):
 *   EAF_CG_FORM_REFERENCE      the reference's PCG recurrences
 *     (src/mod_solver_3d.f90:531-559), two group all-reduces per iteration;
 *     every per-cell value is the reference's, only the dot association
 *     differs (bit-identical to the oracle in the kernels' association);
 *   EAF_CG_FORM_ONE_REDUCTION  the same PCG rearranged (Chronopoulos-Gear)
 *     so that each iteration has ONE all-reduce; the same preconditioner,
 *     stencil, exit tests and NaN outcome, different rounding: it reaches the
 *     same tolerance in a few per cent more or fewer iterations.
 * No reference counterpart (the reference has one form). */
#define EAF_CG_FORM_REFERENCE 0
#define EAF_CG_FORM_ONE_REDUCTION 1
int eaf_cg_set_form(eaf_cg_t h, int form);
int eaf_cg_get_form(eaf_cg_t h, int* form);

/* Bound on every device-side barrier wait, in milliseconds (default 2000). */
int eaf_cg_set_timeout_ms(eaf_cg_t h, double ms);

/* Device time of the last solve (pack + solve + unpack) and of its solver
 * kernel alone, in milliseconds; 1 if the matrix was taken in the symmetric
 * 4-array form, 0 for the general 7-array form; kernels launched. */
int eaf_cg_last_timing(eaf_cg_t h, double* solve_ms, double* kernel_ms,
                       int* symmetric, int* kernels);

/* Device time of the last host-pointer solve from the first upload to the
 * end of the phi download, in milliseconds. */
double eaf_cg_last_e2e_ms(eaf_cg_t h);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their
 * own device work against the solver. */
void* eaf_cg_stream(eaf_cg_t h);

/* Pinned host memory helpers (cudaHostAlloc / cudaFreeHost). */
int eaf_host_alloc(void** ptr, size_t bytes);
int eaf_host_free(void* ptr);
/* Page-lock an existing host range for faster uploads (cudaHostRegister). */
int eaf_host_register(void* ptr, size_t bytes);
int eaf_host_unregister(void* ptr);

/* ---- batched solves ------------------------------------------------------ */
/* No reference counterpart: many independent pressure systems of uneven
 * mesh size solved in ONE persistent cooperative launch, replayed from a
 * CUDA graph. Each system is solved on a lane of blocks whose width depends
 * only on its mesh size (tuned table, or eaf_batch_set_width), so its
 * result is bit-identical whatever else is in the batch. Array contract per
 * system: that of eaf_cg_solve_f64. */
typedef struct eaf_batch* eaf_batch_t;
/* dims: 3*nsys ints, (nr, nth, nz) per system. Allocates all device state. */
int eaf_batch_create(eaf_batch_t* out, int nsys, const int* dims, int device);
int eaf_batch_destroy(eaf_batch_t b);
/* Lane width override for one system (0 = tuned width); replans. */
int eaf_batch_set_width(eaf_batch_t b, int sys, int width);
int eaf_batch_lane_width(eaf_batch_t b, int sys, int* width);
/* Plans lanes and queues (done by the first solve otherwise). */
int eaf_batch_plan(eaf_batch_t b, int* grid, int* block, int* nlanes);
/* Launch whose association a system's FP64 dot products follow (the
 * oracle's plan): its lane (width blocks of 512 threads) or, for a system of
 * at least 300,000 cells without an explicit width, the single-system
 * launch of its mesh: such systems run after the batched launch, one after
 * another over the whole GPU, in the same graph. */
int eaf_batch_system_plan(eaf_batch_t b, int sys, int* grid, int* block, int* cluster);
/* Host inputs of one system, uploaded on the batch stream (phi is the
 * warm start and, after a solve, is read back with eaf_batch_get_phi). */
int eaf_batch_set_system(eaf_batch_t b, int sys, const double* aW,
                         const double* aE, const double* aS, const double* aN,
                         const double* aB, const double* aT, const double* aP,
                         const double* Su, const double* phi);
/* Device inputs of one system: read in place by every later solve; phi is
 * updated in place. */
int eaf_batch_set_system_device(eaf_batch_t b, int sys, const double* aW,
                                const double* aE, const double* aS,
                                const double* aN, const double* aB,
                                const double* aT, const double* aP,
                                const double* Su, double* phi);
/* Solves every system: plain FP64 (mixed = 0; max_iter, tol as
 * eaf_cg_solve_f64) or mixed (mixed = 1; max_iter = inner iterations per
 * refinement step, max_outer refinement steps, inner_tol as
 * eaf_cg_solve_mixed). Returns EAF_OK, or the first non-OK system status
 * (EAF_ETIMEOUT first). */
int eaf_batch_solve(eaf_batch_t b, int mixed, int max_iter, double tol,
                    int max_outer, double inner_tol);
int eaf_batch_result(eaf_batch_t b, int sys, double* residual, int* n_iter,
                     int* n_outer, int* status);
int eaf_batch_get_phi(eaf_batch_t b, int sys, double* phi);
/* Device time of the last solve's persistent launch, milliseconds. */
double eaf_batch_last_ms(eaf_batch_t b);
void* eaf_batch_stream(eaf_batch_t b);

/* ---- serving loop --------------------------------------------------------- */
/* No reference counterpart. A host-side request loop for concurrent
 * simulated furnace runs: each run's state (coefficients, Krylov workspace,
 * and phi as the warm start) stays on the device between its solves; runs
 * are admitted against an HBM budget; requests are solved in batched
 * persistent launches (continuous batching: new requests go out in the next
 * batch as soon as a stream slot and blocks are free; two batches may be in
 * flight). A run's result does not depend on which other runs share its
 * batches. Thread-safe; a submitted request reads the caller's input arrays
 * until its ticket completes and writes phi_out (if not NULL) before. */
typedef struct eaf_srv* eaf_srv_t;
typedef struct {
  long long solves, batches, admitted_runs, refused_runs, active_runs;
  double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> completion latency */
  double solves_per_s;                     /* first submit to last completion */
  double mean_batch, used_bytes, budget_bytes;
} eaf_srv_stats_t;
enum { EAF_FAULT_DEVICE_LOST = 1 };

/* mixed = 0: plain FP64 (max_iter, tol as eaf_cg_solve_f64); mixed = 1:
 * max_iter inner iterations per refinement step, max_outer steps,
 * inner_tol (as eaf_cg_solve_mixed). max_batch bounds requests per batch. */
int eaf_srv_create(eaf_srv_t* out, int device, double hbm_budget_bytes,
                   int mixed, int max_iter, double tol, int max_outer,
                   double inner_tol, int max_batch);
/* Finishes every queued and in-flight request, then frees everything. */
int eaf_srv_destroy(eaf_srv_t s);
/* Admission: EAF_EADMIT if the run's device state would exceed the budget.
 * The run's warm start starts at zero. */
int eaf_srv_open_run(eaf_srv_t s, int nr, int nth, int nz, int* run_id);
/* EAF_EBUSY while the run has a request outstanding. */
int eaf_srv_close_run(eaf_srv_t s, int run_id);
/* One pressure solve for the run (reference halo-layout host arrays; phi_out
 * receives the solution in the same layout). EAF_EBUSY if the run already
 * has a request outstanding (SIMPLE is sequential per run). */
int eaf_srv_submit(eaf_srv_t s, int run_id, const double* aW, const double* aE,
                   const double* aS, const double* aN, const double* aB,
                   const double* aT, const double* aP, const double* Su,
                   double* phi_out, long long* ticket);
/* EAF_EBUSY until the request is done; then its result (once). */
int eaf_srv_poll(eaf_srv_t s, long long ticket, double* residual, int* n_iter,
                 int* n_outer, int* status);
/* Waits at most timeout_ms (EAF_ETIMEOUT otherwise). */
int eaf_srv_wait(eaf_srv_t s, long long ticket, double timeout_ms,
                 double* residual, int* n_iter, int* n_outer, int* status);
int eaf_srv_stats(eaf_srv_t s, eaf_srv_stats_t* st);
int eaf_srv_reset_stats(eaf_srv_t s);
/* Failure-detection hook: simulates the loss of the device in the server's
 * host logic (no GPU fault): queued and in-flight requests complete with
 * EAF_ECUDA and new work is refused with EAF_ECLOSED. */
int eaf_srv_inject_fault(eaf_srv_t s, int kind);

/* ---- no-allocation entry point ----------------------------------------- */
/* No counterpart in the reference. For callers that must not allocate
 * device memory: a simulator whose device memory is owned by its own pool
 * allocator or fixed budget, or code on a latency-critical path where
 * cudaMalloc/cudaFree would synchronise the device. Same contract and
 * result as eaf_cg_solve_f64_device (device pointers, reference layout),
 * but without a handle: all working memory is one static device array of
 * EAF_NOALLOC_MAX_CELLS cells' worth (about 3.5 MiB) that every GPU loading
 * the library holds until process exit. Larger meshes return EAF_EINVAL
 * (see eaf_last_error()). The array is shared by all calls on a device and
 * keeps the last call's contents; calls whose GPU work overlaps on one
 * device race, so serialise them. The first call on a device looks up the
 * array's device address and should come before any stream capture on
 * that device. `stream` is a cudaStream_t (NULL: the default stream); the
 * call returns after the stream has finished the solve. */
#define EAF_NOALLOC_MAX_CELLS 32768
int eaf_cg_solve_f64_noalloc(int nr, int nth, int nz, int device, void* stream,
                             const double* aW, const double* aE,
                             const double* aS, const double* aN,
                             const double* aB, const double* aT,
                             const double* aP, const double* Su, double* phi,
                             int max_iter, double tol, double* residual,
                             int* n_iter);

/* Self-test of the bounded barrier: launches two blocks that wait at a group
 * barrier whose arrival target can never be met, with the given bound. It
 * must return EAF_ETIMEOUT after about timeout_ms, with the device context
 * intact. No reference counterpart (failure-detection test hook). */
int eaf_selftest_barrier_timeout(int device, double timeout_ms);

/* Self-test of the bounded waits of the flat solver's release-free p.q
 * all-reduce. mode 0: two blocks of a group declared with three members,
 * so the arrival count never completes; mode 1: one block of a group of two
 * whose count is preset as if the other had arrived but whose slot is never
 * written, so the re-load of the missing partial never succeeds. Either must
 * return EAF_ETIMEOUT after about timeout_ms with the device context intact.
 * No reference counterpart (failure-detection test hook). */
int eaf_selftest_allreduce_timeout(int device, double timeout_ms, int mode);

/* Diagnostics (no reference counterpart): checks, on n generated operand
 * pairs (random over a wide exponent range, exact and near-halfway
 * quotients, zeros, infinities, NaN), that the division the TDMA sweeps use
 * (q = t*y refined by one FMA correction from y = 1/m) returns the same
 * bits as the IEEE division `/`; mismatches must be 0. */
int eaf_diag_div_check(int device, long long n, unsigned long long seed,
                       long long* mismatches, long long* fast_path);

/* Diagnostics (no reference counterpart): device time of one group
 * all-reduce of two sums -- block reduction, bounded group barrier, staging
 * and fold of the block partials -- averaged over `iters` in one cooperative
 * launch of blocks x threads, in form 0, 1 or 2 (full block barriers around
 * a counter barrier with three memory-ordering variants) or 3 (warp 0
 * exchanges while the other warps wait once on a named barrier; the form
 * the solvers use). All forms fold in the same order. */
int eaf_diag_allreduce_us(int device, int blocks, int threads, int iters,
                          int form, double* us_per_allreduce);

/* Library version string. */
const char* eaf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* EAFCG_H */
