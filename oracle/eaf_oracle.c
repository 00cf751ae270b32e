/*
 * eaf_oracle.c -- the oracle. TEST INFRASTRUCTURE ONLY: it checks the CUDA
 * path and times the CPU baseline; the product never links or calls it.
 *
 * A plain-C restatement of the reference Jacobi-preconditioned CG
 * `cg_3d_mpi` (src/mod_solver_3d.f90:485-620), serial branch
 * (m%is_parallel = .false.), FP64, in the reference's own data layout:
 * every array is Fortran `real(dp) (-1:nr+2, -1:nth+2, -1:nz+2)`,
 * column-major with r fastest, so Fortran (i,j,k) sits at linear index
 * (i+1) + (nr+4)*((j+1) + (nth+4)*(k+1)).
 *
 * Followed line by line:
 *   - allocation + zeroing of r, z, pv, q ............ mod_solver_3d.f90:505-507
 *   - r = Su - A*phi (matvec refreshes phi's halos) .. :510-513
 *   - bnorm = sqrt(dot(Su,Su)); early return ......... :515-521
 *   - z = r / max(|aP|, SMALL); pv = z (whole array) . :523-526
 *   - rz = dot(r,z); residual = ||r||/bnorm .......... :527-530
 *   - loop: matvec, pq, |pq|<SMALL exit, alpha,
 *     phi/r updates, residual < tol exit (strict,
 *     after the update, before preconditioning),
 *     z, rz_new, beta = rz_new/max(rz,SMALL), pv ..... :532-559
 *   - final halo exchange of phi ...................... :567
 *   - matvec: halo exchange, y = 0 everywhere, stencil  :588-605
 *   - dot: sequential sum over the interior section ... :607-618
 *   - serial theta-periodic halo copy ................. src/mod_mpi_topology.f90:303-311
 *   - SMALL = 1e-30 ................................... src/mod_constants.f90:53
 *
 * Fortran `sum(a*b)` over the section is a sequential sum in column-major
 * order (k outer, i inner); gfortran at the reference's default -O2 (no
 * -march, so no FMA on x86-64) neither reassociates nor contracts it. This
 * file is built with -ffp-contract=off for the same reason.
 * `max(x, SMALL)` is written `x > SMALL ? x : SMALL`, the same expression the
 * CUDA kernels use (a NaN x selects SMALL in both).
 *
 * The same file restates two more routines of that module, serial branch:
 *   - tdma_3d_mpi, line-by-line TDMA sweeps ......... src/mod_solver_3d.f90:252-366
 *     with the 1D Thomas solve `tdma` .............. src/mod_solver_3d.f90:22-46
 *   - compute_residual_3d_mpi ....................... src/mod_solver_3d.f90:625-694
 * (see eaf_oracle_tdma_3d and eaf_oracle_residual_3d below), and the serial
 * post-CG corrections of solve_pressure_correction
 *   - flux export, halo refresh, velocity and pressure corrections, sealed
 *     cells ..................................... src/mod_pressure_3d.f90:333-397
 *   - correct_velocities ........................ src/mod_pressure_3d.f90:689-746
 * (eaf_oracle_pressure_correct), and the assembly before the CG
 *   - masks in, gradients, phase contributions, compressibility, aP,
 *     boundary folding, continuity residual .... src/mod_pressure_3d.f90:135-310
 *     (cell_gradients :621-651, add_phase_contribution :469-619, helpers
 *     :405-458, :654-681; pgrad src/mod_constants.f90:274-287;
 *     apply_pressure_bc src/mod_boundary_3d.f90:180-277)
 * (eaf_oracle_pressure_assemble). It also restates the single-reduction
 * (Chronopoulos-Gear) rearrangement of the same CG that the CUDA library
 * offers as an option (eaf_oracle_cg1): not reference arithmetic, the
 * checker of that form only.
 *
 * PARITY UNPINNED: the reference is Fortran + MPI and no Fortran compiler or
 * MPI exists where this is built or run, and the reference's tests pin only
 * whole-simulator outcomes, never cg_3d_mpi's iterates. This restatement is
 * cross-checked instead against an exact rational-arithmetic CG on tiny
 * meshes, an independent numpy restatement, scipy's CG and analytic
 * known-answer systems (tests/test_oracle.py).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SMALL 1.0e-30

typedef struct {
    int nr, nth, nz;
    size_t sx, sxy, n;  /* strides and total halo-array length */
} dims_t;

static dims_t mkdims(int nr, int nth, int nz) {
    dims_t d;
    d.nr = nr; d.nth = nth; d.nz = nz;
    d.sx = (size_t)nr + 4;
    d.sxy = d.sx * ((size_t)nth + 4);
    d.n = d.sxy * ((size_t)nz + 4);
    return d;
}

static inline size_t at(const dims_t* d, int i, int j, int k) {
    return (size_t)(i + 1) * 1 + d->sx * (size_t)(j + 1) + d->sxy * (size_t)(k + 1);
}

static inline double guard(double v) { return v > SMALL ? v : SMALL; }

/* Serial theta-periodic halo copy over the full (i, k) halo ranges. */
void eaf_oracle_theta_wrap(int nr, int nth, int nz, double* x) {
    dims_t d = mkdims(nr, nth, nz);
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nr + 2; ++i) x[at(&d, i, 0, k)] = x[at(&d, i, nth, k)];
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nr + 2; ++i) x[at(&d, i, -1, k)] = x[at(&d, i, nth - 1, k)];
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nr + 2; ++i) x[at(&d, i, nth + 1, k)] = x[at(&d, i, 1, k)];
    for (int k = -1; k <= nz + 2; ++k)
        for (int i = -1; i <= nr + 2; ++i) x[at(&d, i, nth + 2, k)] = x[at(&d, i, 2, k)];
}

/* Association of the interior dot products. G == 0: the reference's
 * sequential column-major sum. G > 0: the fixed reduction tree of the CUDA
 * kernels launched with G blocks of B threads (cg_common.cuh, stencil.cuh):
 * block b owns compact cells [b*ceil(n/G), ...); thread t of it sums cells
 * begin+t, begin+t+B, ... sequentially; each warp folds its 32 lane sums by
 * an xor butterfly (offsets 16, 8, 4, 2, 1); warp 0 folds the warp sums
 * (zero-padded to 32 lanes) the same way; with G > 1, lane l of warp 0 sums
 * block partials l, l+32, ... sequentially from 0.0 and the lanes are folded
 * by the butterfly once more. */
typedef struct {
    int G, B;
    int C;  /* blocks per thread-block cluster (0 or 1: no clusters) */
} plan_t;

typedef struct {
    dims_t d;
    const double *aW, *aE, *aS, *aN, *aB, *aT, *aP;
    int nthreads;
    plan_t plan;
} op_t;

static void matvec(const op_t* o, double* x, double* y) {
    const dims_t* d = &o->d;
    eaf_oracle_theta_wrap(d->nr, d->nth, d->nz, x);
    memset(y, 0, d->n * sizeof(double));
#pragma omp parallel for schedule(static) num_threads(o->nthreads) if (o->nthreads > 1)
    for (int k = 1; k <= d->nz; ++k)
        for (int j = 1; j <= d->nth; ++j)
            for (int i = 1; i <= d->nr; ++i) {
                size_t c = at(d, i, j, k);
                y[c] = o->aP[c] * x[c]
                     - o->aW[c] * x[c - 1] - o->aE[c] * x[c + 1]
                     - o->aS[c] * x[c - d->sx] - o->aN[c] * x[c + d->sx]
                     - o->aB[c] * x[c - d->sxy] - o->aT[c] * x[c + d->sxy];
            }
}

static inline size_t compact_to_halo(const dims_t* d, int c) {
    int i = c % d->nr;
    int t = c / d->nr;
    int j = t % d->nth;
    int k = t / d->nth;
    return at(d, i + 1, j + 1, k + 1);
}

/* In-place xor butterfly over 32 lanes; every lane ends with the same sum. */
static void butterfly32(double* v) {
    double w[32];
    for (int o = 16; o > 0; o >>= 1) {
        for (int l = 0; l < 32; ++l) w[l] = v[l] + v[l ^ o];
        memcpy(v, w, sizeof(w));
    }
}

static double block_tree(const double* lane_sums, int B) {
    int nw = (B + 31) / 32;
    double ws[32];
    for (int w = 0; w < 32; ++w) ws[w] = 0.0;
    for (int w = 0; w < nw; ++w) {
        double v[32];
        for (int l = 0; l < 32; ++l) {
            int t = w * 32 + l;
            v[l] = t < B ? lane_sums[t] : 0.0;
        }
        butterfly32(v);
        ws[w] = v[0];
    }
    butterfly32(ws);
    return ws[0];
}

static double dot_tree(const dims_t* d, const plan_t* pl, const double* a,
                       const double* b) {
    const int n = d->nr * d->nth * d->nz, G = pl->G, B = pl->B;
    const int chunk = (n + G - 1) / G;
    double* lane = (double*)malloc(sizeof(double) * (size_t)B);
    double* part = (double*)malloc(sizeof(double) * (size_t)G);
    for (int g = 0; g < G; ++g) {
        int begin = g * chunk < n ? g * chunk : n;
        int end = begin + chunk < n ? begin + chunk : n;
        for (int t = 0; t < B; ++t) {
            double s = 0.0;
            for (int c = begin + t; c < end; c += B) {
                size_t h = compact_to_halo(d, c);
                s = s + a[h] * b[h];
            }
            lane[t] = s;
        }
        part[g] = block_tree(lane, B);
    }
    /* Cluster grid (csrc/cluster_red.cuh): the leader of each cluster of C
     * consecutive blocks folds their partials in rank order, starting from
     * the first; the cluster partials then take the place of the block
     * partials in the stage below (one cluster: its partial is the total). */
    int np = G;
    if (pl->C > 1) {
        np = G / pl->C;
        for (int c = 0; c < np; ++c) {
            double cp = part[c * pl->C];
            for (int r = 1; r < pl->C; ++r) cp = cp + part[c * pl->C + r];
            part[c] = cp;
        }
    }
    double tot;
    if (np == 1) {
        tot = part[0];
    } else {
        double v[32];
        for (int l = 0; l < 32; ++l) {
            double s = 0.0;
            for (int g = l; g < np; g += 32) s = s + part[g];
            v[l] = s;
        }
        butterfly32(v);
        tot = v[0];
    }
    free(lane);
    free(part);
    return tot;
}

/* Sequential (serial) or per-plane-partial (threaded) interior dot. The
 * threaded form sums each k-plane sequentially, then the planes in order:
 * deterministic, but a different association than the serial sum, so it is
 * only used for CPU timing. */
static double dot(const op_t* o, const double* a, const double* b) {
    const dims_t* d = &o->d;
    if (o->plan.G > 0) return dot_tree(d, &o->plan, a, b);
    if (o->nthreads <= 1) {
        double s = 0.0;
        for (int k = 1; k <= d->nz; ++k)
            for (int j = 1; j <= d->nth; ++j)
                for (int i = 1; i <= d->nr; ++i) {
                    size_t c = at(d, i, j, k);
                    s = s + a[c] * b[c];
                }
        return s;
    }
    double* part = (double*)malloc(sizeof(double) * (size_t)d->nz);
#pragma omp parallel for schedule(static) num_threads(o->nthreads)
    for (int k = 1; k <= d->nz; ++k) {
        double s = 0.0;
        for (int j = 1; j <= d->nth; ++j)
            for (int i = 1; i <= d->nr; ++i) {
                size_t c = at(d, i, j, k);
                s = s + a[c] * b[c];
            }
        part[k - 1] = s;
    }
    double s = 0.0;
    for (int k = 0; k < d->nz; ++k) s += part[k];
    free(part);
    return s;
}

static int cg_impl(int nr, int nth, int nz, const double* aW, const double* aE,
                   const double* aS, const double* aN, const double* aB,
                   const double* aT, const double* aP, const double* Su,
                   double* phi, int max_iter, double tol, double* residual,
                   int* n_iter, int nthreads, plan_t plan) {
    if (nr < 1 || nth < 1 || nz < 1) return 2;
    if (plan.G < 0 || (plan.G > 0 && plan.B < 1)) return 2;
    if (plan.C > 1 && (plan.G < plan.C || plan.G % plan.C != 0)) return 2;
    op_t o;
    o.plan = plan;
    o.d = mkdims(nr, nth, nz);
    o.aW = aW; o.aE = aE; o.aS = aS; o.aN = aN; o.aB = aB; o.aT = aT; o.aP = aP;
    o.nthreads = nthreads;
    const dims_t* d = &o.d;
    double* r = (double*)calloc(d->n, sizeof(double));
    double* z = (double*)calloc(d->n, sizeof(double));
    double* pv = (double*)calloc(d->n, sizeof(double));
    double* q = (double*)calloc(d->n, sizeof(double));
    if (!r || !z || !pv || !q) { free(r); free(z); free(pv); free(q); return 6; }

    matvec(&o, phi, q);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                size_t c = at(d, i, j, k);
                r[c] = Su[c] - q[c];
            }

    double bnorm = sqrt(dot(&o, Su, Su));
    if (bnorm < SMALL) {
        *residual = 0.0;
        *n_iter = 0;
        free(r); free(z); free(pv); free(q);
        return 0;
    }

#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                size_t c = at(d, i, j, k);
                z[c] = r[c] / guard(fabs(aP[c]));
            }
    memcpy(pv, z, d->n * sizeof(double));
    double rz = dot(&o, r, z);
    double res = sqrt(dot(&o, r, r)) / bnorm;
    int nit = 0;

    for (int iter = 1; iter <= max_iter; ++iter) {
        matvec(&o, pv, q);
        double pq = dot(&o, pv, q);
        if (fabs(pq) < SMALL) break;
        double alpha = rz / pq;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nth; ++j)
                for (int i = 1; i <= nr; ++i) {
                    size_t c = at(d, i, j, k);
                    phi[c] = phi[c] + alpha * pv[c];
                }
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nth; ++j)
                for (int i = 1; i <= nr; ++i) {
                    size_t c = at(d, i, j, k);
                    r[c] = r[c] - alpha * q[c];
                }
        double rnorm = sqrt(dot(&o, r, r));
        res = rnorm / bnorm;
        nit = iter;
        if (res < tol) break;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nth; ++j)
                for (int i = 1; i <= nr; ++i) {
                    size_t c = at(d, i, j, k);
                    z[c] = r[c] / guard(fabs(aP[c]));
                }
        double rz_new = dot(&o, r, z);
        double beta = rz_new / guard(rz);
        rz = rz_new;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nth; ++j)
                for (int i = 1; i <= nr; ++i) {
                    size_t c = at(d, i, j, k);
                    pv[c] = z[c] + beta * pv[c];
                }
    }

    eaf_oracle_theta_wrap(nr, nth, nz, phi);
    *residual = res;
    *n_iter = nit;
    free(r); free(z); free(pv); free(q);
    return 0;
}

/* Serial restatement: the parity oracle. Returns 0, 2 (bad dims) or 6 (OOM). */
int eaf_oracle_cg(int nr, int nth, int nz, const double* aW, const double* aE,
                  const double* aS, const double* aN, const double* aB,
                  const double* aT, const double* aP, const double* Su,
                  double* phi, int max_iter, double tol, double* residual,
                  int* n_iter) {
    plan_t seq = {0, 0, 0};
    return cg_impl(nr, nth, nz, aW, aE, aS, aN, aB, aT, aP, Su, phi, max_iter,
                   tol, residual, n_iter, 1, seq);
}

/* The same restatement with the dot products associated as the CUDA kernels
 * associate them for a launch of G blocks x B threads (block g owns the g-th
 * contiguous slice of ceil(n/G) cells): every other operation is unchanged,
 * so a CUDA solve launched that way must agree bit for bit. */
int eaf_oracle_cg_tree(int nr, int nth, int nz, const double* aW,
                       const double* aE, const double* aS, const double* aN,
                       const double* aB, const double* aT, const double* aP,
                       const double* Su, double* phi, int max_iter, double tol,
                       double* residual, int* n_iter, int G, int B) {
    if (G < 1 || B < 1) return 2;
    plan_t pl = {G, B, 0};
    return cg_impl(nr, nth, nz, aW, aE, aS, aN, aB, aT, aP, Su, phi, max_iter,
                   tol, residual, n_iter, 1, pl);
}

/* The same with the launch on a grid of thread-block clusters of C blocks
 * (G a multiple of C): the dots are associated per cluster as the cluster
 * all-reduce does (see dot_tree). C <= 1 is eaf_oracle_cg_tree. */
int eaf_oracle_cg_cluster(int nr, int nth, int nz, const double* aW,
                          const double* aE, const double* aS, const double* aN,
                          const double* aB, const double* aT, const double* aP,
                          const double* Su, double* phi, int max_iter, double tol,
                          double* residual, int* n_iter, int G, int B, int C) {
    if (G < 1 || B < 1 || C < 0) return 2;
    plan_t pl = {G, B, C};
    return cg_impl(nr, nth, nz, aW, aE, aS, aN, aB, aT, aP, Su, phi, max_iter,
                   tol, residual, n_iter, 1, pl);
}

/* ----------------------------------------------------------------------
 * Single-reduction form of the same preconditioned CG (Chronopoulos and
 * Gear, "s-step iterative methods for symmetric linear systems", J. Comput.
 * Appl. Math. 25, 1989): the reference's recurrences rearranged so that the
 * three scalars of an iteration -- gamma = r.u, delta = w.u (u = M^-1 r,
 * w = A u) and r.r -- come from ONE reduction; s = A p is carried by the
 * recurrence s = w + beta s, and p.q by delta - beta gamma / alpha_prev.
 * Not the reference's arithmetic: it lands elsewhere in the residual ball
 * (test bar: both residuals < tol, iterations within a few per cent), and
 * the Jacobi step multiplies by 1 / max(|aP|, SMALL) instead of dividing.
 * The matvec expression order, the exit tests (strict
 * < tol after the update, breakdown |p.q| < SMALL, beta guard
 * max(gamma_prev, SMALL)) and the NaN behaviour are the reference's.
 * First iteration: p = u, s = w exactly. With plan.G > 0 the dots take the
 * kernels' association: this is the parity oracle of the CUDA
 * single-reduction kernel, bit for bit.
 * ---------------------------------------------------------------------- */
static int cg1_impl(int nr, int nth, int nz, const double* aW, const double* aE,
                    const double* aS, const double* aN, const double* aB,
                    const double* aT, const double* aP, const double* Su,
                    double* phi, int max_iter, double tol, double* residual,
                    int* n_iter, plan_t plan) {
    if (nr < 1 || nth < 1 || nz < 1) return 2;
    if (plan.G < 0 || (plan.G > 0 && plan.B < 1)) return 2;
    if (plan.C > 1 && (plan.G < plan.C || plan.G % plan.C != 0)) return 2;
    op_t o;
    o.plan = plan;
    o.d = mkdims(nr, nth, nz);
    o.aW = aW; o.aE = aE; o.aS = aS; o.aN = aN; o.aB = aB; o.aT = aT; o.aP = aP;
    o.nthreads = 1;
    const dims_t* d = &o.d;
    double* r = (double*)calloc(d->n, sizeof(double));
    double* u = (double*)calloc(d->n, sizeof(double));
    double* w = (double*)calloc(d->n, sizeof(double));
    double* pv = (double*)calloc(d->n, sizeof(double));
    double* sv = (double*)calloc(d->n, sizeof(double));
    if (!r || !u || !w || !pv || !sv) {
        free(r); free(u); free(w); free(pv); free(sv);
        return 6;
    }
    matvec(&o, phi, w);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                size_t c = at(d, i, j, k);
                r[c] = Su[c] - w[c];
            }
    double bnorm = sqrt(dot(&o, Su, Su));
    if (bnorm < SMALL) {
        *residual = 0.0;
        *n_iter = 0;
        free(r); free(u); free(w); free(pv); free(sv);
        return 0;
    }
#define PRECOND()                                                       \
    for (int k = 1; k <= nz; ++k)                                       \
        for (int j = 1; j <= nth; ++j)                                  \
            for (int i = 1; i <= nr; ++i) {                             \
                size_t c = at(d, i, j, k);                              \
                u[c] = r[c] * (1.0 / guard(fabs(aP[c])));               \
            }
    PRECOND();
    matvec(&o, u, w);
    double gam = dot(&o, r, u), dlt = dot(&o, w, u);
    double res = sqrt(dot(&o, r, r)) / bnorm;
    double alpha_prev = 0.0, gam_prev = 0.0;
    int nit = 0;
    for (int iter = 1; iter <= max_iter; ++iter) {
        double beta = 0.0, den;
        if (iter == 1) {
            den = dlt;
        } else {
            beta = gam / guard(gam_prev);
            den = dlt - beta * gam / alpha_prev;
        }
        if (fabs(den) < SMALL) break;
        double alpha = gam / den;
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nth; ++j)
                for (int i = 1; i <= nr; ++i) {
                    size_t c = at(d, i, j, k);
                    if (iter == 1) {
                        pv[c] = u[c];
                        sv[c] = w[c];
                    } else {
                        pv[c] = u[c] + beta * pv[c];
                        sv[c] = w[c] + beta * sv[c];
                    }
                    phi[c] = phi[c] + alpha * pv[c];
                    r[c] = r[c] - alpha * sv[c];
                }
        PRECOND();
        matvec(&o, u, w);
        gam_prev = gam;
        alpha_prev = alpha;
        gam = dot(&o, r, u);
        dlt = dot(&o, w, u);
        res = sqrt(dot(&o, r, r)) / bnorm;
        nit = iter;
        if (res < tol) break;
    }
#undef PRECOND
    eaf_oracle_theta_wrap(nr, nth, nz, phi);
    *residual = res;
    *n_iter = nit;
    free(r); free(u); free(w); free(pv); free(sv);
    return 0;
}

/* Single-reduction CG, sequential dots (G == 0) or the kernels' association
 * for a launch of G blocks x B threads. Returns 0, 2 or 6. */
int eaf_oracle_cg1(int nr, int nth, int nz, const double* aW, const double* aE,
                   const double* aS, const double* aN, const double* aB,
                   const double* aT, const double* aP, const double* Su,
                   double* phi, int max_iter, double tol, double* residual,
                   int* n_iter, int G, int B) {
    plan_t pl = {G, B, 0};
    return cg1_impl(nr, nth, nz, aW, aE, aS, aN, aB, aT, aP, Su, phi, max_iter,
                    tol, residual, n_iter, pl);
}

/* Interior dot of two halo-layout arrays in the kernels' association
 * (G, B) or, with G == 0, the reference's sequential order. */
double eaf_oracle_dot(int nr, int nth, int nz, const double* a, const double* b,
                      int G, int B) {
    op_t o;
    memset(&o, 0, sizeof(o));
    o.d = mkdims(nr, nth, nz);
    o.nthreads = 1;
    o.plan.G = G;
    o.plan.B = B;
    o.plan.C = 0;
    return dot(&o, a, b);
}

/* The same on a grid of thread-block clusters of C blocks (G a multiple of
 * C): the association of the cluster all-reduce (see dot_tree). */
double eaf_oracle_dot_cluster(int nr, int nth, int nz, const double* a, const double* b,
                              int G, int B, int C) {
    op_t o;
    memset(&o, 0, sizeof(o));
    o.d = mkdims(nr, nth, nz);
    o.nthreads = 1;
    o.plan.G = G;
    o.plan.B = B;
    o.plan.C = C;
    return dot(&o, a, b);
}

/* Threaded variant (OpenMP over k-planes) used only as the timed CPU
 * baseline: same algorithm and guards, plane-partial dots. */
int eaf_oracle_cg_threads(int nr, int nth, int nz, const double* aW,
                          const double* aE, const double* aS, const double* aN,
                          const double* aB, const double* aT, const double* aP,
                          const double* Su, double* phi, int max_iter,
                          double tol, double* residual, int* n_iter,
                          int nthreads) {
    plan_t seq = {0, 0, 0};
    return cg_impl(nr, nth, nz, aW, aE, aS, aN, aB, aT, aP, Su, phi, max_iter,
                   tol, residual, n_iter, nthreads < 1 ? 1 : nthreads, seq);
}

/* y = A x over the interior exactly as the reference matvec (x's theta halos
 * are refreshed in place; y's halos are zeroed). */
void eaf_oracle_matvec(int nr, int nth, int nz, const double* aW,
                       const double* aE, const double* aS, const double* aN,
                       const double* aB, const double* aT, const double* aP,
                       double* x, double* y) {
    op_t o;
    o.d = mkdims(nr, nth, nz);
    o.aW = aW; o.aE = aE; o.aS = aS; o.aN = aN; o.aB = aB; o.aT = aT; o.aP = aP;
    o.nthreads = 1;
    o.plan.G = 0;
    o.plan.B = 0;
    o.plan.C = 0;
    matvec(&o, x, y);
}

int eaf_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------
 * Line-by-line TDMA, serial branch of tdma_3d_mpi (src/mod_solver_3d.f90:
 * 252-366). Per sweep: theta-halo refresh (mpi_exchange_halos_3d with one
 * rank is the periodic copy, src/mod_mpi_topology.f90:303-311), then r
 * lines for k = 1..nz, j = 1..nth; refresh; theta lines for k, i; refresh;
 * z lines for j, i. Every line solve reads the current phi in place, so a
 * line sees the new values of the lines solved before it in that order
 * (Gauss-Seidel between lines) and the halo values of the last refresh. The
 * right-hand sides keep the reference's statement and operand order; the
 * segment endpoints add the lagged halo couplings after the loop.
 * ---------------------------------------------------------------------- */

/* `tdma` (src/mod_solver_3d.f90:22-46): `sign(SMALL, v)` is copysign (the
 * sign of a negative zero is kept, as gfortran does). */
static void thomas(const double* a, const double* b, const double* c,
                   const double* d, double* x, int n, double* cp, double* dp) {
    double b1 = b[0];
    if (fabs(b1) < SMALL) b1 = copysign(SMALL, b1);
    cp[0] = c[0] / b1;
    dp[0] = d[0] / b1;
    for (int i = 1; i < n; ++i) {
        double m = b[i] - a[i] * cp[i - 1];
        if (fabs(m) < SMALL) m = copysign(SMALL, m);
        cp[i] = c[i] / m;
        dp[i] = (d[i] - a[i] * dp[i - 1]) / m;
    }
    x[n - 1] = dp[n - 1];
    for (int i = n - 2; i >= 0; --i) x[i] = dp[i] - cp[i] * x[i + 1];
}

int eaf_oracle_tdma_3d(int nr, int nth, int nz, const double* aW, const double* aE,
                       const double* aS, const double* aN, const double* aB,
                       const double* aT, const double* aP, const double* Su,
                       double* phi, int n_sweep) {
    if (nr < 1 || nth < 1 || nz < 1) return 2;
    const dims_t D = mkdims(nr, nth, nz);
    const dims_t* d = &D;
    int nmax = nr > nth ? nr : nth;
    if (nz > nmax) nmax = nz;
    double* buf = (double*)malloc(sizeof(double) * 7 * (size_t)nmax);
    if (!buf) return 6;
    double *a = buf, *b = a + nmax, *c = b + nmax, *dd = c + nmax, *x = dd + nmax,
           *cp = x + nmax, *dp = cp + nmax;
    for (int sweep = 1; sweep <= n_sweep; ++sweep) {
        eaf_oracle_theta_wrap(nr, nth, nz, phi);
        for (int k = 1; k <= nz; ++k)          /* r lines (:286-308) */
            for (int j = 1; j <= nth; ++j) {
                for (int i = 1; i <= nr; ++i) {
                    size_t q = at(d, i, j, k);
                    a[i - 1] = -aW[q];
                    b[i - 1] = aP[q];
                    c[i - 1] = -aE[q];
                    double t = Su[q] + aS[q] * phi[at(d, i, j - 1, k)] +
                               aN[q] * phi[at(d, i, j + 1, k)];
                    dd[i - 1] = t + aB[q] * phi[at(d, i, j, k - 1)] +
                                aT[q] * phi[at(d, i, j, k + 1)];
                }
                dd[0] = dd[0] + aW[at(d, 1, j, k)] * phi[at(d, 0, j, k)];
                dd[nr - 1] = dd[nr - 1] + aE[at(d, nr, j, k)] * phi[at(d, nr + 1, j, k)];
                thomas(a, b, c, dd, x, nr, cp, dp);
                for (int i = 1; i <= nr; ++i) phi[at(d, i, j, k)] = x[i - 1];
            }
        eaf_oracle_theta_wrap(nr, nth, nz, phi);
        for (int k = 1; k <= nz; ++k)          /* theta lines (:311-332) */
            for (int i = 1; i <= nr; ++i) {
                for (int j = 1; j <= nth; ++j) {
                    size_t q = at(d, i, j, k);
                    a[j - 1] = -aS[q];
                    b[j - 1] = aP[q];
                    c[j - 1] = -aN[q];
                    double t = Su[q];
                    t = t + aW[q] * phi[at(d, i - 1, j, k)] + aE[q] * phi[at(d, i + 1, j, k)];
                    dd[j - 1] = t + aB[q] * phi[at(d, i, j, k - 1)] +
                                aT[q] * phi[at(d, i, j, k + 1)];
                }
                dd[0] = dd[0] + aS[at(d, i, 1, k)] * phi[at(d, i, 0, k)];
                dd[nth - 1] = dd[nth - 1] + aN[at(d, i, nth, k)] * phi[at(d, i, nth + 1, k)];
                thomas(a, b, c, dd, x, nth, cp, dp);
                for (int j = 1; j <= nth; ++j) phi[at(d, i, j, k)] = x[j - 1];
            }
        eaf_oracle_theta_wrap(nr, nth, nz, phi);
        for (int j = 1; j <= nth; ++j)         /* z lines (:335-359) */
            for (int i = 1; i <= nr; ++i) {
                for (int k = 1; k <= nz; ++k) {
                    size_t q = at(d, i, j, k);
                    a[k - 1] = -aB[q];
                    b[k - 1] = aP[q];
                    c[k - 1] = -aT[q];
                    double t = Su[q] + aS[q] * phi[at(d, i, j - 1, k)] +
                               aN[q] * phi[at(d, i, j + 1, k)];
                    dd[k - 1] = t + aW[q] * phi[at(d, i - 1, j, k)] +
                                aE[q] * phi[at(d, i + 1, j, k)];
                }
                dd[0] = dd[0] + aB[at(d, i, j, 1)] * phi[at(d, i, j, 0)];
                dd[nz - 1] = dd[nz - 1] + aT[at(d, i, j, nz)] * phi[at(d, i, j, nz + 1)];
                thomas(a, b, c, dd, x, nz, cp, dp);
                for (int k = 1; k <= nz; ++k) phi[at(d, i, j, k)] = x[k - 1];
            }
    }
    free(buf);
    return 0;
}

/* compute_residual_3d_mpi (src/mod_solver_3d.f90:625-694), serial: cells
 * whose row is the identity (aP == 1, all links 0) are skipped; r_local and
 * the normalisation term keep the reference's operand order; `x**2` is x*x.
 * G == 0 sums sequentially (k, j, i) as the reference; G > 0 associates the
 * two sums as the CUDA kernel launched with G blocks of B threads does (the
 * plan of the CG dots; a skipped cell adds +0.0 there, which leaves a sum
 * of squares unchanged). */
static void residual_terms(const dims_t* d, const double* aW, const double* aE,
                           const double* aS, const double* aN, const double* aB,
                           const double* aT, const double* aP, const double* Su,
                           const double* phi, size_t q, double* rr, double* bb) {
    if (aP[q] == 1.0 && aW[q] == 0.0 && aE[q] == 0.0 && aS[q] == 0.0 && aN[q] == 0.0 &&
        aB[q] == 0.0 && aT[q] == 0.0) {
        *rr = 0.0;
        *bb = 0.0;
        return;
    }
    double r = Su[q] - aP[q] * phi[q] + aS[q] * phi[q - d->sx] + aN[q] * phi[q + d->sx];
    r = r + aW[q] * phi[q - 1] + aE[q] * phi[q + 1];
    r = r + aB[q] * phi[q - d->sxy] + aT[q] * phi[q + d->sxy];
    double t = fabs(Su[q]) + fabs(aP[q] * phi[q]) + SMALL;
    *rr = r * r;
    *bb = t * t;
}

double eaf_oracle_residual_3d(int nr, int nth, int nz, const double* aW, const double* aE,
                              const double* aS, const double* aN, const double* aB,
                              const double* aT, const double* aP, const double* Su,
                              const double* phi, int G, int B) {
    const dims_t D = mkdims(nr, nth, nz);
    const dims_t* d = &D;
    double sum_r = 0.0, sum_b = 0.0;
    if (G <= 0) {
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nth; ++j)
                for (int i = 1; i <= nr; ++i) {
                    size_t q = at(d, i, j, k);
                    if (aP[q] == 1.0 && aW[q] == 0.0 && aE[q] == 0.0 && aS[q] == 0.0 &&
                        aN[q] == 0.0 && aB[q] == 0.0 && aT[q] == 0.0)
                        continue;
                    double rr, bb;
                    residual_terms(d, aW, aE, aS, aN, aB, aT, aP, Su, phi, q, &rr, &bb);
                    sum_r = sum_r + rr;
                    sum_b = sum_b + bb;
                }
    } else {
        const int n = nr * nth * nz;
        const int chunk = (n + G - 1) / G;
        double* lane_r = (double*)malloc(sizeof(double) * (size_t)B * 2);
        double* part = (double*)malloc(sizeof(double) * (size_t)G * 2);
        if (!lane_r || !part) {
            free(lane_r);
            free(part);
            return NAN;
        }
        double* lane_b = lane_r + B;
        for (int g = 0; g < G; ++g) {
            int begin = g * chunk < n ? g * chunk : n;
            int end = begin + chunk < n ? begin + chunk : n;
            for (int t = 0; t < B; ++t) {
                double sr = 0.0, sb = 0.0;
                for (int c = begin + t; c < end; c += B) {
                    double rr, bb;
                    residual_terms(d, aW, aE, aS, aN, aB, aT, aP, Su, phi,
                                   compact_to_halo(d, c), &rr, &bb);
                    sr = sr + rr;
                    sb = sb + bb;
                }
                lane_r[t] = sr;
                lane_b[t] = sb;
            }
            part[g] = block_tree(lane_r, B);
            part[G + g] = block_tree(lane_b, B);
        }
        for (int m = 0; m < 2; ++m) {
            const double* pm = part + (size_t)m * G;
            double tot;
            if (G == 1) {
                tot = pm[0];
            } else {
                double v[32];
                for (int l = 0; l < 32; ++l) {
                    double s = 0.0;
                    for (int g = l; g < G; g += 32) s = s + pm[g];
                    v[l] = s;
                }
                butterfly32(v);
                tot = v[0];
            }
            if (m == 0) sum_r = tot; else sum_b = tot;
        }
        free(lane_r);
        free(part);
    }
    return sqrt(sum_r) / (sqrt(sum_b) + SMALL);
}

/* ------------------------------------------------------------------------
 * Post-CG corrections of solve_pressure_correction, serial branch
 * (src/mod_pressure_3d.f90:333-397, correct_velocities :689-746), in the
 * reference's statement order:
 *   1. conservative face fluxes Fc = Fs + ac (pp_P - pp_nb) where linked;
 *   2. theta-halo refresh of Fc_r/th/z and of the link flags (int);
 *   3. correct_velocities of the liquid (act_l), then of the gas (act_g)
 *      when it is in the pressure equation;
 *   4. p = p + alpha_p pp and p = max(-P_HYDRO_CAP, min(P_HYDRO_CAP, p)),
 *      both over the whole array (halos included);
 *   5. sealed cells (neither phase active): p = mean of the p of their
 *      active neighbours (i-1, i+1, j-1, j+1, k-1, k+1 in that order), 0
 *      without any;
 *   6. theta-halo refresh of p.
 * Fortran min/max are written fmin/fmax (identical on non-NaN values; the
 * result for a NaN p is not pinned). Logical masks are default-kind
 * Fortran logicals (4 bytes, nonzero = true).
 * dv: pp, Fs_r, Fs_th, Fs_z, ac_r, ac_th, ac_z, Fc_r, Fc_th, Fc_z, vol,
 *     r, theta, z (cell centres, index -1..n+2), p, then per phase (liquid,
 *     gas) alpha, aP_ur, aP_uth, aP_uz, ur, uth, uz.
 * iv: lk_r, lk_th, lk_z, cell_type, act_l, act_g.
 * ---------------------------------------------------------------------- */
#define P_HYDRO_CAP 2.0e6

static void theta_wrap_int(const dims_t* d, int* x) {
    for (int k = -1; k <= d->nz + 2; ++k)
        for (int i = -1; i <= d->nr + 2; ++i) x[at(d, i, 0, k)] = x[at(d, i, d->nth, k)];
    for (int k = -1; k <= d->nz + 2; ++k)
        for (int i = -1; i <= d->nr + 2; ++i) x[at(d, i, -1, k)] = x[at(d, i, d->nth - 1, k)];
    for (int k = -1; k <= d->nz + 2; ++k)
        for (int i = -1; i <= d->nr + 2; ++i) x[at(d, i, d->nth + 1, k)] = x[at(d, i, 1, k)];
    for (int k = -1; k <= d->nz + 2; ++k)
        for (int i = -1; i <= d->nr + 2; ++i) x[at(d, i, d->nth + 2, k)] = x[at(d, i, 2, k)];
}

static void correct_velocities(const dims_t* d, double* const* ph, const double* pp,
                               const double* vol, const double* r, const double* th,
                               const double* z, const int* ct, const int* act) {
    const double *alpha = ph[0], *aur = ph[1], *auth = ph[2], *auz = ph[3];
    double *ur = ph[4], *uth = ph[5], *uz = ph[6];
    for (int k = 1; k <= d->nz; ++k)
        for (int j = 1; j <= d->nth; ++j)
            for (int i = 1; i <= d->nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (ct[q] == 0) continue;
                if (!act[q]) continue;
                const int skip_r = (i == 1) || (i == d->nr);
                if (!skip_r && fabs(aur[q]) > SMALL) {
                    double dc = alpha[q] * vol[q] / aur[q];
                    ur[q] = ur[q] - dc * (pp[q + 1] - pp[q - 1]) / (r[i + 2] - r[i]);
                }
                if (fabs(auth[q]) > SMALL) {
                    double dc = alpha[q] * vol[q] / auth[q];
                    uth[q] = uth[q] - dc * (pp[q + d->sx] - pp[q - d->sx]) /
                                          (r[i + 1] * (th[j + 2] - th[j]));
                }
                const int skip_z = (k == 1) || (k == d->nz);
                if (!skip_z && fabs(auz[q]) > SMALL) {
                    double dc = alpha[q] * vol[q] / auz[q];
                    uz[q] = uz[q] - dc * (pp[q + d->sxy] - pp[q - d->sxy]) / (z[k + 2] - z[k]);
                }
            }
}

int eaf_oracle_pressure_correct(int nr, int nth, int nz, double* const* dv, int* const* iv,
                                int has_gas, double alpha_p) {
    if (nr < 1 || nth < 1 || nz < 1) return 2;
    const dims_t D = mkdims(nr, nth, nz);
    const dims_t* d = &D;
    const double *pp = dv[0], *Fs_r = dv[1], *Fs_th = dv[2], *Fs_z = dv[3], *ac_r = dv[4],
                 *ac_th = dv[5], *ac_z = dv[6], *vol = dv[10], *r = dv[11], *th = dv[12],
                 *z = dv[13];
    double *Fc_r = dv[7], *Fc_th = dv[8], *Fc_z = dv[9], *p = dv[14];
    int *lk_r = iv[0], *lk_th = iv[1], *lk_z = iv[2];
    const int *ct = iv[3], *act_l = iv[4], *act_g = iv[5];
    /* 1. (:333-345) */
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (ct[q] == 0) continue;
                if (lk_r[q] == 1) Fc_r[q] = Fs_r[q] + ac_r[q] * (pp[q] - pp[q + 1]);
                if (lk_th[q] == 1) Fc_th[q] = Fs_th[q] + ac_th[q] * (pp[q] - pp[q + d->sx]);
                if (lk_z[q] == 1) Fc_z[q] = Fs_z[q] + ac_z[q] * (pp[q] - pp[q + d->sxy]);
            }
    /* 2. (:346-351) */
    eaf_oracle_theta_wrap(nr, nth, nz, Fc_r);
    eaf_oracle_theta_wrap(nr, nth, nz, Fc_th);
    eaf_oracle_theta_wrap(nr, nth, nz, Fc_z);
    theta_wrap_int(d, lk_r);
    theta_wrap_int(d, lk_th);
    theta_wrap_int(d, lk_z);
    /* 3. (:354-356) */
    correct_velocities(d, dv + 15, pp, vol, r, th, z, ct, act_l);
    if (has_gas) correct_velocities(d, dv + 22, pp, vol, r, th, z, ct, act_g);
    /* 4. (:358-360) */
    for (size_t q = 0; q < d->n; ++q) p[q] = p[q] + alpha_p * pp[q];
    for (size_t q = 0; q < d->n; ++q) p[q] = fmax(-P_HYDRO_CAP, fmin(P_HYDRO_CAP, p[q]));
    /* 5. (:373-395, acc_nb :451-458) */
    static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0},
                                  {0, 0, -1}, {0, 0, 1}};
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (ct[q] == 0) continue;
                if (act_l[q] || act_g[q]) continue;
                double psum = 0.0;
                int nnb = 0;
                for (int t = 0; t < 6; ++t) {
                    const size_t b = at(d, i + off[t][0], j + off[t][1], k + off[t][2]);
                    if (ct[b] == 0) continue;
                    if (!act_l[b] && !act_g[b]) continue;
                    psum = psum + p[b];
                    nnb = nnb + 1;
                }
                p[q] = nnb > 0 ? psum / (double)nnb : 0.0;
            }
    /* 6. (:396) */
    eaf_oracle_theta_wrap(nr, nth, nz, p);
    return 0;
}

/* ------------------------------------------------------------------------
 * Assembly of the pressure-correction equation, serial branch of
 * solve_pressure_correction up to the CG call (src/mod_pressure_3d.f90:
 * 135-310), in the reference's statement and operand order.
 * dv (double, halo layout unless noted):
 *   0 vol, 1 Ar, 2 Ath, 3 Az, 4 r, 5 theta, 6 z (cell centres, -1..n+2),
 *   7 p, 8 liq_room,
 *   9-16 liquid alpha, rho, ur, uth, uz, aP_ur, aP_uth, aP_uz, 17 liquid T,
 *   18-25 gas (same order), 26 gas T_old,
 *   outputs 27-35 aW, aE, aS, aN, aB, aT, aP, Su, pp,
 *           36-44 Fs_r, Fs_th, Fs_z, ac_r, ac_th, ac_z, Fc_r, Fc_th, Fc_z.
 * iv (int, halo layout): 0 cell_type, 1 outlet (nonzero: electrode hole at
 *   k = nz), 2 act_l, 3 act_g, outputs 4-6 lk_r, lk_th, lk_z.
 * flags: 1 liq_room_valid, 2 gas in the pressure equation, 4 gas
 *   compressibility. sc: dt, rho_gas, T_ambient, beta_expansion.
 * Fortran MAX/MIN are fmax/fmin (identical on non-NaN values).
 * ---------------------------------------------------------------------- */
#define GRAVITY_C 9.81
#define PP_COMPLIANCE_C 1.0e-6
#define COMP_SRC_CAP_C 0.2
#define P0_THERMO_C 101325.0
#define C_SOUND_LIQ_C 4000.0
#define T_MIN_GAS_C 100.0
#define ROOM_EPS_C 1.0e-4

typedef struct {
    const dims_t* d;
    double* const* dv;
    int* const* iv;
    int flags;
    const double* sc;
} asm_t;

static inline int pv_cell(const asm_t* A, size_t q) {
    return A->iv[0][q] != 0 && (A->iv[2][q] || A->iv[3][q]);
}

/* pgrad (src/mod_constants.f90:274-287) */
static double pgrad(double pm, double p0, double pp_, double xm, double x0, double xp,
                    int okm, int okp) {
    if (okm && okp) return (pp_ - pm) / (xp - xm);
    if (okp) return (pp_ - p0) / (xp - x0);
    if (okm) return (p0 - pm) / (x0 - xm);
    return 0.0;
}

/* liq_weight_f (:407-417) between cells qa and qb of one column */
static double liq_weight_f(const asm_t* A, size_t qa, size_t qb) {
    const double *al = A->dv[9], *rho = A->dv[10], *T = A->dv[17];
    const int* act = A->iv[2];
    const double beta = A->sc[3], Tamb = A->sc[2];
    return 0.5 * GRAVITY_C *
           ((act[qa] ? 1.0 : 0.0) * al[qa] * rho[qa] * (1.0 - beta * (T[qa] - Tamb)) +
            (act[qb] ? 1.0 : 0.0) * al[qb] * rho[qb] * (1.0 - beta * (T[qb] - Tamb)));
}

/* cell_gradients (:621-651) of p into gr, gth, gz (whole arrays zeroed,
 * interior non-solid cells computed, theta halos refreshed); with isg the
 * vertical gradient is gas_gz (:421-440). */
static void cell_gradients(const asm_t* A, int isg, double* gr, double* gth, double* gz) {
    const dims_t* d = A->d;
    const double *p = A->dv[7], *r = A->dv[4], *th = A->dv[5], *z = A->dv[6];
    memset(gr, 0, d->n * sizeof(double));
    memset(gth, 0, d->n * sizeof(double));
    memset(gz, 0, d->n * sizeof(double));
    for (int k = 1; k <= d->nz; ++k)
        for (int j = 1; j <= d->nth; ++j)
            for (int i = 1; i <= d->nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (A->iv[0][q] == 0) continue;
                const size_t qw = q - 1, qe = q + 1, qs = q - d->sx, qn = q + d->sx,
                             qb = q - d->sxy, qt = q + d->sxy;
                gr[q] = pgrad(p[qw], p[q], p[qe], r[i], r[i + 1], r[i + 2],
                              i > 1 && pv_cell(A, qw), i < d->nr && pv_cell(A, qe));
                gth[q] = pgrad(p[qs], p[q], p[qn], r[i + 1] * th[j], r[i + 1] * th[j + 1],
                               r[i + 1] * th[j + 2], pv_cell(A, qs), pv_cell(A, qn));
                const int okm = k > 1 && pv_cell(A, qb), okp = k < d->nz && pv_cell(A, qt);
                gz[q] = pgrad(p[qb], p[q], p[qt], z[k], z[k + 1], z[k + 2], okm, okp);
                if (isg) {
                    double gb = 0.0, gt = 0.0, g;
                    if (okm) gb = (p[q] - p[qb]) / (z[k + 1] - z[k]) + liq_weight_f(A, qb, q);
                    if (okp) gt = (p[qt] - p[q]) / (z[k + 2] - z[k + 1]) + liq_weight_f(A, q, qt);
                    if (okm && okp) g = 0.5 * (gb + gt);
                    else if (okp) g = gt;
                    else if (okm) g = gb;
                    else g = 0.0;
                    gz[q] = g;
                }
            }
    eaf_oracle_theta_wrap(d->nr, d->nth, d->nz, gr);
    eaf_oracle_theta_wrap(d->nr, d->nth, d->nz, gth);
    eaf_oracle_theta_wrap(d->nr, d->nth, d->nz, gz);
}

/* face_open (:660-668) */
static int face_open(const asm_t* A, int isg, double u_f, double room_neg, double room_pos) {
    if (isg || !(A->flags & 1)) return 1;
    int open = 1;
    if (u_f > 0.0 && room_pos <= ROOM_EPS_C) open = 0;
    if (u_f < 0.0 && room_neg <= ROOM_EPS_C) open = 0;
    return open;
}

/* add_phase_contribution (:469-619) of one phase (ph = dv index of its
 * alpha; aef = its alpha), accumulating into the coefficients, Su and
 * flux_ref; export writes the + faces' Fs/ac/lk. */
static void add_phase(const asm_t* A, int ph, const int* act, int export_, const double* gr,
                      const double* gth, const double* gz, int isg, double* flux_ref) {
    const dims_t* d = A->d;
    double* const* dv = A->dv;
    const double *aef = dv[ph], *ur = dv[ph + 2], *uth = dv[ph + 3], *uz = dv[ph + 4],
                 *apr = dv[ph + 5], *apt = dv[ph + 6], *apz = dv[ph + 7];
    const double *vol = dv[0], *Ar = dv[1], *Ath = dv[2], *Az = dv[3], *r = dv[4],
                 *th = dv[5], *z = dv[6], *pf = dv[7], *rm = dv[8];
    double *aW = dv[27], *aE = dv[28], *aS = dv[29], *aN = dv[30], *aB = dv[31],
           *aT = dv[32], *Su = dv[34];
    double *Fs_r = dv[36], *Fs_th = dv[37], *Fs_z = dv[38], *ac_r = dv[39], *ac_th = dv[40],
           *ac_z = dv[41];
    int *lk_r = A->iv[4], *lk_th = A->iv[5], *lk_z = A->iv[6];
    const int* ct = A->iv[0];
#define LINK(x) (ct[x] != 0 && act[x])
#define DF(ap, x) (0.5 * (aef[q] * vol[q] / fmax(ap[q], SMALL) + aef[x] * vol[x] / fmax(ap[x], SMALL)))
    for (int k = 1; k <= d->nz; ++k)
        for (int j = 1; j <= d->nth; ++j)
            for (int i = 1; i <= d->nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (ct[q] == 0) continue;
                if (!act[q]) continue;
                const size_t w = q - 1, e = q + 1, s = q - d->sx, n = q + d->sx, b = q - d->sxy,
                             t = q + d->sxy;
                double d_f, af, u_f, delta;
                if (LINK(w)) {
                    d_f = DF(apr, w);
                    af = 0.5 * (aef[q] + aef[w]);
                    delta = r[i + 1] - r[i];
                    u_f = 0.5 * (ur[w] + ur[q]) +
                          d_f * (0.5 * (gr[w] + gr[q]) - (pf[q] - pf[w]) / delta);
                    if (face_open(A, isg, u_f, rm[w], rm[q])) {
                        aW[q] = aW[q] + af * d_f * Ar[w] / delta;
                        Su[q] = Su[q] + af * u_f * Ar[w];
                        *flux_ref = *flux_ref + fabs(af * u_f * Ar[w]);
                    }
                }
                if (LINK(e)) {
                    d_f = DF(apr, e);
                    af = 0.5 * (aef[q] + aef[e]);
                    delta = r[i + 2] - r[i + 1];
                    u_f = 0.5 * (ur[q] + ur[e]) +
                          d_f * (0.5 * (gr[q] + gr[e]) - (pf[e] - pf[q]) / delta);
                    if (face_open(A, isg, u_f, rm[q], rm[e])) {
                        aE[q] = aE[q] + af * d_f * Ar[q] / delta;
                        Su[q] = Su[q] - af * u_f * Ar[q];
                        *flux_ref = *flux_ref + fabs(af * u_f * Ar[q]);
                        if (export_) {
                            Fs_r[q] = af * u_f * Ar[q];
                            ac_r[q] = af * d_f * Ar[q] / delta;
                            lk_r[q] = 1;
                        }
                    }
                }
                if (LINK(s)) {
                    d_f = DF(apt, s);
                    af = 0.5 * (aef[q] + aef[s]);
                    delta = r[i + 1] * (th[j + 1] - th[j]);
                    u_f = 0.5 * (uth[s] + uth[q]) +
                          d_f * (0.5 * (gth[s] + gth[q]) - (pf[q] - pf[s]) / delta);
                    if (face_open(A, isg, u_f, rm[s], rm[q])) {
                        aS[q] = aS[q] + af * d_f * Ath[q] / delta;
                        Su[q] = Su[q] + af * u_f * Ath[q];
                        *flux_ref = *flux_ref + fabs(af * u_f * Ath[q]);
                    }
                }
                if (LINK(n)) {
                    d_f = DF(apt, n);
                    af = 0.5 * (aef[q] + aef[n]);
                    delta = r[i + 1] * (th[j + 2] - th[j + 1]);
                    u_f = 0.5 * (uth[q] + uth[n]) +
                          d_f * (0.5 * (gth[q] + gth[n]) - (pf[n] - pf[q]) / delta);
                    if (face_open(A, isg, u_f, rm[q], rm[n])) {
                        aN[q] = aN[q] + af * d_f * Ath[q] / delta;
                        Su[q] = Su[q] - af * u_f * Ath[q];
                        *flux_ref = *flux_ref + fabs(af * u_f * Ath[q]);
                        if (export_) {
                            Fs_th[q] = af * u_f * Ath[q];
                            ac_th[q] = af * d_f * Ath[q] / delta;
                            lk_th[q] = 1;
                        }
                    }
                }
                if (LINK(b)) {
                    d_f = DF(apz, b);
                    af = 0.5 * (aef[q] + aef[b]);
                    delta = z[k + 1] - z[k];
                    const double lw = isg ? liq_weight_f(A, b, q) : 0.0;
                    u_f = 0.5 * (uz[b] + uz[q]) +
                          d_f * (0.5 * (gz[b] + gz[q]) - (pf[q] - pf[b]) / delta - lw);
                    if (face_open(A, isg, u_f, rm[b], rm[q])) {
                        aB[q] = aB[q] + af * d_f * Az[b] / delta;
                        Su[q] = Su[q] + af * u_f * Az[b];
                        *flux_ref = *flux_ref + fabs(af * u_f * Az[b]);
                    }
                }
                if (LINK(t)) {
                    d_f = DF(apz, t);
                    af = 0.5 * (aef[q] + aef[t]);
                    delta = z[k + 2] - z[k + 1];
                    const double lw = isg ? liq_weight_f(A, q, t) : 0.0;
                    u_f = 0.5 * (uz[q] + uz[t]) +
                          d_f * (0.5 * (gz[q] + gz[t]) - (pf[t] - pf[q]) / delta - lw);
                    if (face_open(A, isg, u_f, rm[q], rm[t])) {
                        aT[q] = aT[q] + af * d_f * Az[q] / delta;
                        Su[q] = Su[q] - af * u_f * Az[q];
                        *flux_ref = *flux_ref + fabs(af * u_f * Az[q]);
                        if (export_) {
                            Fs_z[q] = af * u_f * Az[q];
                            ac_z[q] = af * d_f * Az[q] / delta;
                            lk_z[q] = 1;
                        }
                    }
                }
            }
#undef LINK
#undef DF
}

int eaf_oracle_pressure_assemble(int nr, int nth, int nz, double* const* dv, int* const* iv,
                                 int flags, const double* sc, double* residual) {
    if (nr < 1 || nth < 1 || nz < 1) return 2;
    const dims_t D = mkdims(nr, nth, nz);
    const dims_t* d = &D;
    asm_t A = {d, dv, iv, flags, sc};
    const int gas_in = (flags & 2) != 0, gas_comp = (flags & 4) != 0;
    double* g = (double*)malloc(sizeof(double) * 6 * d->n);
    if (!g) return 6;
    double *gpr = g, *gpth = g + d->n, *gpz = g + 2 * d->n;
    double *gpr_g = g + 3 * d->n, *gpth_g = g + 4 * d->n, *gpz_g = g + 5 * d->n;
    /* (:140-146, :171-173) whole arrays zeroed */
    for (int a = 27; a <= 44; ++a) memset(dv[a], 0, d->n * sizeof(double));
    for (int a = 4; a <= 6; ++a) memset(iv[a], 0, d->n * sizeof(int));
    /* (:180-185) */
    cell_gradients(&A, 0, gpr, gpth, gpz);
    if (gas_in) cell_gradients(&A, 1, gpr_g, gpth_g, gpz_g);
    /* (:205-210) */
    double flux_ref = 0.0;
    add_phase(&A, 9, iv[2], 1, gpr, gpth, gpz, 0, &flux_ref);
    if (gas_in) add_phase(&A, 18, iv[3], 0, gpr_g, gpth_g, gpz_g, 1, &flux_ref);
    double *aW = dv[27], *aE = dv[28], *aS = dv[29], *aN = dv[30], *aB = dv[31],
           *aT = dv[32], *aP = dv[33], *Su = dv[34];
    const int *ct = iv[0], *out = iv[1], *act_l = iv[2], *act_g = iv[3];
    const double *vol = dv[0], *al_g = dv[18], *rho_g = dv[19], *Told = dv[26],
                 *al_l = dv[9], *rho_l = dv[10];
    const double dt = sc[0], rho_gas = sc[1], Tamb = sc[2];
    /* (:228-247) gas compressibility source */
    if (gas_comp) {
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nth; ++j)
                for (int i = 1; i <= nr; ++i) {
                    const size_t q = at(d, i, j, k);
                    if (ct[q] == 0) continue;
                    if (!act_g[q]) continue;
                    const double src = al_g[q] * vol[q] / dt *
                                       (rho_g[q] - rho_gas * Tamb / fmax(Told[q], T_MIN_GAS_C)) /
                                       fmax(rho_g[q], SMALL);
                    const double cap = COMP_SRC_CAP_C * al_g[q] * vol[q] / dt;
                    Su[q] = Su[q] - fmax(-cap, fmin(cap, src));
                }
    }
    /* (:250-285) trivial cells and the diagonal */
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (ct[q] == 0) continue;
                if (!act_l[q] && !act_g[q]) {
                    aW[q] = 0.0; aE[q] = 0.0; aS[q] = 0.0; aN[q] = 0.0;
                    aB[q] = 0.0; aT[q] = 0.0; aP[q] = 1.0; Su[q] = 0.0;
                } else {
                    aP[q] = (aW[q] + aE[q] + aS[q] + aN[q] + aB[q] + aT[q]) *
                            (1.0 + PP_COMPLIANCE_C);
                    if (gas_comp && act_g[q])
                        aP[q] = aP[q] + al_g[q] / P0_THERMO_C * vol[q] / dt;
                    if (act_l[q])
                        aP[q] = aP[q] + al_l[q] * vol[q] /
                                            (rho_l[q] * (C_SOUND_LIQ_C * C_SOUND_LIQ_C) * dt);
                }
            }
    /* apply_pressure_bc (src/mod_boundary_3d.f90:180-277), serial */
#define OUT(x) (out[x] != 0 && (x) / d->sxy == (size_t)(nz + 1))
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (ct[q] == 0) {
                    aW[q] = 0.0; aE[q] = 0.0; aS[q] = 0.0; aN[q] = 0.0;
                    aB[q] = 0.0; aT[q] = 0.0; aP[q] = 1.0; Su[q] = 0.0;
                    continue;
                }
                if (i == 1) aW[q] = 0.0;
                if (i == nr) aE[q] = 0.0;
                if (k == 1) aB[q] = 0.0;
                if (k == nz) {
                    if (OUT(q)) {
                        aW[q] = 0.0; aE[q] = 0.0; aS[q] = 0.0; aN[q] = 0.0;
                        aB[q] = 0.0; aT[q] = 0.0; aP[q] = 1.0; Su[q] = 0.0;
                        continue;
                    }
                    aT[q] = 0.0;
                }
                if (i > 1 && ct[q - 1] == 0) aW[q] = 0.0;
                if (i < nr && ct[q + 1] == 0) aE[q] = 0.0;
                if (k > 1 && ct[q - d->sxy] == 0) aB[q] = 0.0;
                if (k < nz && ct[q + d->sxy] == 0) aT[q] = 0.0;
                if (OUT(q - 1)) aW[q] = 0.0;
                if (OUT(q + 1)) aE[q] = 0.0;
                if (OUT(q - d->sx)) aS[q] = 0.0;
                if (OUT(q + d->sx)) aN[q] = 0.0;
                if (OUT(q - d->sxy)) aB[q] = 0.0;
                if (OUT(q + d->sxy)) aT[q] = 0.0;
            }
#undef OUT
    /* (:292-307) continuity residual */
    double sum_su = 0.0;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nth; ++j)
            for (int i = 1; i <= nr; ++i) {
                const size_t q = at(d, i, j, k);
                if (ct[q] == 0) continue;
                if (act_l[q] || act_g[q]) sum_su = sum_su + fabs(Su[q]);
            }
    *residual = sum_su / fmax(flux_ref, SMALL);
    free(g);
    return 0;
}
