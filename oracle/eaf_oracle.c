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
    double tot;
    if (G == 1) {
        tot = part[0];
    } else {
        double v[32];
        for (int l = 0; l < 32; ++l) {
            double s = 0.0;
            for (int g = l; g < G; g += 32) s = s + part[g];
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
    plan_t seq = {0, 0};
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
    plan_t pl = {G, B};
    return cg_impl(nr, nth, nz, aW, aE, aS, aN, aB, aT, aP, Su, phi, max_iter,
                   tol, residual, n_iter, 1, pl);
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
    plan_t seq = {0, 0};
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
    matvec(&o, x, y);
}

int eaf_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
