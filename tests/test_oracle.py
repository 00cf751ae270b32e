"""Pins the oracle (CPU restatement of cg_3d_mpi) without a GPU.

No reference binary or reference CG golden vector exists, so the oracle is
cross-checked against independent restatements and known answers:
  * its matvec against a vectorised numpy stencil, bit for bit;
  * its full solve against a separate numpy restatement that sums dots
    sequentially (np.cumsum), bit for bit;
  * a few iterations against exact rational arithmetic (fractions);
  * converged solutions against scipy's sparse direct solve and against
    analytic known-answer systems b = A x*;
  * the reference's edge behaviour (zero RHS, max_iter 0, NaN, theta halos);
  * its kernel-order dot against a pure-Python model of the CUDA reduction.
"""
import math
from fractions import Fraction

import numpy as np
import pytest

from conftest import gen

SMALL = 1e-30


def seq_dot(a, b):
    return float(np.cumsum((a * b).ravel())[-1])


def numpy_cg(s, phi, max_iter, tol):
    """Second restatement of src/mod_solver_3d.f90:485-620 (numpy)."""
    g = gen()
    I = g.interior
    guard = lambda v: np.where(v > SMALL, v, SMALL)
    q = g.apply_operator(s, phi)
    r = I(s.Su) - q
    bnorm = math.sqrt(seq_dot(I(s.Su), I(s.Su)))
    wrap(phi)
    if bnorm < SMALL:
        return 0.0, 0
    d = guard(np.abs(I(s.aP)))
    z = r / d
    p = np.zeros_like(phi)
    I(p)[...] = z
    rz = seq_dot(r, z)
    res = math.sqrt(seq_dot(r, r)) / bnorm
    nit = 0
    for it in range(1, max_iter + 1):
        qv = g.apply_operator(s, p)
        pq = seq_dot(I(p), qv)
        if abs(pq) < SMALL:
            break
        alpha = rz / pq
        I(phi)[...] = I(phi) + alpha * I(p)
        r = r - alpha * qv
        res = math.sqrt(seq_dot(r, r)) / bnorm
        nit = it
        if res < tol:
            break
        z = r / d
        rzn = seq_dot(r, z)
        beta = rzn / max(rz, SMALL) if rz > SMALL else rzn / SMALL
        rz = rzn
        I(p)[...] = z + beta * I(p)
    wrap(phi)
    return res, nit


def wrap(x):
    nth = x.shape[1] - 4
    x[:, 1, :] = x[:, nth + 1, :]
    x[:, 0, :] = x[:, nth, :]
    x[:, nth + 2, :] = x[:, 2, :]
    x[:, nth + 3, :] = x[:, 3, :]


def test_matvec_bitwise_vs_numpy(orc):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    x = np.random.default_rng(0).normal(size=s.aP.shape)
    y = orc.matvec(s, x.copy())
    assert np.array_equal(g.interior(y), g.apply_operator(s, x))
    # y is zero outside the interior, as `y = 0.0_dp` leaves it
    y2 = y.copy()
    g.interior(y2)[...] = 0
    assert not y2.any()


def test_full_solve_bitwise_vs_numpy_restatement(orc):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    p1 = g.zeros_phi(12, 24, 16)
    r1, n1 = orc.cg(s, p1, 100000, 1e-8)
    p2 = g.zeros_phi(12, 24, 16)
    r2, n2 = numpy_cg(s, p2, 100000, 1e-8)
    assert (n1, r1) == (n2, r2)
    assert np.array_equal(p1, p2)


def test_warm_start_bitwise_vs_numpy_restatement(orc):
    g = gen()
    s = g.make_system(6, 8, 10, 3, seed=5, resolve=1)
    phi0 = np.random.default_rng(3).normal(0, 1e-3, size=s.aP.shape)
    p1, p2 = phi0.copy(), phi0.copy()
    assert orc.cg(s, p1, 500, 1e-9) == numpy_cg(s, p2, 500, 1e-9)
    assert np.array_equal(p1, p2)


def test_few_iterations_vs_exact_rational(orc):
    g = gen()
    s = g.make_system(3, 4, 2, 1, seed=11)
    n_it = 4
    phi = g.zeros_phi(3, 4, 2)
    orc.cg(s, phi, n_it, 0.0)
    # exact CG in rationals on the dense operator
    A, b = dense_operator(s)
    F = Fraction
    Af = [[F(v) for v in row] for row in A]
    bf = [F(v) for v in b]
    d = [max(abs(Af[i][i]), F(SMALL)) for i in range(len(bf))]
    x = [F(0)] * len(bf)
    r = bf[:]
    z = [r[i] / d[i] for i in range(len(r))]
    p = z[:]
    rz = sum(r[i] * z[i] for i in range(len(r)))
    for _ in range(n_it):
        q = [sum(Af[i][j] * p[j] for j in range(len(p))) for i in range(len(p))]
        alpha = rz / sum(p[i] * q[i] for i in range(len(p)))
        x = [x[i] + alpha * p[i] for i in range(len(x))]
        r = [r[i] - alpha * q[i] for i in range(len(r))]
        z = [r[i] / d[i] for i in range(len(r))]
        rzn = sum(r[i] * z[i] for i in range(len(r)))
        beta = rzn / rz
        rz = rzn
        p = [z[i] + beta * p[i] for i in range(len(p))]
    xe = np.array([float(v) for v in x])
    got = g.interior(phi).ravel()
    assert np.linalg.norm(got - xe) <= 1e-12 * np.linalg.norm(xe)


def dense_operator(s):
    """Dense A and b of a (small) system, compact order, theta wrapped."""
    g = gen()
    nr, nth, nz = s.nr, s.nth, s.nz
    n = nr * nth * nz
    A = np.zeros((n, n))
    I = g.interior
    idx = lambda i, j, k: i + nr * (j + nth * k)
    for k in range(nz):
        for j in range(nth):
            for i in range(nr):
                c = idx(i, j, k)
                A[c, c] += I(s.aP)[k, j, i]
                if i > 0:
                    A[c, idx(i - 1, j, k)] -= I(s.aW)[k, j, i]
                if i < nr - 1:
                    A[c, idx(i + 1, j, k)] -= I(s.aE)[k, j, i]
                A[c, idx(i, (j - 1) % nth, k)] -= I(s.aS)[k, j, i]
                A[c, idx(i, (j + 1) % nth, k)] -= I(s.aN)[k, j, i]
                if k > 0:
                    A[c, idx(i, j, k - 1)] -= I(s.aB)[k, j, i]
                if k < nz - 1:
                    A[c, idx(i, j, k + 1)] -= I(s.aT)[k, j, i]
    return A, I(s.Su).ravel().copy()


def sparse_operator(s):
    import scipy.sparse as sp
    g = gen()
    nr, nth, nz = s.nr, s.nth, s.nz
    I = g.interior
    k, j, i = np.meshgrid(np.arange(nz), np.arange(nth), np.arange(nr), indexing="ij")
    c = (i + nr * (j + nth * k)).ravel()
    rows, cols, vals = [c], [c], [I(s.aP).ravel()]
    for arr, di, dj, dk in ((s.aW, -1, 0, 0), (s.aE, 1, 0, 0), (s.aS, 0, -1, 0),
                            (s.aN, 0, 1, 0), (s.aB, 0, 0, -1), (s.aT, 0, 0, 1)):
        ii, jj, kk = i + di, (j + dj) % nth, k + dk
        ok = ((ii >= 0) & (ii < nr) & (kk >= 0) & (kk < nz)).ravel()
        cc = (np.clip(ii, 0, nr - 1) + nr * (jj + nth * np.clip(kk, 0, nz - 1))).ravel()
        rows.append(c[ok]); cols.append(cc[ok]); vals.append(-I(arr).ravel()[ok])
    n = nr * nth * nz
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                                                 np.concatenate(cols))), shape=(n, n))


def test_converged_solution_vs_scipy_direct(orc):
    import scipy.sparse.linalg as spla
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    A = sparse_operator(s)
    xd = spla.spsolve(A.tocsc(), g.interior(s.Su).ravel())
    phi = g.zeros_phi(12, 24, 16)
    res, nit = orc.cg(s, phi, 100000, 1e-13)
    assert res < 1e-13
    got = g.interior(phi).ravel()
    assert np.linalg.norm(got - xd) <= 1e-8 * np.linalg.norm(xd)
    # the operator is symmetric by construction
    assert abs(A - A.T).max() == 0.0


def test_known_answer_system(orc):
    g = gen()
    s, xs = g.make_known_answer(18, 36, 24, 8, seed=2)
    phi = g.zeros_phi(18, 36, 24)
    res, nit = orc.cg(s, phi, 100000, 1e-14)
    assert res < 1e-14
    err = np.linalg.norm(g.interior(phi) - g.interior(xs)) / np.linalg.norm(g.interior(xs))
    assert err < 1e-7


def test_zero_rhs_returns_early_with_theta_fill(orc):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    s.Su[...] = 0
    phi = np.random.default_rng(0).normal(size=s.aP.shape)
    ref = phi.copy()
    assert orc.cg(s, phi, 100, 1e-8) == (0.0, 0)
    assert np.array_equal(g.interior(phi), g.interior(ref))
    wrap(ref)
    assert np.array_equal(phi, ref)


def test_nan_runs_to_max_iter(orc):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    g.interior(s.aE)[1, 2, 3] = np.nan
    phi = g.zeros_phi(12, 24, 16)
    res, nit = orc.cg(s, phi, 25, 1e-8)
    assert math.isnan(res) and nit == 25
    assert np.isnan(g.interior(phi)).all()


def test_max_iter_zero(orc):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    phi = g.zeros_phi(12, 24, 16)
    res, nit = orc.cg(s, phi, 0, 1e-8)
    assert nit == 0 and abs(res - 1.0) < 1e-15   # x0 = 0: r = b
    assert not g.interior(phi).any()


def py_tree_dot(a, b, G, B, C=1):
    """Pure-Python model of the CUDA reduction tree (cg_common.cuh) and, with
    C > 1, of the cluster all-reduce (cluster_red.cuh): block partials of a
    cluster folded in rank order from the first, the cluster partials in
    place of the block partials in the last stage."""
    prod = (a * b).ravel()
    n = prod.size
    chunk = -(-n // G)

    def bfly(v):
        v = list(v)
        for o in (16, 8, 4, 2, 1):
            v = [v[l] + v[l ^ o] for l in range(32)]
        return v[0]

    parts = []
    for gb in range(G):
        beg = min(n, gb * chunk)
        end = min(n, beg + chunk)
        lanes = []
        for t in range(B):
            sacc = 0.0
            for c in range(beg + t, end, B):
                sacc = sacc + float(prod[c])
            lanes.append(sacc)
        nw = -(-B // 32)
        ws = [bfly([lanes[w * 32 + l] if w * 32 + l < B else 0.0 for l in range(32)])
              for w in range(nw)]
        parts.append(bfly(ws + [0.0] * (32 - nw)))
    if C > 1:
        cps = []
        for c0 in range(0, G, C):
            cp = parts[c0]
            for r in range(1, C):
                cp = cp + parts[c0 + r]
            cps.append(cp)
        parts = cps
    if len(parts) == 1:
        return parts[0]
    return bfly([sum_seq(parts[l::32]) for l in range(32)])


def sum_seq(v):
    s = 0.0
    for x in v:
        s = s + x
    return s


@pytest.mark.parametrize("plan", [(1, 1024), (3, 64), (40, 128), (70, 32)])
def test_kernel_order_dot_matches_python_model(orc, plan):
    g = gen()
    rng = np.random.default_rng(9)
    a = rng.normal(size=g.halo_shape(12, 24, 16))
    b = rng.normal(size=a.shape)
    got = orc.dot(12, 24, 16, a, b, plan)
    want = py_tree_dot(g.interior(a), g.interior(b), *plan)
    assert got == want
    assert abs(got - orc.dot(12, 24, 16, a, b)) < 1e-9


@pytest.mark.parametrize("plan", [(16, 288, 16), (8, 64, 2), (40, 32, 4), (148, 32, 4),
                                  (150, 32, 2), (16, 128, 1)])
def test_cluster_plan_dot_matches_python_model(orc, plan):
    """The oracle's cluster association (one cluster, several, more than 32
    and more than 64 clusters) against the Python model; C = 1 is the flat
    association."""
    g = gen()
    rng = np.random.default_rng(10)
    a = rng.normal(size=g.halo_shape(12, 24, 16))
    b = rng.normal(size=a.shape)
    got = orc.dot(12, 24, 16, a, b, plan)
    assert got == py_tree_dot(g.interior(a), g.interior(b), *plan)
    if plan[2] == 1:
        assert got == orc.dot(12, 24, 16, a, b, plan[:2])


def test_cluster_plan_of_one_block_clusters_equals_flat_plan(orc):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    p1, p2 = g.zeros_phi(12, 24, 16), g.zeros_phi(12, 24, 16)
    assert orc.cg(s, p1, 200, 0.0, plan=(9, 256)) == orc.cg(s, p2, 200, 0.0, plan=(9, 256, 1))
    assert np.array_equal(p1, p2)


def test_kernel_order_solve_agrees_with_sequential_closely(orc):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    p1 = g.zeros_phi(12, 24, 16)
    p2 = g.zeros_phi(12, 24, 16)
    orc.cg(s, p1, 60, 0.0)
    orc.cg(s, p2, 60, 0.0, plan=(3, 512))
    I = g.interior
    assert np.linalg.norm(I(p1) - I(p2)) <= 1e-13 * np.linalg.norm(I(p1))


@pytest.mark.parametrize("dims,seed", [((12, 24, 16), 0), ((18, 36, 24), 1)])
def test_single_reduction_form_reaches_the_reference_ball(dims, seed):
    """oracle.cg1 (Chronopoulos-Gear rearrangement): same tolerance, iteration
    count within a few per cent of the reference recurrences in the kernels'
    association, solution within the spread of two correct FP64 CGs."""
    import oracle
    g = gen()
    s = g.make_system(*dims, nsph=8, seed=seed)
    plan = (8, 256)
    a = g.zeros_phi(*dims)
    b = g.zeros_phi(*dims)
    ra, na = oracle.cg(s, a, 100000, 1e-8, plan=plan)
    rb, nb = oracle.cg1(s, b, 100000, 1e-8, plan=plan)
    assert ra < 1e-8 and rb < 1e-8
    assert abs(na - nb) <= max(2, 0.06 * na), (na, nb)
    ia, ib = g.interior(a), g.interior(b)
    assert np.linalg.norm(ia - ib) / np.linalg.norm(ia) < 2e-8
    # the theta-halo post-condition holds for the new form too
    nth = dims[1]
    assert np.array_equal(b[:, 1, :], b[:, nth + 1, :])
