"""Pins the oracle's line-by-line TDMA and residual restatements on the CPU.

tdma_3d_mpi (src/mod_solver_3d.f90:252-366, serial branch) and
compute_residual_3d_mpi (:625-694) have no golden vectors in the reference
(it is Fortran + MPI, nothing here can build it, and its tests pin whole-run
outcomes), so the C restatement is cross-checked:
  * bit for bit against a second, pure-Python restatement (scalar IEEE
    doubles, the reference's statement and operand order) on tiny meshes,
    including one-cell lines and one-cell-thick meshes;
  * by meaning: many sweeps of a diagonally dominant system converge to the
    direct sparse solution of the same theta-periodic operator;
  * its residual against the Python restatement (sequential sum, bitwise)
    and in the CUDA association (plan) against the sequential one.
"""
import math

import numpy as np
import pytest

from conftest import gen

SMALL = 1e-30


def _idx(i, j, k):
    """Fortran (i, j, k) -> numpy index of the (nz+4, nth+4, nr+4) array."""
    return (k + 1, j + 1, i + 1)


def py_wrap(phi, nr, nth, nz):
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            phi[_idx(i, 0, k)] = phi[_idx(i, nth, k)]
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            phi[_idx(i, -1, k)] = phi[_idx(i, nth - 1, k)]
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            phi[_idx(i, nth + 1, k)] = phi[_idx(i, 1, k)]
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            phi[_idx(i, nth + 2, k)] = phi[_idx(i, 2, k)]


def py_thomas(a, b, c, d):
    n = len(b)
    cp = [0.0] * n
    dp = [0.0] * n
    b1 = b[0]
    if abs(b1) < SMALL:
        b1 = math.copysign(SMALL, b1)
    cp[0] = c[0] / b1
    dp[0] = d[0] / b1
    for i in range(1, n):
        m = b[i] - a[i] * cp[i - 1]
        if abs(m) < SMALL:
            m = math.copysign(SMALL, m)
        cp[i] = c[i] / m
        dp[i] = (d[i] - a[i] * dp[i - 1]) / m
    x = [0.0] * n
    x[n - 1] = dp[n - 1]
    for i in range(n - 2, -1, -1):
        x[i] = dp[i] - cp[i] * x[i + 1]
    return x


def py_tdma(s, phi, n_sweep):
    """Second restatement of the serial tdma_3d_mpi, scalar Python."""
    nr, nth, nz = s.nr, s.nth, s.nz
    W, E, S, N, B, T, P, U = [a.tolist() for a in s.arrays()]
    f = phi.tolist()

    def g(arr, i, j, k):
        return arr[k + 1][j + 1][i + 1]

    def wrap():
        a = np.array(f)
        py_wrap(a, nr, nth, nz)
        return a.tolist()

    for _ in range(n_sweep):
        f = wrap()
        for k in range(1, nz + 1):
            for j in range(1, nth + 1):
                a, b, c, d = [], [], [], []
                for i in range(1, nr + 1):
                    a.append(-g(W, i, j, k))
                    b.append(g(P, i, j, k))
                    c.append(-g(E, i, j, k))
                    t = g(U, i, j, k) + g(S, i, j, k) * g(f, i, j - 1, k) \
                        + g(N, i, j, k) * g(f, i, j + 1, k)
                    d.append(t + g(B, i, j, k) * g(f, i, j, k - 1)
                             + g(T, i, j, k) * g(f, i, j, k + 1))
                d[0] = d[0] + g(W, 1, j, k) * g(f, 0, j, k)
                d[-1] = d[-1] + g(E, nr, j, k) * g(f, nr + 1, j, k)
                x = py_thomas(a, b, c, d)
                for i in range(1, nr + 1):
                    f[k + 1][j + 1][i + 1] = x[i - 1]
        f = wrap()
        for k in range(1, nz + 1):
            for i in range(1, nr + 1):
                a, b, c, d = [], [], [], []
                for j in range(1, nth + 1):
                    a.append(-g(S, i, j, k))
                    b.append(g(P, i, j, k))
                    c.append(-g(N, i, j, k))
                    t = g(U, i, j, k)
                    t = t + g(W, i, j, k) * g(f, i - 1, j, k) \
                        + g(E, i, j, k) * g(f, i + 1, j, k)
                    d.append(t + g(B, i, j, k) * g(f, i, j, k - 1)
                             + g(T, i, j, k) * g(f, i, j, k + 1))
                d[0] = d[0] + g(S, i, 1, k) * g(f, i, 0, k)
                d[-1] = d[-1] + g(N, i, nth, k) * g(f, i, nth + 1, k)
                x = py_thomas(a, b, c, d)
                for j in range(1, nth + 1):
                    f[k + 1][j + 1][i + 1] = x[j - 1]
        f = wrap()
        for j in range(1, nth + 1):
            for i in range(1, nr + 1):
                a, b, c, d = [], [], [], []
                for k in range(1, nz + 1):
                    a.append(-g(B, i, j, k))
                    b.append(g(P, i, j, k))
                    c.append(-g(T, i, j, k))
                    t = g(U, i, j, k) + g(S, i, j, k) * g(f, i, j - 1, k) \
                        + g(N, i, j, k) * g(f, i, j + 1, k)
                    d.append(t + g(W, i, j, k) * g(f, i - 1, j, k)
                             + g(E, i, j, k) * g(f, i + 1, j, k))
                d[0] = d[0] + g(B, i, j, 1) * g(f, i, j, 0)
                d[-1] = d[-1] + g(T, i, j, nz) * g(f, i, j, nz + 1)
                x = py_thomas(a, b, c, d)
                for k in range(1, nz + 1):
                    f[k + 1][j + 1][i + 1] = x[k - 1]
    phi[...] = np.array(f)


def py_residual(s, phi):
    nr, nth, nz = s.nr, s.nth, s.nz
    W, E, S, N, B, T, P, U = [a.tolist() for a in s.arrays()]
    f = phi.tolist()
    sr = 0.0
    sb = 0.0
    for k in range(1, nz + 1):
        for j in range(1, nth + 1):
            for i in range(1, nr + 1):
                q = (k + 1, j + 1, i + 1)
                def v(a, di=0, dj=0, dk=0):
                    return a[q[0] + dk][q[1] + dj][q[2] + di]
                if (v(P) == 1.0 and v(W) == 0.0 and v(E) == 0.0 and v(S) == 0.0
                        and v(N) == 0.0 and v(B) == 0.0 and v(T) == 0.0):
                    continue
                r = v(U) - v(P) * v(f) + v(S) * v(f, dj=-1) + v(N) * v(f, dj=1)
                r = r + v(W) * v(f, di=-1) + v(E) * v(f, di=1)
                r = r + v(B) * v(f, dk=-1) + v(T) * v(f, dk=1)
                sr = sr + r * r
                t = abs(v(U)) + abs(v(P) * v(f)) + SMALL
                sb = sb + t * t
    return math.sqrt(sr) / (math.sqrt(sb) + SMALL)


def random_phi(rng, nr, nth, nz):
    """Initial phi with nonzero values everywhere, halos included (the r/z
    halos meet zero wall links: 0 * h must be formed as the reference does)."""
    return rng.normal(0.0, 1.0, size=gen().halo_shape(nr, nth, nz))


@pytest.mark.parametrize("dims", [(3, 4, 3), (1, 1, 1), (2, 1, 3), (1, 5, 2),
                                  (4, 2, 1), (5, 3, 4)])
@pytest.mark.parametrize("n_sweep", [1, 2])
def test_tdma_matches_python_restatement_bitwise(orc, dims, n_sweep):
    g = gen()
    nr, nth, nz = dims
    s = g.make_transport_system(nr, nth, nz, seed=11, trivial_frac=0.15)
    rng = np.random.default_rng(3)
    phi0 = random_phi(rng, nr, nth, nz)
    a = phi0.copy()
    b = phi0.copy()
    orc.tdma_3d(s, a, n_sweep)
    py_tdma(s, b, n_sweep)
    assert np.array_equal(a, b)


def test_tdma_pressure_system_matches_python_bitwise(orc):
    """The symmetric pressure operator (pinned cell, folded links) too."""
    g = gen()
    s = g.make_system(5, 6, 4, nsph=2, seed=4)
    phi0 = g.zeros_phi(5, 6, 4)
    a = phi0.copy()
    b = phi0.copy()
    orc.tdma_3d(s, a, 3)
    py_tdma(s, b, 3)
    assert np.array_equal(a, b)


def _sparse_operator(s):
    """The 7-point operator with theta wrap as a scipy sparse matrix over the
    interior (r/z wall links are zero by construction)."""
    import scipy.sparse as sp
    g = gen()
    nr, nth, nz = s.nr, s.nth, s.nz
    I = g.interior
    idx = np.arange(nr * nth * nz).reshape(nz, nth, nr)
    rows, cols, vals = [], [], []

    def add(coef, di, dj, dk, sign):
        c = I(coef)
        kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(nth), np.arange(nr),
                                 indexing="ij")
        ni, nj, nk = ii + di, (jj + dj) % nth, kk + dk
        ok = (ni >= 0) & (ni < nr) & (nk >= 0) & (nk < nz) & (c != 0.0)
        rows.append(idx[ok])
        cols.append(idx[nk[ok], nj[ok], ni[ok]])
        vals.append(sign * c[ok])

    add(s.aP, 0, 0, 0, 1.0)
    add(s.aW, -1, 0, 0, -1.0)
    add(s.aE, 1, 0, 0, -1.0)
    add(s.aS, 0, -1, 0, -1.0)
    add(s.aN, 0, 1, 0, -1.0)
    add(s.aB, 0, 0, -1, -1.0)
    add(s.aT, 0, 0, 1, -1.0)
    n = nr * nth * nz
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                                                 np.concatenate(cols))), shape=(n, n))


def test_tdma_sweeps_converge_to_direct_solution(orc):
    from scipy.sparse.linalg import spsolve
    g = gen()
    s = g.make_transport_system(8, 12, 6, seed=5, sp_frac=0.3)
    A = _sparse_operator(s)
    x_star = spsolve(A.tocsc(), g.interior(s.Su).ravel())
    phi = g.zeros_phi(8, 12, 6)
    orc.tdma_3d(s, phi, 150)
    x = g.interior(phi).ravel()
    assert np.linalg.norm(x - x_star) <= 1e-10 * np.linalg.norm(x_star)
    assert orc.residual_3d(s, phi) < 1e-12


def test_residual_matches_python_and_plans(orc):
    g = gen()
    s = g.make_transport_system(7, 9, 5, seed=8, trivial_frac=0.2)
    rng = np.random.default_rng(9)
    phi = random_phi(rng, 7, 9, 5)
    r_seq = orc.residual_3d(s, phi)
    assert r_seq == py_residual(s, phi)
    for plan in [(1, 64), (3, 32), (5, 128)]:
        r_plan = orc.residual_3d(s, phi, plan=plan)
        assert abs(r_plan - r_seq) <= 1e-14 * r_seq


def test_residual_skips_identity_rows(orc):
    """All-identity system: every cell skipped, 0 / (0 + SMALL) = 0."""
    g = gen()
    s = g.make_transport_system(3, 4, 2, seed=1, trivial_frac=1.0)
    phi = random_phi(np.random.default_rng(2), 3, 4, 2)
    assert orc.residual_3d(s, phi) == 0.0
    assert orc.residual_3d(s, phi, plan=(2, 64)) == 0.0
