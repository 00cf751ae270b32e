"""Mixed-precision solve (FP32 inner CG, FP64 refinement) through the C ABI.

The convergence test of the mixed form is the FP64 relative residual
||Su - A phi|| / ||Su||, recomputed here independently in numpy. Its error
is stated against the FP64 oracle solve of the same system. Two solvers
that stop at the same residual differ in the solution by up to about
cond(A) times that residual: FP64 CG runs that differ only in rounding
follow nearly the same Krylov path (3e-9 apart at tol 1e-8), but refinement
with FP32 inner solves lands elsewhere in the residual ball -- measured
1e-8 (12x24x16) to 1.1e-7 (18x36x24) at tol 1e-8. The bounds below are
those measurements with margin; at tol 1e-10 the error falls under 1e-8.
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu


def true_residual(s, phi):
    g = gen()
    r = g.interior(s.Su) - g.apply_operator(s, phi)
    return float(np.linalg.norm(r) / np.linalg.norm(g.interior(s.Su)))


def rel_l2(a, b):
    g = gen()
    return float(np.linalg.norm(g.interior(a) - g.interior(b)) /
                 np.linalg.norm(g.interior(b)))


def mixed(s, phi, tol, inner_tol=0.1, max_outer=60, max_inner=4000):
    eaf = pkg()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        return cg.solve_mixed(s.arrays(), phi, tol=tol, inner_tol=inner_tol,
                              max_outer=max_outer, max_inner=max_inner)


@pytest.mark.parametrize("dims,tol,err_bound", [
    ((12, 24, 16, 8), 1e-8, 5e-7),
    ((12, 24, 16, 8), 1e-10, 1e-8),
    ((18, 36, 24, 8), 1e-8, 5e-7),
    ((18, 36, 24, 8), 1e-10, 1e-8),
])
def test_mixed_converges_and_matches_fp64_oracle(dims, tol, err_bound):
    import oracle
    g = gen()
    s = g.make_system(*dims, seed=1)
    phi = g.zeros_phi(*dims[:3])
    res, nit, nout, st = mixed(s, phi, tol)
    assert st == 0 and res < tol and nout >= 1 and nit > 0
    assert true_residual(s, phi) < tol * 1.001
    ref = g.zeros_phi(*dims[:3])
    r_o, n_o = oracle.cg(s, ref, 200000, tol)
    assert r_o < tol
    assert rel_l2(phi, ref) <= err_bound


def test_mixed_deterministic():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=2)
    a, b = g.zeros_phi(12, 24, 16), g.zeros_phi(12, 24, 16)
    ra = mixed(s, a, 1e-8)
    rb = mixed(s, b, 1e-8)
    assert ra == rb and np.array_equal(a, b)


def test_mixed_zero_rhs_and_max_outer_zero():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    phi0 = np.random.default_rng(1).normal(size=s.aP.shape)
    z = g.make_system(*g.SMOKE, seed=0)
    z.Su[...] = 0.0
    phi = phi0.copy()
    res, nit, nout, st = mixed(z, phi, 1e-8)
    assert (res, nit, nout, st) == (0.0, 0, 0, 0)
    assert np.array_equal(g.interior(phi), g.interior(phi0))
    phi = g.zeros_phi(12, 24, 16)
    res, nit, nout, st = mixed(s, phi, 1e-8, max_outer=0)
    assert st == 0 and nit == 0 and nout == 0 and abs(res - 1.0) < 1e-12


def test_mixed_nan_is_reported():
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    g.interior(s.aN)[3, 3, 3] = np.nan
    res, nit, nout, st = mixed(s, g.zeros_phi(12, 24, 16), 1e-8)
    assert st == eaf._lib.EAF_ENONFINITE and np.isnan(res)


def test_mixed_rejects_bad_inner_tolerance():
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    with pytest.raises(eaf.EafError):
        mixed(s, g.zeros_phi(12, 24, 16), 1e-8, inner_tol=1.5)


def test_mixed_trace_records_every_refinement_step():
    """The per-step trace: one entry per refinement step, inner iterations
    summing to the reported total, the last outer residual equal to the
    returned one, and each step but the last reaching its inner reduction
    (inner_tol, compared in FP32) unless capped."""
    eaf = pkg()
    g = gen()
    s = g.make_system(12, 24, 16, 8, seed=1)
    phi = g.zeros_phi(12, 24, 16)
    with eaf.CGSolver(12, 24, 16) as cg:
        res, nit, nout, st = cg.solve_mixed(s.arrays(), phi, tol=1e-10, inner_tol=0.1,
                                            max_outer=60, max_inner=4000)
        trace = cg.mixed_trace()
        assert len(trace) == nout and st == 0
        assert sum(t["inner_iterations"] for t in trace) == nit
        assert trace[-1]["residual"] == res
        assert all(t["inner_reduction"] <= 0.1 * (1 + 1e-6) or t["inner_iterations"] == 4000
                   for t in trace[:-1])
        cg.solve(s.arrays(), g.zeros_phi(12, 24, 16), 100, 1e-8)
        assert cg.mixed_trace() == []
