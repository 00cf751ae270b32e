"""The bulk-copy streaming form of the FP64 CG, against the oracle and the
per-thread-load kernel.

The streaming kernel stages each phase's operands in shared memory with
bulk copies a few tiles ahead (z-planes above and below included), but a
thread visits the same cells in the same order as the per-thread-load
kernel and every per-cell operation is the same, so on one launch shape the
two are bit-identical to each other and to the oracle's plan (grid, block):
iteration count, residual and every phi value.
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

TOL = 1e-8


def solve(s, phi, max_iter, tol, block, grid, kernel):
    eaf = pkg()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        cg.set_launch(block, grid)
        cg.set_kernel(kernel)
        res, nit, st = cg.solve(s.arrays(), phi, max_iter, tol)
        return res, nit, st, cg.last_launch(), cg.last_kernel()


def assert_stream_bitwise(s, phi0, max_iter, tol, block, grid, expect_stream=True):
    import oracle
    eaf = pkg()
    phi_s = phi0.copy()
    res_s, nit_s, st_s, plan, kern = solve(s, phi_s, max_iter, tol, block, grid,
                                           eaf.CGSolver.KERNEL_STREAM)
    if expect_stream:
        assert kern == eaf.CGSolver.KERNEL_STREAM
    phi_l = phi0.copy()
    res_l, nit_l, st_l, plan_l, kern_l = solve(s, phi_l, max_iter, tol, block, grid,
                                               eaf.CGSolver.KERNEL_LOADS)
    assert kern_l == eaf.CGSolver.KERNEL_LOADS and plan == plan_l
    assert (nit_s, st_s) == (nit_l, st_l)
    assert res_s == res_l or (np.isnan(res_s) and np.isnan(res_l))
    assert np.array_equal(phi_s, phi_l, equal_nan=True), (
        "max |diff| %g" % np.nanmax(np.abs(phi_s - phi_l)))
    phi_o = phi0.copy()
    res_o, nit_o = oracle.cg(s, phi_o, max_iter, tol, plan=plan)
    assert nit_o == nit_s and (res_o == res_s or (np.isnan(res_o) and np.isnan(res_s)))
    assert np.array_equal(phi_s, phi_o, equal_nan=True)
    return res_s, nit_s, st_s, plan


@pytest.mark.parametrize("block,grid", [(512, 148), (1024, 148), (256, 37)])
def test_production_mesh_fixed_iterations(block, grid):
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=0)
    res, nit, st, plan = assert_stream_bitwise(s, g.zeros_phi(60, 120, 84), 150, 0.0,
                                               block, grid)
    assert nit == 150 and plan == (grid, block)


def test_mesh_beyond_l2_fixed_iterations():
    g = gen()
    s = g.make_system(100, 100, 80, 16, seed=2)
    res, nit, st, plan = assert_stream_bitwise(s, g.zeros_phi(100, 100, 80), 40, 0.0,
                                               1024, 148)
    assert nit == 40


@pytest.mark.parametrize("dims,block,grid", [((12, 24, 16, 8), 256, 8),
                                             ((35, 70, 50, 16), 512, 148),
                                             ((9, 7, 5, 2), 64, 3),      # odd cell count
                                             ((7, 1, 9, 2), 64, 2),      # nth = 1
                                             ((6, 5, 1, 2), 64, 2),      # nz = 1
                                             ((1, 6, 7, 2), 64, 4)])     # nr = 1
def test_meshes_to_tol(dims, block, grid):
    g = gen()
    s = g.make_system(*dims, seed=5)
    rng = np.random.default_rng(3)
    nr, nth, nz = dims[:3]
    g.interior(s.Su)[...] = rng.normal(0, 1e-3, size=(nz, nth, nr))
    res, nit, st, plan = assert_stream_bitwise(s, g.zeros_phi(nr, nth, nz), 100000, TOL,
                                               block, grid)
    assert st == 0 and res < TOL


def test_warm_start_zero_rhs_nan_and_general_form():
    eaf = pkg()
    g = gen()
    rng = np.random.default_rng(7)
    s = g.make_system(*g.SMOKE, seed=1, resolve=2)
    assert_stream_bitwise(s, rng.normal(0, 1e-4, size=s.aP.shape), 300, TOL, 256, 8)
    z = g.make_system(*g.SMOKE, seed=0)
    z.Su[...] = 0.0
    res, nit, st, _ = assert_stream_bitwise(z, rng.normal(size=z.aP.shape), 100, TOL, 256, 8)
    assert (res, nit, st) == (0.0, 0, 0)
    n = g.make_system(*g.SMOKE, seed=0)
    g.interior(n.aP)[5, 6, 7] = np.nan
    res, nit, st, _ = assert_stream_bitwise(n, g.zeros_phi(12, 24, 16), 40, TOL, 256, 8)
    assert st == eaf._lib.EAF_ENONFINITE and np.isnan(res) and nit == 40
    a = g.make_system(*g.SMOKE, seed=0)
    g.interior(a.aS)[3, 4, 5] *= 1.5      # 7-array form: per-thread loads in-kernel
    assert_stream_bitwise(a, g.zeros_phi(12, 24, 16), 300, TOL, 256, 8, expect_stream=False)


def test_kernel_setting_is_validated():
    eaf = pkg()
    with eaf.CGSolver(12, 24, 16) as cg:
        with pytest.raises(eaf.EafError):
            cg.set_kernel(5)
        with pytest.raises(eaf.EafError):
            cg.set_kernel(-1)


@pytest.mark.parametrize("dims,block,grid,iters,tol", [((60, 120, 84, 24), 512, 148, 150, 0.0),
                                                       ((35, 70, 50, 16), 256, 148, 100000, TOL),
                                                       ((12, 24, 16, 8), 256, 8, 100000, TOL)])
def test_slot_polling_all_reduce_bitwise(dims, block, grid, iters, tol):
    """The flat grid whose all-reduce polls every block's partial in its slot
    (clusters of one block): the same association as the counter form, so the
    same bits as the per-thread-load kernel and the oracle's plan (G, B)."""
    import oracle
    eaf = pkg()
    g = gen()
    s = g.make_system(*dims, seed=1)
    phi_s = g.zeros_phi(*dims[:3])
    res_s, nit_s, st_s, plan, kern = solve(s, phi_s, iters, tol, block, grid,
                                           eaf.CGSolver.KERNEL_SLOTS)
    assert kern == eaf.CGSolver.KERNEL_SLOTS and plan == (grid, block)
    phi_l = g.zeros_phi(*dims[:3])
    res_l, nit_l, st_l, _, _ = solve(s, phi_l, iters, tol, block, grid,
                                     eaf.CGSolver.KERNEL_LOADS)
    assert (res_s, nit_s, st_s) == (res_l, nit_l, st_l) and np.array_equal(phi_s, phi_l)
    phi_o = g.zeros_phi(*dims[:3])
    assert oracle.cg(s, phi_o, iters, tol, plan=plan) == (res_s, nit_s)
    assert np.array_equal(phi_s, phi_o)
