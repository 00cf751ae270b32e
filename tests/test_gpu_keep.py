"""The FP64 CG with each block's own cells' update operands kept in shared
memory, against the oracle and the per-thread-load kernel.

A thread updates the same cells in the stencil phase and the update phase of
every iteration, so its own cells' x, r, aP and A p can stay in its block's
shared memory for the whole solve; only z and the direction go to global
memory (the neighbours read them). Every per-cell operation and every sum
runs in the same order as in the per-thread-load kernel, so on one launch
shape the two are bit-identical to each other and to the oracle's plan
(grid, block): iteration count, residual and every phi value.
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

TOL = 1e-8


def solve(s, phi, max_iter, tol, block, grid, kernel):
    eaf = pkg()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        if block:
            cg.set_launch(block, grid)
        cg.set_kernel(kernel)
        res, nit, st = cg.solve(s.arrays(), phi, max_iter, tol)
        return res, nit, st, cg.last_launch(), cg.last_kernel()


def assert_keep_bitwise(s, phi0, max_iter, tol, block, grid, expect_keep=True):
    import oracle
    eaf = pkg()
    phi_k = phi0.copy()
    res_k, nit_k, st_k, plan, kern = solve(s, phi_k, max_iter, tol, block, grid,
                                           eaf.CGSolver.KERNEL_KEEP)
    assert kern == (eaf.CGSolver.KERNEL_KEEP if expect_keep else eaf.CGSolver.KERNEL_LOADS)
    phi_l = phi0.copy()
    res_l, nit_l, st_l, plan_l, kern_l = solve(s, phi_l, max_iter, tol, block, grid,
                                               eaf.CGSolver.KERNEL_LOADS)
    assert kern_l == eaf.CGSolver.KERNEL_LOADS and plan == plan_l
    assert (nit_k, st_k) == (nit_l, st_l)
    assert res_k == res_l or (np.isnan(res_k) and np.isnan(res_l))
    assert np.array_equal(phi_k, phi_l, equal_nan=True), (
        "max |diff| %g" % np.nanmax(np.abs(phi_k - phi_l)))
    phi_o = phi0.copy()
    res_o, nit_o = oracle.cg(s, phi_o, max_iter, tol, plan=plan)
    assert nit_o == nit_k and (res_o == res_k or (np.isnan(res_o) and np.isnan(res_k)))
    assert np.array_equal(phi_k, phi_o, equal_nan=True)
    return res_k, nit_k, st_k, plan


@pytest.mark.parametrize("block,grid", [(512, 148), (1024, 148), (256, 148), (512, 140),
                                        (512, 96)])
def test_production_mesh_fixed_iterations(block, grid):
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=0)
    res, nit, st, plan = assert_keep_bitwise(s, g.zeros_phi(60, 120, 84), 150, 0.0,
                                             block, grid)
    assert nit == 150 and plan == (grid, block)


@pytest.mark.parametrize("dims,block,grid", [((12, 24, 16, 8), 256, 8),
                                             ((35, 70, 50, 16), 256, 148),
                                             ((35, 70, 50, 16), 512, 148),
                                             ((9, 7, 5, 2), 64, 3),      # odd cell count
                                             ((7, 1, 9, 2), 64, 2),      # nth = 1
                                             ((6, 5, 1, 2), 64, 2),      # nz = 1
                                             ((1, 6, 7, 2), 64, 4),      # nr = 1
                                             ((3, 2, 2, 1), 64, 16)])    # empty slices
def test_meshes_to_tol(dims, block, grid):
    g = gen()
    s = g.make_system(*dims, seed=5)
    rng = np.random.default_rng(3)
    nr, nth, nz = dims[:3]
    g.interior(s.Su)[...] = rng.normal(0, 1e-3, size=(nz, nth, nr))
    res, nit, st, plan = assert_keep_bitwise(s, g.zeros_phi(nr, nth, nz), 100000, TOL,
                                             block, grid)
    assert st == 0 and res < TOL


def test_warm_start_zero_rhs_nan_and_general_form():
    eaf = pkg()
    g = gen()
    rng = np.random.default_rng(7)
    s = g.make_system(*g.SMOKE, seed=1, resolve=2)
    assert_keep_bitwise(s, rng.normal(0, 1e-4, size=s.aP.shape), 300, TOL, 256, 8)
    z = g.make_system(*g.SMOKE, seed=0)
    z.Su[...] = 0.0
    phi0 = rng.normal(size=z.aP.shape)
    res, nit, st, _ = assert_keep_bitwise(z, phi0, 100, TOL, 256, 8)
    assert (res, nit, st) == (0.0, 0, 0)
    n = g.make_system(*g.SMOKE, seed=0)
    g.interior(n.aP)[5, 6, 7] = np.nan
    res, nit, st, _ = assert_keep_bitwise(n, g.zeros_phi(12, 24, 16), 40, TOL, 256, 8)
    assert st == eaf._lib.EAF_ENONFINITE and np.isnan(res) and nit == 40
    a = g.make_system(*g.SMOKE, seed=0)
    g.interior(a.aS)[3, 4, 5] *= 1.5      # 7-array (non-symmetric) form
    assert_keep_bitwise(a, g.zeros_phi(12, 24, 16), 300, TOL, 256, 8)


def test_slice_too_large_runs_the_load_kernel():
    """At 120x240x168 on 148 blocks a slice needs 1.1 MB of shared memory:
    the per-thread-load kernel runs, with the same bits as asking for it."""
    g = gen()
    s = g.make_system(120, 240, 168, 24, seed=3)
    assert_keep_bitwise(s, g.zeros_phi(120, 240, 168), 20, 0.0, 1024, 148,
                        expect_keep=False)


def test_warm_started_repeat_solves_on_one_handle():
    """Consecutive solves on one handle (a SIMPLE loop's pressure calls) keep
    nothing between calls: each gives the bits of a fresh handle."""
    import oracle
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=4)
    phi = g.zeros_phi(60, 120, 84)
    ref = g.zeros_phi(60, 120, 84)
    with eaf.CGSolver(60, 120, 84) as cg:
        cg.set_launch(512, 148)
        cg.set_kernel(cg.KERNEL_KEEP)
        for k in range(3):
            res, nit, st = cg.solve(s.arrays(), phi, 60, 0.0)
            assert cg.last_kernel() == cg.KERNEL_KEEP
            ro, no = oracle.cg(s, ref, 60, 0.0, plan=(148, 512))
            assert (res, nit) == (ro, no) and np.array_equal(phi, ref), k


def test_concurrent_solves_on_two_host_threads():
    """Two host threads solving different meshes at once through the kept
    form (different dynamic shared-memory sizes of one kernel) get the bits
    each gets alone: the size attribute and the launch are taken together."""
    import threading
    eaf = pkg()
    g = gen()
    cases = [(g.make_system(*g.PRODUCTION, seed=6), 120), (g.make_system(35, 70, 50, 16, seed=7), 200)]

    def run(s, iters, out):
        phi = g.zeros_phi(s.nr, s.nth, s.nz)
        with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
            for _ in range(6):
                phi[...] = 0.0
                res, nit, st = cg.solve(s.arrays(), phi, iters, 0.0)
                out.append((res, nit, st, cg.last_kernel(), phi.copy()))

    alone = []
    for s, iters in cases:
        o = []
        run(s, iters, o)
        alone.append(o[0])
    outs = [[], []]
    threads = [threading.Thread(target=run, args=(s, iters, outs[i]))
               for i, (s, iters) in enumerate(cases)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i in range(2):
        assert len(outs[i]) == 6
        for res, nit, st, kern, phi in outs[i]:
            assert kern == eaf.CGSolver.KERNEL_KEEP
            assert (res, nit, st) == alone[i][:3] and np.array_equal(phi, alone[i][4])


@pytest.mark.parametrize("dims,block,grid,iters,tol", [
    ((60, 120, 84, 24), 64, 296, 150, 0.0),     # more blocks than the p.q slot form takes
    ((12, 24, 16, 8), 256, 1, 100000, TOL),     # one block: no group stage at all
    ((18, 36, 24, 8), 128, 160, 100000, TOL)])  # the slot form's largest grid
def test_grid_sizes_around_the_slot_all_reduce(dims, block, grid, iters, tol):
    """The p.q all-reduce without a release runs on flat grids of 2 to 160
    blocks; one block needs no group stage and larger grids keep the counter
    form. All give the oracle's bits for their plan."""
    g = gen()
    s = g.make_system(*dims, seed=9)
    res, nit, st, plan = assert_keep_bitwise(s, g.zeros_phi(*dims[:3]), iters, tol, block, grid)
    assert plan == (grid, block) and st == 0


@pytest.mark.parametrize("mode", [0, 1])
def test_release_free_all_reduce_waits_are_bounded(mode):
    """The p.q all-reduce's two waits -- for the arrival count (mode 0: a
    member never arrives) and for a partial whose doorbell came first (mode
    1: the partial is never written) -- give up after their bound with
    EAF_ETIMEOUT, and the context stays usable: a solve afterwards gives the
    oracle's bits."""
    import oracle
    eaf = pkg()
    g = gen()
    assert eaf.allreduce_timeout_selftest(0, 20.0, mode) == eaf._lib.EAF_ETIMEOUT
    s = g.make_system(*g.PRODUCTION, seed=2)
    phi = g.zeros_phi(60, 120, 84)
    with eaf.CGSolver(60, 120, 84) as cg:
        cg.set_launch(512, 148)
        cg.set_kernel(cg.KERNEL_KEEP)
        res, nit, st = cg.solve(s.arrays(), phi, 50, 0.0)
        assert cg.last_kernel() == cg.KERNEL_KEEP and st == 0
    ref = g.zeros_phi(60, 120, 84)
    assert oracle.cg(s, ref, 50, 0.0, plan=(148, 512)) == (res, nit)
    assert np.array_equal(phi, ref)
