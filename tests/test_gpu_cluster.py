"""The FP64 CG on a grid of thread-block clusters, against the oracle.

On a cluster grid the all-reduces fold the block partials through the
cluster leader's shared memory and only the leaders meet in global memory,
so the dot products are associated per cluster. The oracle's plan
(grid, block, cluster) restates that association; every other operation is
the reference's, so the solve must agree BIT FOR BIT with it: iteration
count, residual and every phi value (interior and theta halos). Against the
reference's own sequential association the cluster form is held to the same
bars as the flat form (tests/test_gpu_parity_serial.py).
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

TOL = 1e-8


def solve(s, phi, max_iter, tol, block, grid, cluster):
    eaf = pkg()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        cg.set_launch(block, grid)
        cg.set_cluster(cluster)
        res, nit, st = cg.solve(s.arrays(), phi, max_iter, tol)
        plan = cg.last_launch()
    return res, nit, st, plan


def assert_bitwise(s, phi0, max_iter, tol, block, grid, cluster):
    import oracle
    phi_g = phi0.copy()
    res_g, nit_g, st, plan = solve(s, phi_g, max_iter, tol, block, grid, cluster)
    assert len(plan) == 3 and plan[2] == cluster and plan[0] % cluster == 0, plan
    phi_o = phi0.copy()
    res_o, nit_o = oracle.cg(s, phi_o, max_iter, tol, plan=plan)
    assert nit_g == nit_o, (nit_g, nit_o, plan)
    assert res_g == res_o or (np.isnan(res_g) and np.isnan(res_o)), (res_g, res_o, plan)
    assert np.array_equal(phi_g, phi_o, equal_nan=True), (
        "max |diff| %g" % np.nanmax(np.abs(phi_g - phi_o)))
    return res_g, nit_g, st, plan


@pytest.mark.parametrize("block,grid,cluster", [(256, 2, 2), (256, 4, 4), (256, 8, 8),
                                                (128, 16, 16), (256, 8, 2), (512, 16, 4),
                                                (1024, 4, 2)])
def test_smoke_mesh_to_tol_bitwise(block, grid, cluster):
    """12x24x16 to tol: one cluster (no global stage) and several."""
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    res, nit, st, plan = assert_bitwise(s, g.zeros_phi(*g.SMOKE[:3]), 100000, TOL,
                                        block, grid, cluster)
    assert st == 0 and res < TOL


@pytest.mark.parametrize("cluster", [2, 4, 8])
def test_mid_mesh_to_tol_bitwise(cluster):
    """35x70x50 to tol across many clusters."""
    g = gen()
    s = g.make_system(35, 70, 50, 16, seed=3)
    res, nit, st, plan = assert_bitwise(s, g.zeros_phi(35, 70, 50), 100000, TOL,
                                        256, 144, cluster)
    assert st == 0 and res < TOL and plan[0] >= 8 * cluster


@pytest.mark.parametrize("block,cluster", [(512, 4), (512, 8), (1024, 8), (512, 16)])
def test_production_mesh_fixed_iterations_bitwise(block, cluster):
    """60x120x84, 150 iterations (tol 0), as many clusters as fit."""
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=0)
    res, nit, st, plan = assert_bitwise(s, g.zeros_phi(*g.PRODUCTION[:3]), 150, 0.0,
                                        block, 148, cluster)
    assert nit == 150 and plan[0] // cluster > 1


def test_warm_start_general_form_and_tiny_meshes_bitwise():
    """A warm start with halo values, the 7-array form and meshes smaller
    than the grid (blocks with empty slices) on a 4-block cluster grid."""
    g = gen()
    s = g.make_system(*g.SMOKE, seed=1, resolve=2)
    rng = np.random.default_rng(5)
    g.interior(s.aS)[3, 4, 5] *= 1.5
    assert_bitwise(s, rng.normal(0, 1e-4, size=s.aP.shape), 300, TOL, 256, 8, 4)
    for dims in [(1, 1, 1), (3, 2, 2), (5, 7, 6)]:
        t = g.make_system(*dims, nsph=2, seed=7)
        g.interior(t.Su)[...] = rng.normal(0, 1e-3, size=(dims[2], dims[1], dims[0]))
        assert_bitwise(t, g.zeros_phi(*dims), 500, TOL, 64, 8, 4)


def test_zero_rhs_max_iter_zero_and_nan():
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    z = g.make_system(*g.SMOKE, seed=0)
    z.Su[...] = 0.0
    res, nit, st, _ = assert_bitwise(z, g.zeros_phi(12, 24, 16), 100, TOL, 256, 8, 4)
    assert (res, nit, st) == (0.0, 0, 0)
    res, nit, st, _ = assert_bitwise(s, g.zeros_phi(12, 24, 16), 0, TOL, 256, 8, 4)
    assert nit == 0
    g.interior(s.aP)[5, 6, 7] = np.nan
    res, nit, st, _ = assert_bitwise(s, g.zeros_phi(12, 24, 16), 40, TOL, 256, 8, 4)
    assert st == eaf._lib.EAF_ENONFINITE and np.isnan(res) and nit == 40


def test_cluster_form_vs_serial_oracle_in_reference_regime():
    """60x120x84, 50 iterations (the reference's max_inner_pres): the same
    bars as the flat form against the sequential association."""
    import oracle
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=0)
    phi_g = g.zeros_phi(*g.PRODUCTION[:3])
    res_g, nit_g, st, plan = solve(s, phi_g, 50, TOL, 512, 148, 8)
    phi_o = g.zeros_phi(*g.PRODUCTION[:3])
    res_o, nit_o = oracle.cg(s, phi_o, 50, TOL)
    I = g.interior
    err = np.linalg.norm(I(phi_g) - I(phi_o)) / np.linalg.norm(I(phi_o))
    assert st == 0 and nit_g == nit_o and err <= 1e-10
    assert abs(res_g - res_o) <= 1e-10 * res_o


def test_cluster_setting_is_validated_and_reported():
    eaf = pkg()
    with eaf.CGSolver(12, 24, 16) as cg:
        with pytest.raises(eaf.EafError):
            cg.set_cluster(17)
        with pytest.raises(eaf.EafError):
            cg.set_cluster(-1)
        cg.set_launch(256, 8)
        cg.set_cluster(4)
        assert cg.cluster() == 4
        cg.set_cluster(1)
        assert cg.cluster() == 1


def _solve_resident(s, phi, max_iter, tol, block, cluster, resident):
    eaf = pkg()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        cg.set_launch(block, cluster)
        cg.set_cluster(cluster)
        cg.set_resident(resident)
        out = cg.solve(s.arrays(), phi, max_iter, tol)
        return out, cg.last_launch()


@pytest.mark.parametrize("dims,block,cluster", [((12, 24, 16, 8), 288, 16),
                                                ((12, 24, 16, 8), 512, 8),
                                                ((18, 36, 24, 8), 512, 16),
                                                ((18, 36, 24, 8), 1024, 16),
                                                ((10, 20, 12, 4), 256, 2)])
def test_resident_kernel_matches_global_cluster_kernel_and_oracle(dims, block, cluster):
    """A one-cluster launch keeps the system in distributed shared memory:
    the same bits as the global-memory cluster kernel and the oracle."""
    import oracle
    g = gen()
    s = g.make_system(*dims, seed=4)
    phi_r = g.zeros_phi(*dims[:3])
    (res_r, nit_r, st_r), plan = _solve_resident(s, phi_r, 100000, TOL, block, cluster, 1)
    phi_g = g.zeros_phi(*dims[:3])
    (res_g, nit_g, st_g), plan_g = _solve_resident(s, phi_g, 100000, TOL, block, cluster, 0)
    assert plan == plan_g == (cluster, block, cluster)
    assert st_r == st_g == 0 and res_r < TOL
    assert (nit_r, res_r) == (nit_g, res_g)
    assert np.array_equal(phi_r, phi_g)
    phi_b = g.zeros_phi(*dims[:3])           # mbarrier signalling
    (res_b, nit_b, st_b), plan_b = _solve_resident(s, phi_b, 100000, TOL, block, cluster, 2)
    assert plan_b == plan and (nit_b, res_b, st_b) == (nit_r, res_r, 0)
    assert np.array_equal(phi_b, phi_r)
    phi_o = g.zeros_phi(*dims[:3])
    assert oracle.cg(s, phi_o, 100000, TOL, plan=plan) == (res_r, nit_r)
    assert np.array_equal(phi_r, phi_o)


def test_resident_kernel_edge_cases_bitwise():
    """Warm start with halo values, the 7-array form, NaN, zero RHS and
    meshes with fewer cells than blocks, on one resident cluster."""
    eaf = pkg()
    g = gen()
    rng = np.random.default_rng(9)
    s = g.make_system(*g.SMOKE, seed=1, resolve=2)
    g.interior(s.aS)[3, 4, 5] *= 1.5
    assert_bitwise(s, rng.normal(0, 1e-4, size=s.aP.shape), 300, TOL, 256, 8, 8)
    for dims in [(1, 1, 1), (3, 2, 2), (5, 7, 6)]:
        t = g.make_system(*dims, nsph=2, seed=7)
        g.interior(t.Su)[...] = rng.normal(0, 1e-3, size=(dims[2], dims[1], dims[0]))
        assert_bitwise(t, g.zeros_phi(*dims), 500, TOL, 64, 4, 4)
    z = g.make_system(*g.SMOKE, seed=0)
    z.Su[...] = 0.0
    res, nit, st, _ = assert_bitwise(z, rng.normal(size=z.aP.shape), 100, TOL, 256, 16, 16)
    assert (res, nit, st) == (0.0, 0, 0)
    n = g.make_system(*g.SMOKE, seed=0)
    g.interior(n.aP)[5, 6, 7] = np.nan
    res, nit, st, _ = assert_bitwise(n, g.zeros_phi(12, 24, 16), 40, TOL, 256, 16, 16)
    assert st == eaf._lib.EAF_ENONFINITE and np.isnan(res) and nit == 40


def test_mesh_too_large_for_shared_memory_runs_global_cluster_kernel():
    """35x70x50 (122,500 cells) on one 16-block cluster does not fit the
    cluster's shared memory: the global-memory cluster kernel runs it."""
    g = gen()
    s = g.make_system(35, 70, 50, 16, seed=3)
    res, nit, st, plan = assert_bitwise(s, g.zeros_phi(35, 70, 50), 300, 0.0, 512, 16, 16)
    assert plan == (16, 512, 16) and nit == 300
