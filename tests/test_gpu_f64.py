"""Parity of the plain FP64 CUDA CG (through the C ABI) with the oracle.

Two oracle forms are used:

* the *kernel-order* oracle (``plan=(G, B)``): the reference algorithm with
  its dot products associated exactly as a G-block x B-thread launch of the
  CUDA kernel associates them. Every other operation is the reference's, in
  the reference's order and rounding, so the CUDA solve must agree BIT FOR BIT:
  same iteration count, same residual, same phi (interior and theta halos);
* the *sequential* oracle: the reference's own association. Two correct FP64
  CGs that differ only in how their dots are associated drift apart on these
  ill-conditioned systems (density contrast 26,000:1): the oracle run serial
  vs 4-thread on the 12x24x16 system already differs by 1 iteration and
  3e-9 in relative L2 of the solution, 25 iterations at 35x70x50. Against it
  the test therefore asserts the spread such implementations show:
  both residuals below tol, iteration counts within 5 % (at least 2; the
  serial and 8-thread oracles differ by 2.5 % at 60x120x84) and
  solution relative-L2 difference <= 2e-8. The reference's own operating
  regime (50 iterations per call, src/mod_config_3d.f90:41) and the
  production mesh to tol are held to tighter bars against the serial oracle
  in tests/test_gpu_parity_serial.py.
"""
import ctypes

import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

TOL = 1e-8
SEQ_ITER_FRAC = 0.05
SEQ_SOL_RTOL = 2e-8


def rel_l2(a, b):
    g = gen()
    ia, ib = g.interior(a), g.interior(b)
    return float(np.linalg.norm(ia - ib) / max(np.linalg.norm(ib), 1e-300))


def gpu_solve(s, phi, max_iter=200000, tol=TOL, launch=None):
    """Solve through the C ABI; returns the oracle plan (grid, block) the
    solve ran with. launch=(block, grid) sets the launch shape (0 = auto)."""
    eaf = pkg()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        if launch is not None:
            cg.set_launch(*launch)
        res, nit, st = cg.solve(s.arrays(), phi, max_iter, tol)
        timing = cg.last_timing()
        plan = cg.last_launch()
    return res, nit, st, plan, timing


def assert_bitwise(s, phi0, max_iter=200000, tol=TOL, launch=None):
    import oracle
    phi_g = phi0.copy()
    res_g, nit_g, st, plan, timing = gpu_solve(s, phi_g, max_iter, tol, launch)
    phi_o = phi0.copy()
    res_o, nit_o = oracle.cg(s, phi_o, max_iter, tol, plan=plan)
    assert nit_g == nit_o, (nit_g, nit_o, plan)
    assert (res_g == res_o) or (np.isnan(res_g) and np.isnan(res_o)), (res_g, res_o)
    assert np.array_equal(phi_g, phi_o, equal_nan=True), (
        "max |diff| %g" % np.nanmax(np.abs(phi_g - phi_o)))
    return res_g, nit_g, st, plan, timing


@pytest.mark.parametrize("launch", [None, (256, 4), (512, 9), (128, 37), (1024, 2)])
def test_smoke_mesh_bitwise_kernel_order(launch):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    res, nit, st, plan, timing = assert_bitwise(s, g.zeros_phi(12, 24, 16),
                                                launch=launch)
    assert st == 0 and res < TOL and timing["symmetric"] == 1


def test_smoke_mesh_vs_sequential_oracle():
    import oracle
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    phi_g = g.zeros_phi(12, 24, 16)
    res_g, nit_g, st, _, _ = gpu_solve(s, phi_g)
    phi_o = g.zeros_phi(12, 24, 16)
    res_o, nit_o = oracle.cg(s, phi_o, 200000, TOL)
    assert res_g < TOL and res_o < TOL
    assert abs(nit_g - nit_o) <= max(2, SEQ_ITER_FRAC * nit_o), (nit_g, nit_o)
    assert rel_l2(phi_g, phi_o) <= SEQ_SOL_RTOL


@pytest.mark.parametrize("dims", [(18, 36, 24, 8), (35, 70, 50, 16)])
def test_mid_meshes_bitwise_kernel_order(dims):
    g = gen()
    s = g.make_system(*dims, seed=3)
    res, nit, st, plan, _ = assert_bitwise(s, g.zeros_phi(*dims[:3]))
    assert st == 0 and res < TOL


@pytest.mark.parametrize("launch", [None, (1024, 148)])
def test_production_mesh_fixed_iterations_bitwise(launch):
    """60x120x84, 150 iterations with tol 0: kernel-order bitwise."""
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=0)
    res, nit, st, plan, _ = assert_bitwise(s, g.zeros_phi(60, 120, 84),
                                           max_iter=150, tol=0.0, launch=launch)
    assert nit == 150 and plan[0] > 1


@pytest.mark.parametrize("launch", [(1024, 148), (512, 148)])
def test_mesh_beyond_l2_fixed_iterations_bitwise(launch):
    """100x100x80 (800,000 cells, working set beyond L2): at 1024 threads the
    L2-prefetching kernel variant runs; bitwise against the oracle either way."""
    g = gen()
    s = g.make_system(100, 100, 80, 16, seed=2)
    res, nit, st, plan, _ = assert_bitwise(s, g.zeros_phi(100, 100, 80),
                                           max_iter=40, tol=0.0, launch=launch)
    assert nit == 40 and plan == (148, launch[0])


def test_warm_start_with_halo_values_bitwise():
    """Nonzero initial phi, including its r/z halo cells (read by the first
    matvec, multiplied by zero wall links here) and stale theta halos."""
    g = gen()
    s = g.make_system(*g.SMOKE, seed=1, resolve=2)
    rng = np.random.default_rng(5)
    phi0 = rng.normal(0, 1e-4, size=s.aP.shape)
    assert_bitwise(s, phi0)


def test_general_form_asymmetric_operator_bitwise():
    """A link that disagrees with its partner forces the 7-array form."""
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    g.interior(s.aS)[3, 4, 5] *= 1.5
    g.interior(s.aW)[2, 2, 2] *= 0.5
    res, nit, st, plan, timing = assert_bitwise(s, g.zeros_phi(12, 24, 16),
                                                max_iter=300)
    assert timing["symmetric"] == 0


def test_general_form_nonzero_wall_link_reads_phi_halo():
    """A nonzero wall link multiplies phi's r-halo cell in the first matvec."""
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    g.interior(s.aW)[1, 1, 0] = 1e-3       # i = 1 wall link
    phi0 = g.zeros_phi(12, 24, 16)
    phi0[3, 3, 1] = 0.25                   # r-halo cell (i = 0) next to it
    res, nit, st, plan, timing = assert_bitwise(s, phi0, max_iter=200)
    assert timing["symmetric"] == 0


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 3), (3, 2, 2), (1, 5, 4),
                                  (4, 3, 1), (5, 7, 6)])
@pytest.mark.parametrize("launch", [None, (64, 3)])
def test_tiny_meshes_bitwise(dims, launch):
    g = gen()
    nr, nth, nz = dims
    s = g.make_system(nr, nth, nz, nsph=2, seed=7)
    rng = np.random.default_rng(1)
    g.interior(s.Su)[...] = rng.normal(0, 1e-3, size=(nz, nth, nr))
    assert_bitwise(s, g.zeros_phi(nr, nth, nz), max_iter=500, launch=launch)


def test_zero_rhs_early_return():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    s.Su[...] = 0.0
    rng = np.random.default_rng(2)
    phi0 = rng.normal(size=s.aP.shape)
    res, nit, st, _, _ = assert_bitwise(s, phi0)
    assert res == 0.0 and nit == 0 and st == 0
    # interior untouched, theta halos refreshed from it
    assert np.array_equal(g.interior(phi0), g.interior(gpu_copy(s, phi0)))


def gpu_copy(s, phi0):
    phi = phi0.copy()
    gpu_solve(s, phi)
    return phi


def test_max_iter_zero_and_negative():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    for mi in (0, -3):
        res, nit, st, _, _ = assert_bitwise(s, g.zeros_phi(12, 24, 16), max_iter=mi)
        assert nit == 0 and res > 0


def test_nan_coefficient_propagates():
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    g.interior(s.aP)[5, 6, 7] = np.nan
    res, nit, st, _, _ = assert_bitwise(s, g.zeros_phi(12, 24, 16), max_iter=40)
    assert st == eaf._lib.EAF_ENONFINITE and np.isnan(res) and nit == 40


def test_theta_halo_postcondition():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    phi = g.zeros_phi(12, 24, 16)
    phi[:, :, 0] = 7.0        # r-halo cells: untouched but copied around theta
    gpu_solve(s, phi)
    nth = 24
    # Fortran j = 0, -1, nth+1, nth+2 are numpy columns 1, 0, nth+2, nth+3
    assert np.array_equal(phi[:, 1, :], phi[:, nth + 1, :])
    assert np.array_equal(phi[:, 0, :], phi[:, nth, :])
    assert np.array_equal(phi[:, nth + 2, :], phi[:, 2, :])
    assert np.array_equal(phi[:, nth + 3, :], phi[:, 3, :])
    assert np.all(phi[2:-2, 2:-2, 0] == 7.0)


def test_deterministic_repeat():
    g = gen()
    s = g.make_system(35, 70, 50, 16, seed=4)
    a = g.zeros_phi(35, 70, 50)
    b = g.zeros_phi(35, 70, 50)
    ra = gpu_solve(s, a)
    rb = gpu_solve(s, b)
    assert ra[:2] == rb[:2] and np.array_equal(a, b)


def test_device_pointer_path_matches_host_path():
    torch = pytest.importorskip("torch")
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.SMOKE, seed=2)
    phi_h = g.zeros_phi(12, 24, 16)
    with eaf.CGSolver(12, 24, 16) as cg:
        rh = cg.solve(s.arrays(), phi_h, 100000, TOL)
        dev = [torch.from_numpy(a).cuda() for a in s.arrays()]
        phi_d = torch.zeros(phi_h.shape, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rd = cg.solve(dev, phi_d, 100000, TOL, device_ptrs=True)
    assert rh[:2] == rd[:2]
    assert np.array_equal(phi_h, phi_d.cpu().numpy())


def test_errors_are_status_codes():
    eaf = pkg()
    lib = eaf.load()
    h = ctypes.c_void_p()
    assert lib.eaf_cg_create_mesh(ctypes.byref(h), 4, 4, 4, 1, 0) == eaf._lib.EAF_EUNSUPPORTED
    assert lib.eaf_cg_create(ctypes.byref(h), 0, 4, 4, 0) == eaf._lib.EAF_EINVAL
    assert lib.eaf_cg_create(ctypes.byref(h), 4, 4, 4, 0) == 0
    res = ctypes.c_double()
    nit = ctypes.c_int()
    null = [None] * 9
    assert lib.eaf_cg_solve_f64(h, *null, 10, 1e-8, ctypes.byref(res),
                                ctypes.byref(nit)) == eaf._lib.EAF_EINVAL
    assert lib.eaf_cg_set_launch(h, 100, 0) == eaf._lib.EAF_EINVAL
    assert lib.eaf_cg_destroy(h) == 0
    assert lib.eaf_cg_destroy(None) == eaf._lib.EAF_EINVAL


def test_barrier_timeout_reports_and_context_survives():
    eaf = pkg()
    assert eaf.barrier_timeout_selftest(0, 20.0) == eaf._lib.EAF_ETIMEOUT
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    res, nit, st, _, _ = gpu_solve(s, g.zeros_phi(12, 24, 16))
    assert st == 0 and res < TOL
