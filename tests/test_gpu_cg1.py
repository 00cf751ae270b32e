"""The single-reduction (Chronopoulos-Gear) form of the FP64 CG
(eaf_cg_set_form(h, EAF_CG_FORM_ONE_REDUCTION)) through the C ABI.

* Against its own restatement in the kernels' association
  (oracle.cg1(plan=(G, B))): BIT FOR BIT -- iterations, residual, phi
  (interior and theta halos), on the meshes, launch shapes, warm starts,
  general (7-array) operators and edge cases of the reference-form tests.
* Against the reference's PCG (the sequential oracle): the rearranged
  recurrences round differently, so the bar is the one two correct FP64 CGs
  meet on these ill-conditioned systems -- both residuals below tol,
  iteration counts within 6 % (measured on CPU in the kernels' association:
  -2 % to +5 % from 12x24x16 to 60x120x84), solution relative-L2 <= 2e-8.
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

TOL = 1e-8
SEQ_ITER_FRAC = 0.06
SEQ_SOL_RTOL = 2e-8


def rel_l2(a, b):
    g = gen()
    ia, ib = g.interior(a), g.interior(b)
    return float(np.linalg.norm(ia - ib) / max(np.linalg.norm(ib), 1e-300))


def gpu_solve(s, phi, max_iter=200000, tol=TOL, launch=None):
    eaf = pkg()
    with eaf.CGSolver(s.nr, s.nth, s.nz) as cg:
        cg.set_form(cg.FORM_ONE_REDUCTION)
        assert cg.form() == cg.FORM_ONE_REDUCTION
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
    res_o, nit_o = oracle.cg1(s, phi_o, max_iter, tol, plan=plan)
    assert nit_g == nit_o, (nit_g, nit_o, plan)
    assert (res_g == res_o) or (np.isnan(res_g) and np.isnan(res_o)), (res_g, res_o)
    assert np.array_equal(phi_g, phi_o, equal_nan=True), (
        "max |diff| %g" % np.nanmax(np.abs(phi_g - phi_o)))
    return res_g, nit_g, st, plan, timing


@pytest.mark.parametrize("launch", [None, (256, 4), (512, 9), (128, 37), (1024, 2)])
def test_smoke_mesh_bitwise_kernel_order(launch):
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    res, nit, st, plan, timing = assert_bitwise(s, g.zeros_phi(12, 24, 16), launch=launch)
    assert st == 0 and res < TOL and timing["symmetric"] == 1


@pytest.mark.parametrize("dims", [(18, 36, 24, 8), (35, 70, 50, 16)])
def test_mid_meshes_bitwise_kernel_order(dims):
    g = gen()
    s = g.make_system(*dims, seed=3)
    res, nit, st, plan, _ = assert_bitwise(s, g.zeros_phi(*dims[:3]))
    assert st == 0 and res < TOL


@pytest.mark.parametrize("launch", [None, (1024, 148), (256, 148)])
def test_production_mesh_fixed_iterations_bitwise(launch):
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=0)
    res, nit, st, plan, _ = assert_bitwise(s, g.zeros_phi(60, 120, 84), max_iter=150,
                                           tol=0.0, launch=launch)
    assert nit == 150 and plan[0] > 1


@pytest.mark.parametrize("dims", [(12, 24, 16, 8), (35, 70, 50, 16)])
def test_vs_reference_pcg_sequential_oracle(dims):
    import oracle
    g = gen()
    s = g.make_system(*dims, seed=0)
    phi_g = g.zeros_phi(*dims[:3])
    res_g, nit_g, st, _, _ = gpu_solve(s, phi_g)
    phi_o = g.zeros_phi(*dims[:3])
    res_o, nit_o = oracle.cg(s, phi_o, 200000, TOL)
    assert st == 0 and res_g < TOL and res_o < TOL
    assert abs(nit_g - nit_o) <= max(2, SEQ_ITER_FRAC * nit_o), (nit_g, nit_o)
    assert rel_l2(phi_g, phi_o) <= SEQ_SOL_RTOL


def test_production_mesh_to_tol_vs_reference_pcg():
    import oracle
    g = gen()
    s = g.make_system(*g.PRODUCTION, seed=0)
    phi_g = g.zeros_phi(60, 120, 84)
    res_g, nit_g, st, _, _ = gpu_solve(s, phi_g)
    phi_o = g.zeros_phi(60, 120, 84)
    res_o, nit_o = oracle.cg(s, phi_o, 200000, TOL, nthreads=max(1, oracle.max_threads()))
    assert st == 0 and res_g < TOL and res_o < TOL
    assert abs(nit_g - nit_o) <= max(2, SEQ_ITER_FRAC * nit_o), (nit_g, nit_o)
    assert rel_l2(phi_g, phi_o) <= SEQ_SOL_RTOL


def test_warm_start_with_halo_values_bitwise():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=1, resolve=2)
    rng = np.random.default_rng(5)
    assert_bitwise(s, rng.normal(0, 1e-4, size=s.aP.shape))


def test_general_form_bitwise():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    g.interior(s.aS)[3, 4, 5] *= 1.5
    g.interior(s.aW)[2, 2, 2] *= 0.5
    res, nit, st, plan, timing = assert_bitwise(s, g.zeros_phi(12, 24, 16), max_iter=300)
    assert timing["symmetric"] == 0


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 3), (3, 2, 2), (4, 3, 1), (5, 7, 6)])
def test_tiny_meshes_bitwise(dims):
    g = gen()
    nr, nth, nz = dims
    s = g.make_system(nr, nth, nz, nsph=2, seed=7)
    rng = np.random.default_rng(1)
    g.interior(s.Su)[...] = rng.normal(0, 1e-3, size=(nz, nth, nr))
    assert_bitwise(s, g.zeros_phi(nr, nth, nz), max_iter=500)


def test_zero_rhs_and_max_iter_edges():
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    s0 = g.make_system(*g.SMOKE, seed=0)
    s0.Su[...] = 0.0
    res, nit, st, _, _ = assert_bitwise(s0, np.random.default_rng(2).normal(size=s.aP.shape))
    assert res == 0.0 and nit == 0 and st == 0
    for mi in (0, -3, 1, 2):
        res, nit, st, _, _ = assert_bitwise(s, g.zeros_phi(12, 24, 16), max_iter=mi)
        assert nit == max(mi, 0)


def test_nan_coefficient_propagates():
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    g.interior(s.aP)[5, 6, 7] = np.nan
    res, nit, st, _, _ = assert_bitwise(s, g.zeros_phi(12, 24, 16), max_iter=40)
    assert st == eaf._lib.EAF_ENONFINITE and np.isnan(res) and nit == 40


def test_form_is_per_handle_and_reference_form_unchanged():
    """Switching forms on one handle; the reference form still matches its
    own oracle bit for bit after the other form ran."""
    import oracle
    eaf = pkg()
    g = gen()
    s = g.make_system(*g.SMOKE, seed=0)
    with eaf.CGSolver(12, 24, 16) as cg:
        assert cg.form() == cg.FORM_REFERENCE
        a = g.zeros_phi(12, 24, 16)
        cg.set_form(cg.FORM_ONE_REDUCTION)
        cg.solve(s.arrays(), a, 100000, TOL)
        cg.set_form(cg.FORM_REFERENCE)
        b = g.zeros_phi(12, 24, 16)
        rb, nb, _ = cg.solve(s.arrays(), b, 100000, TOL)
        plan = cg.last_launch()
        with pytest.raises(eaf.EafError):
            cg.set_form(7)
    o = g.zeros_phi(12, 24, 16)
    ro, no = oracle.cg(s, o, 100000, TOL, plan=plan)
    assert (rb, nb) == (ro, no) and np.array_equal(b, o)


def test_pressure_step_in_one_reduction_form():
    """The whole pressure step with the single-reduction CG: bit for bit the
    oracle's assembly, single-reduction CG (kernels' association) and
    corrections."""
    import oracle
    eaf = pkg()
    g = gen()
    f = g.make_pressure_state(20, 30, 18, seed=2, flags=7)
    a = f.copy()
    with eaf.CGSolver(20, 30, 18) as cg:
        cg.set_form(cg.FORM_ONE_REDUCTION)
        res, cres, nit, st = cg.pressure_step(a, 0.7, 20000, TOL)
        plan = cg.last_launch()
    b = f.copy()
    oracle.pressure_assemble(b)
    sysb = g.System(nr=20, nth=30, nz=18, **{n: getattr(b, n) for n in g.COEF_NAMES})
    cres_o, nit_o = oracle.cg1(sysb, b.pp, 20000, TOL, plan=plan)
    oracle.pressure_correct(g.pcorr_view(b, 0.7))
    assert st == 0 and (cres, nit) == (cres_o, nit_o)
    for name, arr in a.outputs().items():
        assert np.array_equal(arr, b.outputs()[name]), name
    for name in ("p", "liq_ur", "liq_uth", "liq_uz", "gas_ur", "gas_uth", "gas_uz"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
