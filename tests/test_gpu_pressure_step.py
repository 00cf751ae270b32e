"""One whole pressure step on the device -- assembly, CG, post-CG
corrections (src/mod_pressure_3d.f90:135-397) -- against the same three
steps of the oracle, the CG's dot products associated as the kernel's.

On a consistent furnace state (eafgen.make_pressure_state: cylindrical
metrics, periodic theta halos, bath under gas), every array the step writes
-- coefficients, Su, pp, exported and conservative fluxes, link flags, p,
the velocities of both phases -- must equal the oracle's BIT FOR BIT, and so
must the CG's residual and iteration count; the continuity residual agrees
to 1e-12 relative.
"""
import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

ALPHA_P = 0.7
UPDATED = ("p", "liq_ur", "liq_uth", "liq_uz", "gas_ur", "gas_uth", "gas_uz")


def run_gpu(f, device=False, max_iter=20000, tol=1e-8):
    eaf = pkg()
    out = f.copy()
    with eaf.CGSolver(f.nr, f.nth, f.nz) as cg:
        if device:
            import torch
            dev = out.copy()
            for k, v in list(dev.__dict__.items()):
                if isinstance(v, np.ndarray):
                    setattr(dev, k, torch.from_numpy(v).cuda())
            r = cg.pressure_step(dev, ALPHA_P, max_iter, tol, device_ptrs=True)
            for k, v in dev.__dict__.items():
                if hasattr(v, "data_ptr"):
                    setattr(out, k, v.cpu().numpy())
        else:
            r = cg.pressure_step(out, ALPHA_P, max_iter, tol)
        plan = cg.last_launch()
        t = cg.last_timing()
    return out, r, plan, t


def run_oracle(f, plan, max_iter=20000, tol=1e-8):
    import oracle
    g = gen()
    out = f.copy()
    cont = oracle.pressure_assemble(out)
    s = g.System(nr=f.nr, nth=f.nth, nz=f.nz, **{n: getattr(out, n) for n in g.COEF_NAMES})
    cres, nit = oracle.cg(s, out.pp, max_iter, tol, plan=plan)
    oracle.pressure_correct(g.pcorr_view(out, ALPHA_P))
    return out, cont, cres, nit


def assert_step_equal(a, b):
    for name, arr in a.outputs().items():
        assert np.array_equal(arr, b.outputs()[name]), name
    for name in UPDATED:
        assert np.array_equal(getattr(a, name), getattr(b, name)), name


@pytest.mark.parametrize("dims", [(6, 1, 5), (9, 14, 7), (12, 24, 16), (20, 30, 18)])
@pytest.mark.parametrize("flags", [7, 1, 3])
def test_step_bitwise(dims, flags):
    f = gen().make_pressure_state(*dims, seed=2, flags=flags)
    a, (res, cres, nit, st), plan, t = run_gpu(f)
    b, cont, cres_o, nit_o = run_oracle(f, plan)
    assert st == 0 and cres < 1e-8
    assert (cres, nit) == (cres_o, nit_o)
    assert abs(res - cont) <= 1e-12 * abs(cont)
    assert_step_equal(a, b)
    assert t["kernels"] >= 8


def test_step_bitwise_production_mesh():
    f = gen().make_pressure_state(60, 120, 84, seed=0, flags=7)
    a, (res, cres, nit, st), plan, _ = run_gpu(f)
    b, cont, cres_o, nit_o = run_oracle(f, plan)
    assert st == 0 and (cres, nit) == (cres_o, nit_o)
    assert abs(res - cont) <= 1e-12 * abs(cont)
    assert_step_equal(a, b)


def test_step_device_pointers_match_host_path():
    f = gen().make_pressure_state(11, 16, 9, seed=4, flags=7)
    a, ra, _, _ = run_gpu(f)
    b, rb, _, _ = run_gpu(f, device=True)
    assert ra == rb
    assert_step_equal(a, b)


def test_step_iteration_cap_still_corrects():
    """The reference corrects with whatever the CG returned (no convergence
    check between :316 and :333): a capped CG still yields the oracle's
    corrected fields."""
    f = gen().make_pressure_state(12, 24, 16, seed=5, flags=7)
    a, (res, cres, nit, st), plan, _ = run_gpu(f, max_iter=7)
    b, cont, cres_o, nit_o = run_oracle(f, plan, max_iter=7)
    assert nit == nit_o == 7 and cres == cres_o and cres > 1e-8
    assert_step_equal(a, b)


@pytest.mark.parametrize("flags", [0, 5])
def test_step_bitwise_remaining_switches(flags):
    """No liquid room and no gas (0); compressibility with the gas outside the
    equation (5: gas alpha, rho and T_old read, no gas face or correction)."""
    f = gen().make_pressure_state(12, 24, 16, seed=6, flags=flags)
    a, (res, cres, nit, st), plan, _ = run_gpu(f)
    b, cont, cres_o, nit_o = run_oracle(f, plan)
    assert st == 0 and (cres, nit) == (cres_o, nit_o)
    assert abs(res - cont) <= 1e-12 * abs(cont)
    assert_step_equal(a, b)


def test_step_with_no_cg_iterations_still_corrects():
    """max_iter 0: the CG leaves pp at the assembly's zeros, and the
    corrections run on it as the reference's would."""
    f = gen().make_pressure_state(9, 14, 7, seed=8, flags=7)
    a, (res, cres, nit, st), plan, _ = run_gpu(f, max_iter=0)
    b, cont, cres_o, nit_o = run_oracle(f, plan, max_iter=0)
    assert nit == nit_o == 0 and cres == cres_o
    assert not a.pp.any()
    assert_step_equal(a, b)


def test_step_argument_errors():
    eaf = pkg()
    f = gen().make_pressure_state(6, 8, 5, seed=1, flags=7)
    with eaf.CGSolver(6, 8, 5) as cg:
        bad = f.copy()
        bad.gas_uz = None
        with pytest.raises(eaf.EafError):
            cg.pressure_step(bad, ALPHA_P, 100, 1e-8)
        bad = f.copy()
        bad.scalars[0] = -1.0
        with pytest.raises(eaf.EafError):
            cg.pressure_step(bad, ALPHA_P, 100, 1e-8)
        # the handle stays usable after refused calls
        r = cg.pressure_step(f.copy(), ALPHA_P, 20000, 1e-8)
        assert r[3] == 0
