"""Parity of the device assembly of the pressure-correction equation
(src/mod_pressure_3d.f90:135-310 with apply_pressure_bc,
src/mod_boundary_3d.f90:180-277) with the oracle.

Every output array -- the seven coefficients, Su, pp, the exported face
terms Fs/ac (and the zeroed Fc), the link flags -- must equal the oracle's
BIT FOR BIT over the whole halo layout. The continuity residual divides two
sums the device associates per block: it must agree within 1e-12 relative.
"""
import ctypes

import numpy as np
import pytest

from conftest import gen, pkg

pytestmark = pytest.mark.gpu

RES_RTOL = 1e-12


def run_gpu(f, device=False):
    eaf = pkg()
    out = f.copy()
    with eaf.CGSolver(f.nr, f.nth, f.nz) as cg:
        if device:
            import torch
            dev = out.copy()
            for k, v in list(dev.__dict__.items()):
                if isinstance(v, np.ndarray):
                    setattr(dev, k, torch.from_numpy(v).cuda())
            res = cg.pressure_assemble(dev, device_ptrs=True)
            for k, v in dev.__dict__.items():
                if hasattr(v, "data_ptr"):
                    setattr(out, k, v.cpu().numpy())
        else:
            res = cg.pressure_assemble(out)
        t = cg.last_timing()
    return out, res, t


def run_oracle(f):
    import oracle
    out = f.copy()
    res = oracle.pressure_assemble(out)
    return out, res


def assert_same(a, b):
    for name, arr in a.outputs().items():
        assert np.array_equal(arr, b.outputs()[name]), name


def check(f):
    a, ra, t = run_gpu(f)
    b, rb = run_oracle(f)
    assert_same(a, b)
    assert abs(ra - rb) <= RES_RTOL * abs(rb)
    return t


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 3), (4, 3, 1), (3, 2, 5), (1, 4, 2),
                                  (12, 24, 16)])
@pytest.mark.parametrize("flags", [0, 1, 3, 6, 7])
def test_assembly_bitwise_small(dims, flags):
    t = check(gen().make_assembly_fields(*dims, seed=11, flags=flags))
    assert t["kernels"] == 4


def test_assembly_all_solid_and_all_sealed():
    f = gen().make_assembly_fields(5, 6, 4, seed=2, flags=7, solid_frac=1.0)
    check(f)
    f = gen().make_assembly_fields(5, 6, 4, seed=2, flags=7)
    f.act_l[:] = 0
    f.act_g[:] = 0
    a, ra, _ = run_gpu(f)
    b, rb = run_oracle(f)
    assert_same(a, b)
    assert ra == rb == 0.0


@pytest.mark.parametrize("flags", [1, 7])
def test_assembly_bitwise_production_mesh(flags):
    check(gen().make_assembly_fields(60, 120, 84, seed=3, flags=flags))


def test_assembly_device_pointers_match_host_path():
    f = gen().make_assembly_fields(9, 14, 7, seed=5, flags=7)
    a, ra, _ = run_gpu(f)
    b, rb, _ = run_gpu(f, device=True)
    assert_same(a, b)
    assert ra == rb


def test_assembly_unused_gas_fields_may_be_absent():
    f = gen().make_assembly_fields(6, 8, 5, seed=4, flags=1)
    for n in ("gas_ur", "gas_uth", "gas_uz", "gas_aP_ur", "gas_aP_uth", "gas_aP_uz",
              "gas_alpha", "gas_rho", "gas_T_old", "liq_T"):
        setattr(f, n, None)
    a, ra, _ = run_gpu(f)
    g = gen().make_assembly_fields(6, 8, 5, seed=4, flags=1)
    b, rb = run_oracle(g)
    assert_same(a, b)
    assert abs(ra - rb) <= RES_RTOL * abs(rb)


def test_assembly_missing_fields_are_an_error():
    eaf = pkg()
    f = gen().make_assembly_fields(3, 4, 2, seed=1, flags=7)
    f.gas_ur = None
    with eaf.CGSolver(3, 4, 2) as cg:
        with pytest.raises(eaf.EafError):
            cg.pressure_assemble(f)
        f = gen().make_assembly_fields(3, 4, 2, seed=1, flags=1)
        f.scalars[0] = 0.0
        with pytest.raises(eaf.EafError):
            cg.pressure_assemble(f)
    lib = eaf._lib.load()
    h = ctypes.c_void_p()
    assert lib.eaf_cg_create(ctypes.byref(h), 3, 4, 2, 0) == 0
    try:
        res = ctypes.c_double()
        assert lib.eaf_pressure_assemble_f64(h, None, ctypes.byref(res)) == eaf._lib.EAF_EINVAL
    finally:
        lib.eaf_cg_destroy(h)
