"""Pins the oracle's pressure-equation assembly (src/mod_pressure_3d.f90:
135-310 with cell_gradients, add_phase_contribution, the helpers of
:405-458 and :654-681, pgrad src/mod_constants.f90:274-287, and
apply_pressure_bc src/mod_boundary_3d.f90:180-277; serial branch) on the CPU.

No golden vectors exist, so the C restatement is compared with a second,
pure-Python restatement (scalar IEEE doubles, the reference's statement and
operand order): every coefficient, source, exported face term and link flag
bit for bit; the continuity residual, whose flux_ref is a plain sequential
sum in both, bit for bit too. Tiny meshes, one-cell-thick ones, every
combination of the liquid-room, gas-in-equation and compressibility switches.
"""
import math

import numpy as np
import pytest

from conftest import gen

SMALL = 1e-30
GRAV = 9.81


def ix(i, j, k):
    return (k + 1, j + 1, i + 1)


def wrap(a, nr, nth, nz):
    for jd, js in ((0, nth), (-1, nth - 1), (nth + 1, 1), (nth + 2, 2)):
        for k in range(-1, nz + 3):
            for i in range(-1, nr + 3):
                a[ix(i, jd, k)] = a[ix(i, js, k)]


def py_assemble(f):
    nr, nth, nz = f.nr, f.nth, f.nz
    dt, rho_gas, Tamb, beta = f.scalars
    room_valid, gas_in, gas_comp = f.flags & 1, f.flags & 2, f.flags & 4
    R = lambda i: float(f.r[i + 1])
    TH = lambda j: float(f.theta[j + 1])
    Z = lambda k: float(f.z[k + 1])
    V = lambda a, c: float(a[ix(*c)])
    ct, al_act, ag_act = f.cell_type, f.act_l, f.act_g
    for n in ("aW", "aE", "aS", "aN", "aB", "aT", "aP", "Su", "pp", "Fs_r", "Fs_th", "Fs_z",
              "ac_r", "ac_th", "ac_z", "Fc_r", "Fc_th", "Fc_z"):
        getattr(f, n)[...] = 0.0
    for n in ("lk_r", "lk_th", "lk_z"):
        getattr(f, n)[...] = 0
    cells = [(i, j, k) for k in range(1, nz + 1) for j in range(1, nth + 1)
             for i in range(1, nr + 1)]

    def pv(c):
        return ct[ix(*c)] != 0 and (al_act[ix(*c)] or ag_act[ix(*c)])

    def pgrad(pm, p0, pp_, xm, x0, xp, okm, okp):
        if okm and okp:
            return (pp_ - pm) / (xp - xm)
        if okp:
            return (pp_ - p0) / (xp - x0)
        if okm:
            return (p0 - pm) / (x0 - xm)
        return 0.0

    def lw(ca, cb):
        def term(c):
            m = 1.0 if al_act[ix(*c)] else 0.0
            return m * V(f.liq_alpha, c) * V(f.liq_rho, c) * (1.0 - beta * (V(f.liq_T, c) - Tamb))
        return 0.5 * GRAV * (term(ca) + term(cb))

    def gradients(isg):
        shp = f.p.shape
        gr, gth, gz = np.zeros(shp), np.zeros(shp), np.zeros(shp)
        P = lambda c: V(f.p, c)
        for (i, j, k) in cells:
            if ct[ix(i, j, k)] == 0:
                continue
            c = (i, j, k)
            gr[ix(*c)] = pgrad(P((i - 1, j, k)), P(c), P((i + 1, j, k)), R(i - 1), R(i), R(i + 1),
                               i > 1 and pv((i - 1, j, k)), i < nr and pv((i + 1, j, k)))
            gth[ix(*c)] = pgrad(P((i, j - 1, k)), P(c), P((i, j + 1, k)), R(i) * TH(j - 1),
                                R(i) * TH(j), R(i) * TH(j + 1), pv((i, j - 1, k)), pv((i, j + 1, k)))
            okm = k > 1 and pv((i, j, k - 1))
            okp = k < nz and pv((i, j, k + 1))
            gz[ix(*c)] = pgrad(P((i, j, k - 1)), P(c), P((i, j, k + 1)), Z(k - 1), Z(k), Z(k + 1),
                               okm, okp)
            if isg:
                gb = gt = 0.0
                if okm:
                    gb = (P(c) - P((i, j, k - 1))) / (Z(k) - Z(k - 1)) + lw((i, j, k - 1), c)
                if okp:
                    gt = (P((i, j, k + 1)) - P(c)) / (Z(k + 1) - Z(k)) + lw(c, (i, j, k + 1))
                if okm and okp:
                    g = 0.5 * (gb + gt)
                elif okp:
                    g = gt
                elif okm:
                    g = gb
                else:
                    g = 0.0
                gz[ix(*c)] = g
        for a in (gr, gth, gz):
            wrap(a, nr, nth, nz)
        return gr, gth, gz

    flux = [0.0]

    def face_open(isg, u, rn, rp):
        if isg or not room_valid:
            return True
        ok = True
        if u > 0.0 and rp <= 1.0e-4:
            ok = False
        if u < 0.0 and rn <= 1.0e-4:
            ok = False
        return ok

    def add_phase(ph, act, export, grads, isg):
        gr, gth, gz = grads
        g = lambda n: getattr(f, ph + "_" + n)
        aef = g("alpha")
        rm = lambda c: V(f.liq_room, c)
        P = lambda c: V(f.p, c)

        def df(ap, c, nb):
            return 0.5 * (V(aef, c) * V(f.vol, c) / max(V(ap, c), SMALL)
                          + V(aef, nb) * V(f.vol, nb) / max(V(ap, nb), SMALL))

        def link(nb):
            return ct[ix(*nb)] != 0 and act[ix(*nb)]

        for (i, j, k) in cells:
            c = (i, j, k)
            q = ix(*c)
            if ct[q] == 0 or not act[q]:
                continue
            # west, east, south, north, bottom, top
            specs = [
                ((i - 1, j, k), "aP_ur", "ur", gr, R(i) - R(i - 1), f.Ar, (i - 1, j, k), +1, "aW", None),
                ((i + 1, j, k), "aP_ur", "ur", gr, R(i + 1) - R(i), f.Ar, c, -1, "aE", "r"),
                ((i, j - 1, k), "aP_uth", "uth", gth, R(i) * (TH(j) - TH(j - 1)), f.Ath, c, +1, "aS", None),
                ((i, j + 1, k), "aP_uth", "uth", gth, R(i) * (TH(j + 1) - TH(j)), f.Ath, c, -1, "aN", "th"),
                ((i, j, k - 1), "aP_uz", "uz", gz, Z(k) - Z(k - 1), f.Az, (i, j, k - 1), +1, "aB", None),
                ((i, j, k + 1), "aP_uz", "uz", gz, Z(k + 1) - Z(k), f.Az, c, -1, "aT", "z"),
            ]
            for (nb, apn, un, gg, delta, area, ac_, sgn, coef, exp) in specs:
                if not link(nb):
                    continue
                d_f = df(g(apn), c, nb)
                af = 0.5 * (V(aef, c) + V(aef, nb))
                lo, hi = (nb, c) if sgn > 0 else (c, nb)
                u_f = 0.5 * (V(g(un), lo) + V(g(un), hi))
                corr = 0.5 * (V(gg, lo) + V(gg, hi)) - (P(hi) - P(lo)) / delta
                if un == "uz":
                    corr = corr - (lw(lo, hi) if isg else 0.0)
                u_f = u_f + d_f * corr
                if not face_open(isg, u_f, rm(lo), rm(hi)):
                    continue
                A = V(area, ac_)
                arr = getattr(f, coef)
                arr[q] = float(arr[q]) + af * d_f * A / delta
                if sgn > 0:
                    f.Su[q] = float(f.Su[q]) + af * u_f * A
                else:
                    f.Su[q] = float(f.Su[q]) - af * u_f * A
                flux[0] = flux[0] + abs(af * u_f * A)
                if export and exp:
                    getattr(f, "Fs_" + exp)[q] = af * u_f * A
                    getattr(f, "ac_" + exp)[q] = af * d_f * A / delta
                    getattr(f, "lk_" + exp)[q] = 1

    add_phase("liq", al_act, True, gradients(False), False)
    if gas_in:
        add_phase("gas", ag_act, False, gradients(True), True)
    if gas_comp:
        for c in cells:
            q = ix(*c)
            if ct[q] == 0 or not ag_act[q]:
                continue
            a, vo, rh = V(f.gas_alpha, c), V(f.vol, c), V(f.gas_rho, c)
            src = a * vo / dt * (rh - rho_gas * Tamb / max(V(f.gas_T_old, c), 100.0)) / max(rh, SMALL)
            cap = 0.2 * a * vo / dt
            f.Su[q] = float(f.Su[q]) - max(-cap, min(cap, src))
    links = ("aW", "aE", "aS", "aN", "aB", "aT")
    for c in cells:
        q = ix(*c)
        if ct[q] == 0:
            continue
        if not al_act[q] and not ag_act[q]:
            for n in links:
                getattr(f, n)[q] = 0.0
            f.aP[q] = 1.0
            f.Su[q] = 0.0
        else:
            s = 0.0
            first = True
            for n in links:
                s = float(getattr(f, n)[q]) if first else s + float(getattr(f, n)[q])
                first = False
            ap = s * (1.0 + 1.0e-6)
            if gas_comp and ag_act[q]:
                ap = ap + V(f.gas_alpha, c) / 101325.0 * V(f.vol, c) / dt
            if al_act[q]:
                ap = ap + V(f.liq_alpha, c) * V(f.vol, c) / (V(f.liq_rho, c) * (4000.0 * 4000.0) * dt)
            f.aP[q] = ap
    out = lambda c: c[2] == nz and f.outlet[ix(*c)] != 0
    for (i, j, k) in cells:
        c = (i, j, k)
        q = ix(*c)
        if ct[q] == 0:
            for n in links:
                getattr(f, n)[q] = 0.0
            f.aP[q] = 1.0
            f.Su[q] = 0.0
            continue
        if i == 1:
            f.aW[q] = 0.0
        if i == nr:
            f.aE[q] = 0.0
        if k == 1:
            f.aB[q] = 0.0
        if k == nz:
            if out(c):
                for n in links:
                    getattr(f, n)[q] = 0.0
                f.aP[q] = 1.0
                f.Su[q] = 0.0
                continue
            f.aT[q] = 0.0
        if i > 1 and ct[ix(i - 1, j, k)] == 0:
            f.aW[q] = 0.0
        if i < nr and ct[ix(i + 1, j, k)] == 0:
            f.aE[q] = 0.0
        if k > 1 and ct[ix(i, j, k - 1)] == 0:
            f.aB[q] = 0.0
        if k < nz and ct[ix(i, j, k + 1)] == 0:
            f.aT[q] = 0.0
        for nb, n in (((i - 1, j, k), "aW"), ((i + 1, j, k), "aE"), ((i, j - 1, k), "aS"),
                      ((i, j + 1, k), "aN"), ((i, j, k - 1), "aB"), ((i, j, k + 1), "aT")):
            if out(nb):
                getattr(f, n)[q] = 0.0
    sum_su = 0.0
    for c in cells:
        q = ix(*c)
        if ct[q] == 0:
            continue
        if al_act[q] or ag_act[q]:
            sum_su = sum_su + abs(float(f.Su[q]))
    return sum_su / max(flux[0], SMALL)


@pytest.mark.parametrize("dims", [(3, 4, 3), (1, 1, 1), (2, 1, 3), (4, 3, 1), (5, 6, 4)])
@pytest.mark.parametrize("flags", [0, 1, 3, 7, 6])
def test_assembly_matches_python_restatement_bitwise(orc, dims, flags):
    g = gen()
    f = g.make_assembly_fields(*dims, seed=9, flags=flags)
    a, b = f.copy(), f.copy()
    ra = orc.pressure_assemble(a)
    rb = py_assemble(b)
    for n, arr in a.outputs().items():
        assert np.array_equal(arr, b.outputs()[n]), n
    assert ra == rb


def test_assembly_structure(orc):
    """Identity rows for solid, sealed and outlet cells; wall links zero; the
    halo of every output overwritten with zeros."""
    g = gen()
    f = g.make_assembly_fields(6, 8, 5, seed=4)
    orc.pressure_assemble(f)
    I = g.interior
    ident = (I(f.cell_type) == 0) | ((I(f.act_l) == 0) & (I(f.act_g) == 0))
    ident[-1] |= (I(f.outlet)[-1] != 0) & (I(f.cell_type)[-1] != 0)
    assert (I(f.aP)[ident] == 1.0).all() and (I(f.Su)[ident] == 0.0).all()
    assert (I(f.aW)[:, :, 0] == 0).all() and (I(f.aE)[:, :, -1] == 0).all()
    assert (I(f.aB)[0] == 0).all() and (I(f.aT)[-1] == 0).all()
    halo = np.ones(f.aP.shape, dtype=bool)
    halo[2:-2, 2:-2, 2:-2] = False
    for n in ("aW", "aP", "Su", "pp", "Fs_r", "Fc_z"):
        assert (getattr(f, n)[halo] == 0.0).all()
    assert (f.lk_r[halo] == 0).all()


@pytest.mark.parametrize("dims", [(6, 1, 5), (9, 14, 7), (12, 24, 16)])
def test_consistent_state_assembles_an_spd_operator(dims):
    """eafgen.make_pressure_state: the assembled operator is symmetric (r and
    z links exactly; theta links up to the rounding of the seam's centre
    spacing), weakly diagonally dominant, and the oracle CG solves it; the
    post-CG corrections run over the same arrays (pcorr_view shares them)."""
    import oracle
    g = gen()
    nr, nth, nz = dims
    f = g.make_pressure_state(*dims, seed=1)
    oracle.pressure_assemble(f)
    I = g.interior
    aW, aE, aS, aN, aB, aT, aP, Su = [getattr(f, n) for n in g.COEF_NAMES]
    assert np.array_equal(aE[2:-2, 2:-2, 2:-3], aW[2:-2, 2:-2, 3:-2])
    assert np.array_equal(aT[2:-3, 2:-2, 2:-2], aB[3:-2, 2:-2, 2:-2])
    an, as_ = I(aN), I(aS)
    assert np.allclose(an, np.roll(as_, -1, axis=1), rtol=1e-12, atol=0)
    off = I(aW) + I(aE) + I(aS) + I(aN) + I(aB) + I(aT)
    assert (I(aP) >= off).all() and (I(aP) > 0).all()
    s = g.System(nr=nr, nth=nth, nz=nz, **{n: getattr(f, n) for n in g.COEF_NAMES})
    res, nit = oracle.cg(s, f.pp, 20000, 1e-8)
    assert res < 1e-8
    v = g.pcorr_view(f, 0.7)
    assert v.pp is f.pp and v.p is f.p and v.liq_ur is f.liq_ur and v.has_gas
    p0 = f.p.copy()
    oracle.pressure_correct(v)
    assert not np.array_equal(f.p, p0)
