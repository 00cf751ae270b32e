"""Seeded synthetic pressure-correction systems (the ``eafgen`` generator).

Builds the 7-point finite-volume Poisson operator that the SIMPLE pressure
correction hands to its CG, on a uniform cylindrical (r, theta, z) mesh:

* uniform dr = R/nr, dtheta = 2*pi/nth, dz = H/nz; r-centre (i - 1/2) dr;
* face areas A_r = r_face dtheta dz (zero on the axis), A_theta = dr dz,
  A_z = r dr dtheta -- the uniform-spacing form of the reference mesh metrics
  (src/mod_mesh_3d.f90:125-156);
* per-cell density: liquid steel 7000 kg/m3 where z < 0.6 m and r < 2.5 m,
  gas 0.3 kg/m3 elsewhere, plus seeded scrap spheres at 7800 kg/m3;
* per-cell momentum diagonal abar_P, log-uniform in [1e2, 1e4];
* face link a_f = rho_f A_f^2 / abar_f with harmonic-mean rho_f and abar_f;
* a_P = sum of the six links (W, E, S, N, B, T, in that order);
* no-flux walls at r = R, z = 0 and z = H (links zeroed), periodic in theta;
* cell (nr, 1, 1) pinned to p' = 0 and folded symmetrically the way
  apply_pressure_bc folds its Dirichlet outlets (src/mod_boundary_3d.f90:
  235-242, 263-270): its row becomes the identity with zero source, the links
  of its neighbours into it are zeroed, and their a_P keep the term;
* RHS b ~ N(0, 1e-3) with the mean over the free cells removed, b = 0 at the
  pin; x0 = 0.

Arrays come out in the reference workspace layout (src/mod_workspace.f90:
24-27): Fortran ``(-1:nr+2, -1:nth+2, -1:nz+2)`` column-major with r fastest,
which is a C-order numpy array of shape ``(nz+4, nth+4, nr+4)``. Halo entries
are zero, as the reference assembler leaves them.

Re-solves (the SIMPLE-like sequence) perturb abar_P by a fresh per-cell factor
U[0.9, 1.1] of the base field, draw a fresh zero-mean RHS and are meant to be
warm-started from the previous solution.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

R_FURNACE = 3.8
H_FURNACE = 4.5
RHO_STEEL = 7000.0
RHO_GAS = 0.3
RHO_SCRAP = 7800.0
BATH_DEPTH = 0.6
BATH_RADIUS = 2.5

# Named workloads (mesh nr, nth, nz and scrap-sphere count).
SMOKE = (12, 24, 16, 8)          # 4,608 cells
PRODUCTION = (60, 120, 84, 24)   # 604,800 cells
FINE = (120, 240, 168, 64)       # 4,838,400 cells
BATCH_MIX = [((12, 24, 16, 8), 40), ((18, 36, 24, 8), 30),
             ((35, 70, 50, 16), 20), ((60, 120, 84, 24), 6)]
SERVE_MIX = [((18, 36, 24, 8), 0.50), ((35, 70, 50, 16), 0.35),
             ((60, 120, 84, 24), 0.15)]

COEF_NAMES = ("aW", "aE", "aS", "aN", "aB", "aT", "aP", "Su")


def halo_shape(nr: int, nth: int, nz: int) -> tuple:
    return (nz + 4, nth + 4, nr + 4)


def interior(a: np.ndarray) -> np.ndarray:
    """View of the interior cells 1..n of a halo-layout array."""
    return a[2:-2, 2:-2, 2:-2]


@dataclasses.dataclass
class Mesh:
    nr: int
    nth: int
    nz: int
    nsph: int
    seed: int
    rho: np.ndarray      # (nz, nth, nr) cell density
    abar: np.ndarray     # (nz, nth, nr) base momentum diagonal

    @property
    def ncells(self) -> int:
        return self.nr * self.nth * self.nz


@dataclasses.dataclass
class System:
    """One pressure-correction system in the reference halo layout."""
    nr: int
    nth: int
    nz: int
    aW: np.ndarray
    aE: np.ndarray
    aS: np.ndarray
    aN: np.ndarray
    aB: np.ndarray
    aT: np.ndarray
    aP: np.ndarray
    Su: np.ndarray

    @property
    def ncells(self) -> int:
        return self.nr * self.nth * self.nz

    def arrays(self):
        return [getattr(self, n) for n in COEF_NAMES]


def _hmean(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return 2.0 * a * b / (a + b)


def make_mesh(nr: int, nth: int, nz: int, nsph: int, seed: int) -> Mesh:
    """Density and base abar_P fields; draws spheres first, then abar_P."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dr = R_FURNACE / nr
    dth = 2.0 * math.pi / nth
    dz = H_FURNACE / nz
    rc = (np.arange(nr) + 0.5) * dr
    thc = (np.arange(nth) + 0.5) * dth
    zc = (np.arange(nz) + 0.5) * dz
    Z, TH, RR = np.meshgrid(zc, thc, rc, indexing="ij")
    rho = np.where((Z < BATH_DEPTH) & (RR < BATH_RADIUS), RHO_STEEL, RHO_GAS)
    u = rng.random((nsph, 4))
    X = RR * np.cos(TH)
    Y = RR * np.sin(TH)
    for s in range(nsph):
        rs = R_FURNACE * math.sqrt(u[s, 0])
        ts = 2.0 * math.pi * u[s, 1]
        zs = H_FURNACE * u[s, 2]
        rad = 0.2 + 0.3 * u[s, 3]
        xs, ys = rs * math.cos(ts), rs * math.sin(ts)
        inside = (X - xs) ** 2 + (Y - ys) ** 2 + (Z - zs) ** 2 <= rad * rad
        rho = np.where(inside, RHO_SCRAP, rho)
    abar = np.exp(rng.uniform(math.log(1e2), math.log(1e4), size=(nz, nth, nr)))
    return Mesh(nr, nth, nz, nsph, seed, rho.astype(np.float64), abar)


def assemble(mesh: Mesh, abar: np.ndarray, b: np.ndarray) -> System:
    """Face links, diagonal, pin fold and embedding into the halo layout."""
    nr, nth, nz = mesh.nr, mesh.nth, mesh.nz
    dr = R_FURNACE / nr
    dth = 2.0 * math.pi / nth
    dz = H_FURNACE / nz
    rc = (np.arange(nr) + 0.5) * dr
    rface = (np.arange(nr) + 1.0) * dr          # outer r face of cell i
    rho = mesh.rho

    aE = np.zeros((nz, nth, nr))
    if nr > 1:
        Ar = (rface[:-1] * dth * dz)[None, None, :]
        aE[:, :, :-1] = (_hmean(rho[:, :, :-1], rho[:, :, 1:]) * Ar * Ar
                         / _hmean(abar[:, :, :-1], abar[:, :, 1:]))
    aW = np.zeros_like(aE)
    aW[:, :, 1:] = aE[:, :, :-1]

    Ath = dr * dz
    rho_n = np.roll(rho, -1, axis=1)
    abar_n = np.roll(abar, -1, axis=1)
    aN = _hmean(rho, rho_n) * Ath * Ath / _hmean(abar, abar_n)
    aS = np.roll(aN, 1, axis=1)

    aT = np.zeros_like(aE)
    if nz > 1:
        Az = (rc * dr * dth)[None, None, :]
        aT[:-1] = (_hmean(rho[:-1], rho[1:]) * Az * Az
                   / _hmean(abar[:-1], abar[1:]))
    aB = np.zeros_like(aE)
    aB[1:] = aT[:-1]

    aP = ((((aW + aE) + aS) + aN) + aB) + aT
    Su = b.copy()

    # Pin at Fortran (nr, 1, 1) = numpy [0, 0, nr-1]; fold its links.
    pk, pj, pi = 0, 0, nr - 1
    for arr in (aW, aE, aS, aN, aB, aT):
        arr[pk, pj, pi] = 0.0
    aP[pk, pj, pi] = 1.0
    Su[pk, pj, pi] = 0.0
    if nr > 1:
        aE[pk, pj, pi - 1] = 0.0
    aN[pk, (pj - 1) % nth, pi] = 0.0
    aS[pk, (pj + 1) % nth, pi] = 0.0
    if nz > 1:
        aB[pk + 1, pj, pi] = 0.0

    out = {}
    for name, arr in zip(COEF_NAMES, (aW, aE, aS, aN, aB, aT, aP, Su)):
        h = np.zeros(halo_shape(nr, nth, nz))
        interior(h)[...] = arr
        out[name] = h
    return System(nr, nth, nz, **out)


def draw_rhs(rng: np.random.Generator, nr: int, nth: int, nz: int) -> np.ndarray:
    b = rng.normal(0.0, 1e-3, size=(nz, nth, nr))
    free = np.ones_like(b, dtype=bool)
    free[0, 0, nr - 1] = False
    if free.any():
        b[free] -= b[free].mean()
    b[0, 0, nr - 1] = 0.0
    return b


def make_system(nr: int, nth: int, nz: int, nsph: int = 8, seed: int = 0,
                resolve: int | None = None, mesh: Mesh | None = None) -> System:
    """System ``resolve`` of the seeded sequence (None = the base system).

    The base system uses the base abar_P field; re-solve s multiplies it by a
    fresh per-cell U[0.9, 1.1] factor. Each has its own zero-mean RHS.
    """
    if mesh is None:
        mesh = make_mesh(nr, nth, nz, nsph, seed)
    if resolve is None:
        rng = np.random.Generator(np.random.PCG64([seed, 1]))
        abar = mesh.abar
    else:
        rng = np.random.Generator(np.random.PCG64([seed, 2, resolve]))
        abar = mesh.abar * rng.uniform(0.9, 1.1, size=mesh.abar.shape)
    b = draw_rhs(rng, nr, nth, nz)
    return assemble(mesh, abar, b)


def zeros_phi(nr: int, nth: int, nz: int) -> np.ndarray:
    return np.zeros(halo_shape(nr, nth, nz))


def make_known_answer(nr: int, nth: int, nz: int, nsph: int = 8,
                      seed: int = 0):
    """(system, x_star): the base operator with Su replaced by A x_star.

    x_star is a smooth field (zero at the pin), so the solve has a known
    answer that does not depend on any CG implementation.
    """
    sys_ = make_system(nr, nth, nz, nsph, seed)
    dth = 2.0 * math.pi / nth
    k = np.arange(nz)[:, None, None]
    j = np.arange(nth)[None, :, None]
    i = np.arange(nr)[None, None, :]
    xs = (np.cos((j + 0.5) * dth) * (1.0 + 0.1 * i)
          + 0.05 * np.sin(0.3 * k + 0.2 * i))
    xs = np.broadcast_to(xs, (nz, nth, nr)).copy()
    xs[0, 0, nr - 1] = 0.0
    x_h = zeros_phi(nr, nth, nz)
    interior(x_h)[...] = xs
    interior(sys_.Su)[...] = apply_operator(sys_, x_h)
    return sys_, x_h


def apply_operator(s: System, x_h: np.ndarray) -> np.ndarray:
    """y = A x on the interior (numpy, vectorised; theta wrapped, r/z halos
    read as stored). Same expression order as the reference matvec
    (src/mod_solver_3d.f90:595-603)."""
    x = x_h.copy()
    # theta-periodic halo fill (src/mod_mpi_topology.f90:303-311)
    x[:, 1, :] = x[:, -3, :]
    x[:, 0, :] = x[:, -4, :]
    x[:, -2, :] = x[:, 2, :]
    x[:, -1, :] = x[:, 3, :]
    c = (slice(2, -2),) * 3
    xc = x[c]
    xw = x[2:-2, 2:-2, 1:-3]
    xe = x[2:-2, 2:-2, 3:-1]
    xs = x[2:-2, 1:-3, 2:-2]
    xn = x[2:-2, 3:-1, 2:-2]
    xb = x[1:-3, 2:-2, 2:-2]
    xt = x[3:-1, 2:-2, 2:-2]
    I = interior
    return (I(s.aP) * xc - I(s.aW) * xw - I(s.aE) * xe - I(s.aS) * xs
            - I(s.aN) * xn - I(s.aB) * xb - I(s.aT) * xt)


def make_transport_system(nr: int, nth: int, nz: int, seed: int = 0,
                          trivial_frac: float = 0.05, peclet: float = 2.0,
                          sp_frac: float = 0.1) -> System:
    """A seeded transport-equation system of the kind the line-by-line TDMA
    (tdma_3d_mpi) solves for momentum, energy and species: upwind-style
    links a_E = D_e + max(-F_e, 0), a_W = D_w + max(F_w, 0) (likewise S/N,
    B/T) from per-face diffusion D ~ U[0.5, 1.5] and flux F ~ N(0, peclet/2),
    so the operator is asymmetric; walls zeroed at the axis (i = 1, W), the
    shell (i = nr, E), the floor (k = 1, B) and the roof (k = nz, T); theta
    periodic; a_P = (sum of links) * (1 + U[0, sp_frac]) (diagonally
    dominant, so the sweeps converge); Su ~ N(0, 1). A fraction
    `trivial_frac` of the cells are identity rows (a_P = 1, links 0, Su = 0),
    the form the reference's inactive cells take. Halos are zero."""
    rng = np.random.default_rng(seed)
    shp = (nz, nth, nr)

    def links(axis_len, faces_shape, periodic):
        D = rng.uniform(0.5, 1.5, size=faces_shape)
        F = rng.normal(0.0, peclet / 2.0, size=faces_shape)
        if not periodic:
            idx = [slice(None)] * 3
            ax = {"z": 0, "t": 1, "r": 2}[axis_len]
            idx[ax] = 0
            D[tuple(idx)] = 0.0
            F[tuple(idx)] = 0.0
            idx[ax] = -1
            D[tuple(idx)] = 0.0
            F[tuple(idx)] = 0.0
        return D, F

    # faces: r has nr+1 (axis .. shell), theta nth (periodic), z nz+1
    Dr, Fr = links("r", (nz, nth, nr + 1), False)
    Dt, Ft = links("t", (nz, nth, nr), True)
    Dz, Fz = links("z", (nz + 1, nth, nr), False)
    aW = Dr[:, :, :-1] + np.maximum(Fr[:, :, :-1], 0.0)
    aE = Dr[:, :, 1:] + np.maximum(-Fr[:, :, 1:], 0.0)
    # theta face j+1/2 stored at index j; the south face of j is face j-1/2
    Dt_s, Ft_s = np.roll(Dt, 1, axis=1), np.roll(Ft, 1, axis=1)
    aS = Dt_s + np.maximum(Ft_s, 0.0)
    aN = Dt + np.maximum(-Ft, 0.0)
    aB = Dz[:-1] + np.maximum(Fz[:-1], 0.0)
    aT = Dz[1:] + np.maximum(-Fz[1:], 0.0)
    aW[:, :, 0] = 0.0
    aE[:, :, -1] = 0.0
    aB[0] = 0.0
    aT[-1] = 0.0
    tot = ((((aW + aE) + aS) + aN) + aB) + aT
    aP = tot * (1.0 + rng.uniform(0.0, sp_frac, size=shp))
    Su = rng.normal(0.0, 1.0, size=shp)
    triv = rng.random(shp) < trivial_frac
    for a in (aW, aE, aS, aN, aB, aT, Su):
        a[triv] = 0.0
    aP[triv] = 1.0
    out = {}
    for name, a in zip(COEF_NAMES, (aW, aE, aS, aN, aB, aT, aP, Su)):
        h = zeros_phi(nr, nth, nz)
        interior(h)[...] = a
        out[name] = h
    return System(nr=nr, nth=nth, nz=nz, **out)


# Post-CG correction fields (solve_pressure_correction after the CG):
# double arrays in the halo layout, the coordinate arrays (index -1..n+2),
# int arrays (flags and Fortran default logicals), and per-phase fields.
PCORR_DOUBLES = ("pp", "Fs_r", "Fs_th", "Fs_z", "ac_r", "ac_th", "ac_z",
                 "Fc_r", "Fc_th", "Fc_z", "vol", "r", "theta", "z", "p")
PCORR_PHASE = ("alpha", "aP_ur", "aP_uth", "aP_uz", "ur", "uth", "uz")
PCORR_INTS = ("lk_r", "lk_th", "lk_z", "cell_type", "act_l", "act_g")
P_HYDRO_CAP = 2.0e6


class PcorrFields:
    """Every array the post-CG corrections read or write, for one mesh."""

    def __init__(self, nr, nth, nz, has_gas, alpha_p):
        self.nr, self.nth, self.nz = nr, nth, nz
        self.has_gas = has_gas
        self.alpha_p = alpha_p

    def copy(self):
        c = PcorrFields(self.nr, self.nth, self.nz, self.has_gas, self.alpha_p)
        for k, v in self.__dict__.items():
            if isinstance(v, np.ndarray):
                setattr(c, k, v.copy())
        return c

    def doubles(self):
        """The oracle's ordered double arrays (22 + 7 gas)."""
        out = [getattr(self, n) for n in PCORR_DOUBLES]
        out += [getattr(self, "liq_" + n) for n in PCORR_PHASE]
        out += [getattr(self, "gas_" + n) for n in PCORR_PHASE]
        return out

    def ints(self):
        return [getattr(self, n) for n in PCORR_INTS]

    def outputs(self):
        names = ["Fc_r", "Fc_th", "Fc_z", "p", "lk_r", "lk_th", "lk_z"]
        names += ["liq_ur", "liq_uth", "liq_uz"]
        if self.has_gas:
            names += ["gas_ur", "gas_uth", "gas_uz"]
        return {n: getattr(self, n) for n in names}


def make_pcorr_fields(nr: int, nth: int, nz: int, seed: int = 0, has_gas: bool = True,
                      solid_frac: float = 0.05, sealed_frac: float = 0.08,
                      alpha_p: float = 0.7) -> PcorrFields:
    """Seeded inputs of the post-CG corrections: pp and the assembly's
    face terms Fs/ac (random), link flags mostly 1, a few solid cells
    (cell_type 0), liquid/gas activity masks leaving `sealed_frac` of the
    cells in neither phase, positive volumes, uniform cell centres (r, theta,
    z with halo entries), phase fields with some momentum diagonals at or
    below SMALL (their correction is skipped) and p with some values beyond
    +-P_HYDRO_CAP (clamped). Halo entries are random too."""
    rng = np.random.default_rng(seed)
    shp = halo_shape(nr, nth, nz)
    f = PcorrFields(nr, nth, nz, has_gas, alpha_p)
    f.pp = rng.normal(0.0, 1e3, size=shp)
    for n in ("Fs_r", "Fs_th", "Fs_z", "Fc_r", "Fc_th", "Fc_z"):
        setattr(f, n, rng.normal(0.0, 1.0, size=shp))
    for n in ("ac_r", "ac_th", "ac_z"):
        setattr(f, n, rng.uniform(0.0, 1e-3, size=shp))
    f.vol = rng.uniform(0.5, 1.5, size=shp) * 1e-2
    f.r = (np.arange(-1, nr + 3) - 0.5) * (R_FURNACE / nr)
    f.theta = (np.arange(-1, nth + 3) - 0.5) * (2.0 * math.pi / nth)
    f.z = (np.arange(-1, nz + 3) - 0.5) * (H_FURNACE / nz)
    f.p = rng.normal(0.0, 1e6, size=shp)
    f.p[rng.random(shp) < 0.05] *= 5.0
    for ph in ("liq", "gas"):
        setattr(f, ph + "_alpha", rng.uniform(0.0, 1.0, size=shp))
        for c in ("aP_ur", "aP_uth", "aP_uz"):
            a = rng.uniform(1.0, 1e3, size=shp)
            a[rng.random(shp) < 0.05] = 1e-31
            setattr(f, ph + "_" + c, a)
        for c in ("ur", "uth", "uz"):
            setattr(f, ph + "_" + c, rng.normal(0.0, 1.0, size=shp))
    for n in ("lk_r", "lk_th", "lk_z"):
        setattr(f, n, (rng.random(shp) < 0.9).astype(np.int32))
    f.cell_type = (rng.random(shp) >= solid_frac).astype(np.int32)
    u = rng.random(shp)
    f.act_l = (u < 0.6).astype(np.int32)
    f.act_g = ((u >= 0.6) & (u < 1.0 - sealed_frac)).astype(np.int32)
    f.act_g[rng.random(shp) < 0.2] = 1
    f.act_g[u >= 1.0 - sealed_frac] = 0
    return f


# Assembly of the pressure-correction equation (solve_pressure_correction
# before the CG): ordered like the oracle's arrays.
ASM_DOUBLES_IN = ("vol", "Ar", "Ath", "Az", "r", "theta", "z", "p", "liq_room")
ASM_PHASE = ("alpha", "rho", "ur", "uth", "uz", "aP_ur", "aP_uth", "aP_uz")
ASM_DOUBLES_OUT = ("aW", "aE", "aS", "aN", "aB", "aT", "aP", "Su", "pp",
                   "Fs_r", "Fs_th", "Fs_z", "ac_r", "ac_th", "ac_z", "Fc_r", "Fc_th", "Fc_z")
ASM_INTS = ("cell_type", "outlet", "act_l", "act_g", "lk_r", "lk_th", "lk_z")


class AssemblyFields:
    """Inputs and outputs of the pressure-equation assembly for one mesh."""

    def __init__(self, nr, nth, nz, flags, scalars):
        self.nr, self.nth, self.nz = nr, nth, nz
        self.flags = flags          # 1 liq_room valid, 2 gas in eq., 4 gas compressibility
        self.scalars = scalars      # dt, rho_gas, T_ambient, beta_expansion

    def copy(self):
        c = AssemblyFields(self.nr, self.nth, self.nz, self.flags, list(self.scalars))
        for k, v in self.__dict__.items():
            if isinstance(v, np.ndarray):
                setattr(c, k, v.copy())
        return c

    def doubles(self):
        out = [getattr(self, n) for n in ASM_DOUBLES_IN]
        out += [getattr(self, "liq_" + n) for n in ASM_PHASE] + [self.liq_T]
        out += [getattr(self, "gas_" + n) for n in ASM_PHASE] + [self.gas_T_old]
        out += [getattr(self, n) for n in ASM_DOUBLES_OUT]
        return out

    def ints(self):
        return [getattr(self, n) for n in ASM_INTS]

    def outputs(self):
        names = list(ASM_DOUBLES_OUT) + ["lk_r", "lk_th", "lk_z"]
        return {n: getattr(self, n) for n in names}


def make_assembly_fields(nr: int, nth: int, nz: int, seed: int = 0, flags: int = 7,
                         solid_frac: float = 0.05, sealed_frac: float = 0.08,
                         dt: float = 1e-3) -> AssemblyFields:
    """Seeded inputs of the pressure-equation assembly: uniform cell centres
    and metric arrays, a pressure field, liquid (steel: rho ~7000, T ~1800 K)
    and gas (rho ~0.3, previous T 300-3000 K) states with volume fractions,
    velocities and momentum diagonals (some at or below SMALL), activity
    masks leaving some sealed cells, a liquid-room field with some closed
    pores (<= 1e-4), a few solid cells, electrode holes on the top layer.
    Output arrays start with random values: the assembly must overwrite them
    everywhere. Halo entries are random too."""
    rng = np.random.default_rng(seed)
    shp = halo_shape(nr, nth, nz)
    f = AssemblyFields(nr, nth, nz, flags, [dt, RHO_GAS, 300.0, 1.0e-4])
    f.vol = rng.uniform(0.5, 1.5, size=shp) * 1e-2
    for n in ("Ar", "Ath", "Az"):
        setattr(f, n, rng.uniform(0.5, 1.5, size=shp) * 1e-1)
    f.r = (np.arange(-1, nr + 3) - 0.5) * (R_FURNACE / nr)
    f.theta = (np.arange(-1, nth + 3) - 0.5) * (2.0 * math.pi / nth)
    f.z = (np.arange(-1, nz + 3) - 0.5) * (H_FURNACE / nz)
    f.p = rng.normal(0.0, 1e3, size=shp)
    f.liq_room = rng.uniform(0.0, 1.0, size=shp)
    f.liq_room[rng.random(shp) < 0.1] = 5e-5
    for ph, rho, T in (("liq", 7000.0, 1800.0), ("gas", 0.3, 1500.0)):
        setattr(f, ph + "_alpha", rng.uniform(0.0, 1.0, size=shp))
        setattr(f, ph + "_rho", rho * rng.uniform(0.8, 1.2, size=shp))
        for c in ("ur", "uth", "uz"):
            setattr(f, ph + "_" + c, rng.normal(0.0, 0.5, size=shp))
        for c in ("aP_ur", "aP_uth", "aP_uz"):
            a = rng.uniform(1.0, 1e3, size=shp)
            a[rng.random(shp) < 0.05] = 1e-31
            setattr(f, ph + "_" + c, a)
    f.liq_T = 1800.0 * rng.uniform(0.9, 1.1, size=shp)
    f.gas_T_old = rng.uniform(50.0, 3000.0, size=shp)
    f.cell_type = (rng.random(shp) >= solid_frac).astype(np.int32)
    u = rng.random(shp)
    f.act_l = (u < 0.6).astype(np.int32)
    f.act_g = ((u >= 0.35) & (u < 1.0 - sealed_frac)).astype(np.int32)
    f.outlet = np.zeros(shp, dtype=np.int32)
    f.outlet[nz + 1][rng.random(shp[1:]) < 0.1] = 1
    f.outlet[rng.random(shp) < 0.02] = 1   # ignored below the top layer
    for n in ASM_DOUBLES_OUT:
        setattr(f, n, rng.normal(size=shp))
    for n in ("lk_r", "lk_th", "lk_z"):
        setattr(f, n, rng.integers(0, 3, size=shp).astype(np.int32))
    return f


def _wrap_theta(a: np.ndarray) -> None:
    """Serial theta-periodic halo copy (src/mod_mpi_topology.f90:303-311)."""
    nth = a.shape[1] - 4
    a[:, 1] = a[:, nth + 1]
    a[:, 0] = a[:, nth]
    a[:, nth + 2] = a[:, 2]
    a[:, nth + 3] = a[:, 3]


def make_pressure_state(nr: int, nth: int, nz: int, seed: int = 0, flags: int = 7,
                        dt: float = 1e-3) -> AssemblyFields:
    """A consistent furnace state for one whole pressure step (assembly, CG,
    post-CG corrections): cylindrical metric arrays of a uniform mesh (cell
    volume r dr dtheta dz, face areas r_face dtheta dz, dr dz and r dr
    dtheta, zero at the axis), a steel bath (liquid active, alpha_l ~ 1)
    under gas, a mixed layer where both phases are active, a few solid cells
    and sealed cells, electrode holes on the top layer, momentum diagonals
    that scale with the volume, hydrostatic pressure plus noise. Cells beyond
    a physical r or z boundary are solid; theta halos are periodic copies of
    every field, as the reference keeps them. The assembled operator is then
    symmetric and diagonally dominant, so the CG converges on it. Output
    arrays start random (the assembly overwrites them)."""
    rng = np.random.default_rng(seed)
    shp = halo_shape(nr, nth, nz)
    dr, dth, dz = R_FURNACE / nr, 2.0 * math.pi / nth, H_FURNACE / nz
    f = AssemblyFields(nr, nth, nz, flags, [dt, RHO_GAS, 300.0, 1.0e-4])
    f.r = (np.arange(-1, nr + 3) - 0.5) * dr
    f.theta = (np.arange(-1, nth + 3) - 0.5) * dth
    f.z = (np.arange(-1, nz + 3) - 0.5) * dz
    rc = np.abs(f.r)[None, None, :]
    rface = np.clip(np.arange(-1, nr + 3), 0, None)[None, None, :] * dr
    ones = np.ones(shp)
    f.vol = ones * rc * dr * dth * dz
    f.Ar = ones * rface * dth * dz
    f.Ath = ones * dr * dz
    f.Az = ones * rc * dr * dth
    zc = f.z[:, None, None] * ones
    ii = np.arange(-1, nr + 3)[None, None, :] * np.ones(shp, dtype=int)
    kk = np.arange(-1, nz + 3)[:, None, None] * np.ones(shp, dtype=int)
    inside = (ii >= 1) & (ii <= nr) & (kk >= 1) & (kk <= nz)
    f.cell_type = (inside & (rng.random(shp) >= 0.02)).astype(np.int32)
    bath = 0.3 * H_FURNACE
    f.act_l = (zc < bath + 2 * dz).astype(np.int32)
    f.act_g = (zc > bath - 2 * dz).astype(np.int32)
    sealed = rng.random(shp) < 0.03
    f.act_l[sealed] = 0
    f.act_g[sealed] = 0
    f.liq_alpha = np.clip(0.5 - (zc - bath) / (4 * dz), 0.0, 1.0) * f.act_l
    f.gas_alpha = (1.0 - f.liq_alpha) * f.act_g
    f.liq_rho = 7000.0 * rng.uniform(0.98, 1.02, size=shp)
    f.gas_rho = RHO_GAS * rng.uniform(0.9, 1.1, size=shp)
    f.liq_T = 1800.0 * rng.uniform(0.98, 1.02, size=shp)
    f.gas_T_old = rng.uniform(800.0, 2500.0, size=shp)
    for ph, scale in (("liq", 1e4), ("gas", 1e1)):
        for c in ("ur", "uth", "uz"):
            setattr(f, ph + "_" + c, rng.normal(0.0, 0.05, size=shp))
        for c in ("aP_ur", "aP_uth", "aP_uz"):
            setattr(f, ph + "_" + c, f.vol * scale * rng.uniform(0.5, 2.0, size=shp) + 1e-12)
    f.p = 7000.0 * 9.81 * np.clip(bath - zc, 0.0, None) + rng.normal(0.0, 10.0, size=shp)
    f.liq_room = np.where(rng.random(shp) < 0.05, 5e-5, 1.0)
    f.outlet = np.zeros(shp, dtype=np.int32)
    f.outlet[nz + 1][rng.random(shp[1:]) < 0.03] = 1
    for n in (ASM_DOUBLES_IN[:4] + ("p", "liq_room") + tuple("liq_" + c for c in ASM_PHASE)
              + tuple("gas_" + c for c in ASM_PHASE) + ("liq_T", "gas_T_old")):
        _wrap_theta(getattr(f, n))
    for n in ("cell_type", "outlet", "act_l", "act_g"):
        _wrap_theta(getattr(f, n))
    for n in ASM_DOUBLES_OUT:
        setattr(f, n, rng.normal(size=shp))
    for n in ("lk_r", "lk_th", "lk_z"):
        setattr(f, n, rng.integers(0, 3, size=shp).astype(np.int32))
    return f


def pcorr_view(a, alpha_p: float = 0.7) -> PcorrFields:
    """The post-CG corrections' fields over the SAME arrays (numpy or device
    tensors) as an assembly's: pp, the exported Fs/ac, Fc and link flags,
    the mesh, p, the phase states and masks; the gas is in when the
    assembly's gas-in-equation switch is."""
    v = PcorrFields(a.nr, a.nth, a.nz, bool(a.flags & 2), alpha_p)
    for n in PCORR_DOUBLES + PCORR_INTS:
        setattr(v, n, getattr(a, n))
    for ph in ("liq", "gas"):
        for n in PCORR_PHASE:
            setattr(v, ph + "_" + n, getattr(a, ph + "_" + n))
    return v


def system_bytes(nr: int, nth: int, nz: int) -> int:
    """Host bytes of one system (8 halo-layout FP64 arrays)."""
    return 8 * 8 * (nr + 4) * (nth + 4) * (nz + 4)
