"""eafcg-b200: the EAF3D pressure-correction CG on NVIDIA B200 (sm_100a).

The Python face of libeafcg.so. ``cg_3d`` mirrors the reference subroutine

    cg_3d_mpi(aW, aE, aS, aN, aB, aT, aP, Su, phi, m, max_iter, tol,
              residual, n_iter)            (src/mod_solver_3d.f90:485-496)

argument for argument: the eight coefficient/RHS arrays and ``phi`` are FP64
arrays in the reference workspace layout (Fortran (-1:nr+2,-1:nth+2,-1:nz+2),
i.e. C-order numpy shape (nz+4, nth+4, nr+4)), ``phi`` is updated in place
(interior plus theta-halo columns), and (residual, n_iter) is returned.
As in the reference, a NaN residual is returned rather than raised
(src/mod_pressure_3d.f90:322); every other failure raises EafError.

All compute runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import (EAF_EBUSY, EAF_ENONFINITE, EAF_ETIMEOUT, EAF_OK, EafError,
                   check, load)

SOR_TOL_PRESSURE = 1.0e-8     # src/mod_constants.f90:143
MAX_INNER_PRES = 50           # src/mod_config_3d.f90:41 (default cap)

__all__ = ["CGSolver", "Batch", "Server", "cg_3d", "EafError", "load", "SOR_TOL_PRESSURE",
           "MAX_INNER_PRES", "halo_shape"]


def halo_shape(nr: int, nth: int, nz: int) -> tuple:
    return (nz + 4, nth + 4, nr + 4)


def _ptr(a) -> ctypes.c_void_p:
    """Address of a numpy array (host) or of an object with data_ptr()."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous float64")
        return ctypes.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    raise TypeError(f"unsupported array type {type(a)!r}")


class CGSolver:
    """One mesh's solver handle (device mirrors and workspace on one GPU)."""

    def __init__(self, nr: int, nth: int, nz: int, device: int = 0,
                 is_parallel: bool = False):
        self._lib = load()
        self.nr, self.nth, self.nz, self.device = nr, nth, nz, device
        h = ctypes.c_void_p()
        check(self._lib.eaf_cg_create_mesh(ctypes.byref(h), nr, nth, nz,
                                           int(bool(is_parallel)), device),
              "eaf_cg_create")
        self._h = h

    @property
    def ncells(self) -> int:
        return self.nr * self.nth * self.nz

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.eaf_cg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check_shape(self, arrays) -> None:
        shp = halo_shape(self.nr, self.nth, self.nz)
        for a in arrays:
            if isinstance(a, np.ndarray) and a.shape != shp:
                raise ValueError(f"array shape {a.shape} != halo shape {shp}")

    def solve(self, arrays, phi, max_iter: int = MAX_INNER_PRES,
              tol: float = SOR_TOL_PRESSURE, device_ptrs: bool = False):
        """Plain FP64 solve. ``arrays`` = (aW, aE, aS, aN, aB, aT, aP, Su).

        Returns (residual, n_iter, status); status is EAF_OK or
        EAF_ENONFINITE, anything else raises.
        """
        arrays = list(arrays)
        self._check_shape(arrays + [phi])
        res = ctypes.c_double()
        nit = ctypes.c_int()
        fn = (self._lib.eaf_cg_solve_f64_device if device_ptrs
              else self._lib.eaf_cg_solve_f64)
        st = fn(self._h, *[_ptr(a) for a in arrays], _ptr(phi), int(max_iter),
                float(tol), ctypes.byref(res), ctypes.byref(nit))
        check(st, "eaf_cg_solve_f64", allow=(EAF_OK, EAF_ENONFINITE))
        return res.value, nit.value, st

    def tdma(self, arrays, phi, n_sweep: int, device_ptrs: bool = False) -> None:
        """Line-by-line TDMA sweeps in place on phi (tdma_3d_mpi,
        src/mod_solver_3d.f90:252-366): ``arrays`` = (aW, aE, aS, aN, aB, aT,
        aP, Su) of any (not necessarily symmetric) transport equation."""
        arrays = list(arrays)
        self._check_shape(arrays + [phi])
        fn = (self._lib.eaf_tdma_3d_f64_device if device_ptrs
              else self._lib.eaf_tdma_3d_f64)
        st = fn(self._h, *[_ptr(a) for a in arrays], _ptr(phi), int(n_sweep))
        check(st, "eaf_tdma_3d_f64")

    def residual(self, arrays, phi, device_ptrs: bool = False) -> float:
        """compute_residual_3d_mpi (src/mod_solver_3d.f90:625-694)."""
        arrays = list(arrays)
        self._check_shape(arrays + [phi])
        res = ctypes.c_double()
        fn = (self._lib.eaf_residual_3d_f64_device if device_ptrs
              else self._lib.eaf_residual_3d_f64)
        st = fn(self._h, *[_ptr(a) for a in arrays], _ptr(phi), ctypes.byref(res))
        check(st, "eaf_residual_3d_f64")
        return res.value

    def pressure_correct(self, fields, device_ptrs: bool = False) -> None:
        """Post-CG corrections of the pressure step (src/mod_pressure_3d.f90:
        333-397, correct_velocities :689-746) in place on the arrays of
        ``fields`` (an object with the attributes of eafgen.PcorrFields:
        float64 halo-layout arrays, int32 flag/mask arrays, coordinate
        arrays, ``has_gas``, ``alpha_p``)."""
        from ._lib import PcorrFieldsC, PhaseFields

        def addr(a, kind):
            if isinstance(a, np.ndarray):
                want = np.float64 if kind == "d" else np.int32
                if a.dtype != want or not a.flags.c_contiguous:
                    raise ValueError(f"array must be C-contiguous {np.dtype(want)}")
                return a.ctypes.data
            if hasattr(a, "data_ptr"):
                return a.data_ptr()
            raise TypeError(f"unsupported array type {type(a)!r}")

        c = PcorrFieldsC()
        for n in ("pp", "Fs_r", "Fs_th", "Fs_z", "ac_r", "ac_th", "ac_z", "Fc_r", "Fc_th",
                  "Fc_z", "vol", "r", "theta", "z", "p"):
            setattr(c, n, addr(getattr(fields, n), "d"))
        for n in ("lk_r", "lk_th", "lk_z", "cell_type", "act_l", "act_g"):
            setattr(c, n, addr(getattr(fields, n), "i"))
        for ph in ("liq", "gas") if fields.has_gas else ("liq",):
            pf = PhaseFields(*[addr(getattr(fields, ph + "_" + n), "d") for n in
                               ("alpha", "aP_ur", "aP_uth", "aP_uz", "ur", "uth", "uz")])
            setattr(c, ph, pf)
        c.has_gas = 1 if fields.has_gas else 0
        c.alpha_p = float(fields.alpha_p)
        fn = (self._lib.eaf_pressure_correct_f64_device if device_ptrs
              else self._lib.eaf_pressure_correct_f64)
        check(fn(self._h, ctypes.byref(c)), "eaf_pressure_correct_f64")

    def _assembly_struct(self, fields):
        """eaf_assembly_fields_t of ``fields`` (numpy arrays or device
        tensors; attributes the switches leave unread may be None)."""
        from ._lib import ASSEMBLY_IN, ASSEMBLY_OUT, AssemblyFieldsC, PhaseState

        ints = ("cell_type", "outlet", "act_l", "act_g", "lk_r", "lk_th", "lk_z")

        def addr(name, a):
            if a is None:
                return None
            if isinstance(a, np.ndarray):
                want = np.int32 if name in ints else np.float64
                if a.dtype != want or not a.flags.c_contiguous:
                    raise ValueError(f"{name} must be C-contiguous {np.dtype(want)}")
                return a.ctypes.data
            if hasattr(a, "data_ptr"):
                return a.data_ptr()
            raise TypeError(f"unsupported array type {type(a)!r}")

        c = AssemblyFieldsC()
        for n in ASSEMBLY_IN + ASSEMBLY_OUT:
            setattr(c, n, addr(n, getattr(fields, n, None)))
        for ph in ("liq", "gas"):
            setattr(c, ph, PhaseState(*[addr(n, getattr(fields, ph + "_" + n, None)) for n in
                                        ("alpha", "rho", "ur", "uth", "uz", "aP_ur",
                                         "aP_uth", "aP_uz")]))
        c.liq_T = addr("liq_T", getattr(fields, "liq_T", None))
        c.gas_T_old = addr("gas_T_old", getattr(fields, "gas_T_old", None))
        fl = int(fields.flags)
        c.liq_room_valid, c.gas_in_poisson, c.gas_compressibility = \
            fl & 1, (fl >> 1) & 1, (fl >> 2) & 1
        c.dt, c.rho_gas, c.T_ambient, c.beta_expansion = [float(x) for x in fields.scalars]
        return c

    def pressure_assemble(self, fields, device_ptrs: bool = False) -> float:
        """Assembly of the pressure-correction equation (solve_pressure_correction
        up to the CG, src/mod_pressure_3d.f90:135-310, with apply_pressure_bc,
        src/mod_boundary_3d.f90:180-277) into the output arrays of ``fields``
        (an object with the attributes of eafgen.AssemblyFields: float64
        halo-layout arrays, int32 masks, coordinate arrays, ``flags`` -- 1
        liquid room valid, 2 gas in the equation, 4 gas compressibility -- and
        ``scalars`` = (dt, rho_gas, T_ambient, beta_expansion)). Returns the
        continuity residual sum|Su| / flux_ref."""
        c = self._assembly_struct(fields)
        res = ctypes.c_double()
        fn = (self._lib.eaf_pressure_assemble_f64_device if device_ptrs
              else self._lib.eaf_pressure_assemble_f64)
        check(fn(self._h, ctypes.byref(c), ctypes.byref(res)), "eaf_pressure_assemble_f64")
        return res.value

    def pressure_step(self, fields, alpha_p: float = 0.7, max_iter: int = MAX_INNER_PRES,
                      tol: float = SOR_TOL_PRESSURE, device_ptrs: bool = False):
        """One whole pressure step (src/mod_pressure_3d.f90:135-397): the
        assembly into ``fields`` (as pressure_assemble), the CG into
        ``fields.pp``, the post-CG corrections with under-relaxation
        ``alpha_p`` -- ``fields.p`` and the velocities of the phases in the
        equation are updated in place. Returns (residual, cg_residual,
        n_iter, status): the continuity residual (the CG's when that is NaN),
        the CG's residual and iterations, EAF_OK or EAF_ENONFINITE."""
        c = self._assembly_struct(fields)
        res, cres, nit = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        fn = (self._lib.eaf_pressure_step_f64_device if device_ptrs
              else self._lib.eaf_pressure_step_f64)
        st = fn(self._h, ctypes.byref(c), float(alpha_p), int(max_iter), float(tol),
                ctypes.byref(res), ctypes.byref(cres), ctypes.byref(nit))
        check(st, "eaf_pressure_step_f64", allow=(EAF_OK, EAF_ENONFINITE))
        return res.value, cres.value, nit.value, st

    def solve_mixed(self, arrays, phi, tol: float = SOR_TOL_PRESSURE,
                    inner_tol: float = 0.1, max_outer: int = 200,
                    max_inner: int = 100000, device_ptrs: bool = False):
        """Mixed FP32/FP64 solve. Returns (residual, n_iter, n_outer, status)."""
        arrays = list(arrays)
        self._check_shape(arrays + [phi])
        res = ctypes.c_double()
        nit = ctypes.c_int()
        nout = ctypes.c_int()
        fn = (self._lib.eaf_cg_solve_mixed_device if device_ptrs
              else self._lib.eaf_cg_solve_mixed)
        st = fn(self._h, *[_ptr(a) for a in arrays], _ptr(phi), int(max_outer),
                int(max_inner), float(tol), float(inner_tol), ctypes.byref(res),
                ctypes.byref(nit), ctypes.byref(nout))
        check(st, "eaf_cg_solve_mixed", allow=(EAF_OK, EAF_ENONFINITE))
        return res.value, nit.value, nout.value, st

    def set_launch(self, block: int = 0, grid: int = 0) -> None:
        check(self._lib.eaf_cg_set_launch(self._h, block, grid), "set_launch")

    def launch(self) -> tuple:
        b, g = ctypes.c_int(), ctypes.c_int()
        check(self._lib.eaf_cg_get_launch(self._h, ctypes.byref(b), ctypes.byref(g)))
        return b.value, g.value

    def last_launch(self) -> tuple:
        """The oracle plan of the last solve's dots: (grid, block), or
        (grid, block, cluster) when it ran on a grid of thread-block
        clusters."""
        b, g, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.eaf_cg_last_launch(self._h, ctypes.byref(b), ctypes.byref(g)))
        check(self._lib.eaf_cg_last_cluster(self._h, ctypes.byref(c)))
        return (g.value, b.value) if c.value <= 1 else (g.value, b.value, c.value)

    def set_cluster(self, cluster: int = 0) -> None:
        """Blocks per thread-block cluster of the plain FP64 solve: 2..16,
        1 for none, 0 for the tuned choice of the mesh."""
        check(self._lib.eaf_cg_set_cluster(self._h, int(cluster)), "set_cluster")

    RESIDENT_OFF = 0
    RESIDENT_CLUSTER_BARRIER = 1
    RESIDENT_MBARRIER = 2

    def set_resident(self, mode: int = 1) -> None:
        """One-cluster launches of a mesh that fits keep the system in the
        cluster's shared memory, the blocks signalling their partials by a
        cluster barrier (RESIDENT_CLUSTER_BARRIER, default) or mbarrier
        arrivals (RESIDENT_MBARRIER), or run the global-memory cluster kernel
        (RESIDENT_OFF); all give the same bits."""
        check(self._lib.eaf_cg_set_resident(self._h, int(mode)), "set_resident")

    def mixed_trace(self, max_steps: int = 1000) -> list:
        """Per refinement step of the last mixed-precision solve: inner FP32
        iterations, the inner CG's residual reduction and the FP64 outer
        residual after the step."""
        buf = (ctypes.c_double * (3 * max_steps))()
        n = ctypes.c_int()
        check(self._lib.eaf_cg_mixed_trace(self._h, buf, int(max_steps), ctypes.byref(n)),
              "mixed_trace")
        return [{"inner_iterations": int(buf[3 * k]), "inner_reduction": buf[3 * k + 1],
                 "residual": buf[3 * k + 2]} for k in range(n.value)]

    KERNEL_AUTO = 0
    KERNEL_LOADS = 1
    KERNEL_STREAM = 2
    KERNEL_SLOTS = 3
    KERNEL_KEEP = 4

    def set_kernel(self, kernel: int = 0) -> None:
        """Kernel of the plain FP64 solve on a flat grid: KERNEL_LOADS
        (per-thread loads), KERNEL_STREAM (bulk-copy staging), KERNEL_SLOTS
        (per-thread loads, slot-polling all-reduce), KERNEL_KEEP (own cells'
        update operands kept in shared memory; where a block's slice does not
        fit, per-thread loads run) or KERNEL_AUTO (the tuned choice); the
        same bits either way."""
        check(self._lib.eaf_cg_set_kernel(self._h, int(kernel)), "set_kernel")

    def last_kernel(self) -> int:
        k = ctypes.c_int()
        check(self._lib.eaf_cg_last_kernel(self._h, ctypes.byref(k)), "last_kernel")
        return k.value

    def cluster(self) -> int:
        """Blocks per cluster the next plain FP64 solve runs with."""
        c = ctypes.c_int()
        check(self._lib.eaf_cg_get_cluster(self._h, ctypes.byref(c)), "get_cluster")
        return c.value

    FORM_REFERENCE = 0
    FORM_ONE_REDUCTION = 1

    def set_form(self, form: int) -> None:
        """Recurrences of the plain FP64 solve: FORM_REFERENCE (the
        reference's PCG, two all-reduces per iteration) or FORM_ONE_REDUCTION
        (Chronopoulos-Gear, one all-reduce per iteration)."""
        check(self._lib.eaf_cg_set_form(self._h, int(form)), "set_form")

    def form(self) -> int:
        f = ctypes.c_int()
        check(self._lib.eaf_cg_get_form(self._h, ctypes.byref(f)), "get_form")
        return f.value

    def set_timeout_ms(self, ms: float) -> None:
        check(self._lib.eaf_cg_set_timeout_ms(self._h, float(ms)), "set_timeout")

    def last_timing(self) -> dict:
        s, k = ctypes.c_double(), ctypes.c_double()
        sym, nk = ctypes.c_int(), ctypes.c_int()
        check(self._lib.eaf_cg_last_timing(self._h, ctypes.byref(s), ctypes.byref(k),
                                           ctypes.byref(sym), ctypes.byref(nk)))
        return {"solve_ms": s.value, "kernel_ms": k.value, "symmetric": sym.value,
                "kernels": nk.value, "e2e_ms": self._lib.eaf_cg_last_e2e_ms(self._h)}

    @property
    def stream(self) -> int:
        return self._lib.eaf_cg_stream(self._h) or 0


class Batch:
    """Many independent systems solved in one persistent launch (C ABI
    eaf_batch_*). ``dims`` is a list of (nr, nth, nz)."""

    def __init__(self, dims, device: int = 0):
        self._lib = load()
        self.dims = [tuple(int(v) for v in d) for d in dims]
        flat = (ctypes.c_int * (3 * len(self.dims)))(*[v for d in self.dims for v in d])
        h = ctypes.c_void_p()
        check(self._lib.eaf_batch_create(ctypes.byref(h), len(self.dims), flat, device),
              "eaf_batch_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.eaf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_width(self, sys: int, width: int) -> None:
        check(self._lib.eaf_batch_set_width(self._h, sys, width), "set_width")

    def lane_width(self, sys: int) -> int:
        w = ctypes.c_int()
        check(self._lib.eaf_batch_lane_width(self._h, sys, ctypes.byref(w)))
        return w.value

    def plan(self) -> tuple:
        g, b, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.eaf_batch_plan(self._h, ctypes.byref(g), ctypes.byref(b),
                                       ctypes.byref(n)), "eaf_batch_plan")
        return g.value, b.value, n.value

    def system_plan(self, sys: int) -> tuple:
        """The oracle plan of a system's FP64 dots: (lane width, 512) for a
        system on a lane, or the single-system launch (grid, block[, cluster])
        of a large system solved over the whole GPU after the batched launch."""
        g, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.eaf_batch_system_plan(self._h, int(sys), ctypes.byref(g),
                                              ctypes.byref(b), ctypes.byref(c)),
              "eaf_batch_system_plan")
        return (g.value, b.value) if c.value <= 1 else (g.value, b.value, c.value)

    def set_system(self, sys: int, arrays, phi, device_ptrs: bool = False) -> None:
        arrays = list(arrays)
        fn = (self._lib.eaf_batch_set_system_device if device_ptrs
              else self._lib.eaf_batch_set_system)
        check(fn(self._h, sys, *[_ptr(a) for a in arrays], _ptr(phi)),
              "eaf_batch_set_system")

    def solve(self, mixed: bool = False, max_iter: int = 200000,
              tol: float = SOR_TOL_PRESSURE, max_outer: int = 60,
              inner_tol: float = 0.1) -> int:
        st = self._lib.eaf_batch_solve(self._h, int(bool(mixed)), int(max_iter),
                                       float(tol), int(max_outer), float(inner_tol))
        return check(st, "eaf_batch_solve", allow=(EAF_OK, EAF_ENONFINITE))

    def result(self, sys: int) -> tuple:
        r, n, o, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.eaf_batch_result(self._h, sys, ctypes.byref(r), ctypes.byref(n),
                                         ctypes.byref(o), ctypes.byref(st)))
        return r.value, n.value, o.value, st.value

    def get_phi(self, sys: int, out: np.ndarray) -> np.ndarray:
        check(self._lib.eaf_batch_get_phi(self._h, sys, _ptr(out)), "eaf_batch_get_phi")
        return out

    @property
    def last_ms(self) -> float:
        return self._lib.eaf_batch_last_ms(self._h)


class Server:
    """The serving loop (C ABI eaf_srv_*): device-resident runs, admission
    by HBM budget, continuous batching of their pressure solves."""

    def __init__(self, device: int = 0, budget_bytes: float = 150e9,
                 mixed: bool = False, max_iter: int = 200000,
                 tol: float = SOR_TOL_PRESSURE, max_outer: int = 60,
                 inner_tol: float = 0.1, max_batch: int = 128):
        self._lib = load()
        h = ctypes.c_void_p()
        check(self._lib.eaf_srv_create(ctypes.byref(h), device, float(budget_bytes),
                                       int(bool(mixed)), int(max_iter), float(tol),
                                       int(max_outer), float(inner_tol), int(max_batch)),
              "eaf_srv_create")
        self._h = h
        # The server reads a request's inputs and writes its phi_out until the
        # ticket completes: keep those arrays alive until then.
        self._held: dict = {}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.eaf_srv_destroy(self._h)   # finishes all requests first
            self._h = None
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def open_run(self, nr: int, nth: int, nz: int) -> int:
        rid = ctypes.c_int()
        check(self._lib.eaf_srv_open_run(self._h, nr, nth, nz, ctypes.byref(rid)),
              "eaf_srv_open_run")
        return rid.value

    def try_open_run(self, nr: int, nth: int, nz: int):
        """Run id, or None when the HBM budget refuses the run."""
        rid = ctypes.c_int()
        st = self._lib.eaf_srv_open_run(self._h, nr, nth, nz, ctypes.byref(rid))
        if st == _lib.EAF_EADMIT:
            return None
        check(st, "eaf_srv_open_run")
        return rid.value

    def close_run(self, run: int) -> None:
        check(self._lib.eaf_srv_close_run(self._h, run), "eaf_srv_close_run")

    def submit(self, run: int, arrays, phi_out=None) -> int:
        arrays = list(arrays)
        t = ctypes.c_longlong()
        check(self._lib.eaf_srv_submit(self._h, run, *[_ptr(a) for a in arrays],
                                       _ptr(phi_out) if phi_out is not None else None,
                                       ctypes.byref(t)), "eaf_srv_submit")
        self._held[t.value] = (arrays, phi_out)
        return t.value

    def poll(self, ticket: int):
        """None while pending, else (residual, n_iter, n_outer, status)."""
        r, n, o, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        rc = self._lib.eaf_srv_poll(self._h, ticket, ctypes.byref(r), ctypes.byref(n),
                                    ctypes.byref(o), ctypes.byref(st))
        if rc == _lib.EAF_EBUSY:
            return None
        check(rc, "eaf_srv_poll")
        self._held.pop(ticket, None)
        return r.value, n.value, o.value, st.value

    def wait(self, ticket: int, timeout_ms: float = 60000.0):
        r, n, o, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.eaf_srv_wait(self._h, ticket, float(timeout_ms), ctypes.byref(r),
                                     ctypes.byref(n), ctypes.byref(o), ctypes.byref(st)),
              "eaf_srv_wait")
        self._held.pop(ticket, None)
        return r.value, n.value, o.value, st.value

    def stats(self) -> dict:
        st = _lib.SrvStats()
        check(self._lib.eaf_srv_stats(self._h, ctypes.byref(st)), "eaf_srv_stats")
        return {name: getattr(st, name) for name, _ in st._fields_}

    def reset_stats(self) -> None:
        check(self._lib.eaf_srv_reset_stats(self._h))

    def inject_device_lost(self) -> None:
        check(self._lib.eaf_srv_inject_fault(self._h, _lib.EAF_FAULT_DEVICE_LOST))


_solvers: dict = {}


def cg_3d(aW, aE, aS, aN, aB, aT, aP, Su, phi, max_iter: int = MAX_INNER_PRES,
          tol: float = SOR_TOL_PRESSURE, device: int = 0):
    """Mirror of cg_3d_mpi for a serial mesh; phi is updated in place.

    The mesh size is read from phi's halo shape; one cached solver handle
    per (mesh, device) keeps its device workspace across calls, as the
    reference's persistent workspace arrays do (src/mod_workspace.f90:120-144).
    Returns (residual, n_iter).
    """
    if phi.ndim != 3:
        raise ValueError("phi must be a 3-D halo-layout array")
    nz, nth, nr = (s - 4 for s in phi.shape)
    key = (nr, nth, nz, device)
    if key not in _solvers:
        _solvers[key] = CGSolver(nr, nth, nz, device)
    res, nit, _ = _solvers[key].solve((aW, aE, aS, aN, aB, aT, aP, Su), phi,
                                      max_iter, tol)
    return res, nit


def host_empty(shape, dtype=np.float64) -> np.ndarray:
    """A numpy array over pinned (page-locked) host memory from the library."""
    lib = load()
    nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
    p = ctypes.c_void_p()
    check(lib.eaf_host_alloc(ctypes.byref(p), max(nbytes, 1)), "eaf_host_alloc")
    buf = (ctypes.c_char * max(nbytes, 1)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)
    # keep the allocation alive with the array and free it with the array
    import weakref
    weakref.finalize(buf, lib.eaf_host_free, ctypes.c_void_p(p.value))
    return arr


def barrier_timeout_selftest(device: int = 0, timeout_ms: float = 20.0) -> int:
    return load().eaf_selftest_barrier_timeout(device, float(timeout_ms))


def allreduce_timeout_selftest(device: int = 0, timeout_ms: float = 20.0, mode: int = 0) -> int:
    """The release-free p.q all-reduce's bounded waits (mode 0: the arrival
    count never completes; mode 1: a partial is never written) must give
    EAF_ETIMEOUT."""
    return load().eaf_selftest_allreduce_timeout(device, float(timeout_ms), int(mode))
