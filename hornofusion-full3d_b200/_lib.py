"""ctypes binding of libeafcg.so (the C ABI declared in include/eafcg.h).

Loading fails loudly when the library has not been built: there is no CPU
or PyTorch fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeafcg.so")

EAF_OK = 0
EAF_ECUDA = 1
EAF_EINVAL = 2
EAF_ENONFINITE = 3
EAF_ETIMEOUT = 4
EAF_EUNSUPPORTED = 5
EAF_ENOMEM = 6
EAF_EADMIT = 7
EAF_EBUSY = 8
EAF_ECLOSED = 9
EAF_NOALLOC_MAX_CELLS = 32768
EAF_FAULT_DEVICE_LOST = 1


class SrvStats(ctypes.Structure):
    """eaf_srv_stats_t"""
    _fields_ = [(n, ctypes.c_longlong) for n in
                ("solves", "batches", "admitted_runs", "refused_runs", "active_runs")] + \
               [(n, ctypes.c_double) for n in
                ("p50_ms", "p99_ms", "mean_ms", "max_ms", "solves_per_s",
                 "mean_batch", "used_bytes", "budget_bytes")]

class PhaseFields(ctypes.Structure):
    """eaf_phase_fields_t"""
    _fields_ = [(n, ctypes.c_void_p) for n in
                ("alpha", "aP_ur", "aP_uth", "aP_uz", "ur", "uth", "uz")]


class PcorrFieldsC(ctypes.Structure):
    """eaf_pcorr_fields_t"""
    _fields_ = ([(n, ctypes.c_void_p) for n in
                 ("pp", "Fs_r", "Fs_th", "Fs_z", "ac_r", "ac_th", "ac_z", "Fc_r",
                  "Fc_th", "Fc_z", "vol", "r", "theta", "z", "p")]
                + [("liq", PhaseFields), ("gas", PhaseFields)]
                + [(n, ctypes.c_void_p) for n in
                   ("lk_r", "lk_th", "lk_z", "cell_type", "act_l", "act_g")]
                + [("has_gas", ctypes.c_int), ("alpha_p", ctypes.c_double)])


class PhaseState(ctypes.Structure):
    """eaf_phase_state_t"""
    _fields_ = [(n, ctypes.c_void_p) for n in
                ("alpha", "rho", "ur", "uth", "uz", "aP_ur", "aP_uth", "aP_uz")]


ASSEMBLY_IN = ("cell_type", "outlet", "act_l", "act_g", "vol", "Ar", "Ath", "Az",
               "r", "theta", "z", "p", "liq_room")
ASSEMBLY_OUT = ("aW", "aE", "aS", "aN", "aB", "aT", "aP", "Su", "pp", "Fs_r", "Fs_th",
                "Fs_z", "ac_r", "ac_th", "ac_z", "Fc_r", "Fc_th", "Fc_z",
                "lk_r", "lk_th", "lk_z")


class AssemblyFieldsC(ctypes.Structure):
    """eaf_assembly_fields_t"""
    _fields_ = ([(n, ctypes.c_void_p) for n in ASSEMBLY_IN]
                + [("liq", PhaseState), ("gas", PhaseState)]
                + [("liq_T", ctypes.c_void_p), ("gas_T_old", ctypes.c_void_p)]
                + [(n, ctypes.c_int) for n in
                   ("liq_room_valid", "gas_in_poisson", "gas_compressibility")]
                + [(n, ctypes.c_double) for n in
                   ("dt", "rho_gas", "T_ambient", "beta_expansion")]
                + [(n, ctypes.c_void_p) for n in ASSEMBLY_OUT])


STATUS_NAMES = {
    0: "EAF_OK", 1: "EAF_ECUDA", 2: "EAF_EINVAL", 3: "EAF_ENONFINITE",
    4: "EAF_ETIMEOUT", 5: "EAF_EUNSUPPORTED", 6: "EAF_ENOMEM", 7: "EAF_EADMIT",
    8: "EAF_EBUSY", 9: "EAF_ECLOSED",
}

# (name, restype, argtypes) for every exported symbol of include/eafcg.h.
_ci, _cd, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
_pi, _pd = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
_sz = ctypes.c_size_t
_A8 = [_vp] * 8

SIGNATURES = [
    ("eaf_status_string", ctypes.c_char_p, [_ci]),
    ("eaf_last_error", ctypes.c_char_p, []),
    ("eaf_version", ctypes.c_char_p, []),
    ("eaf_cg_create", _ci, [ctypes.POINTER(_vp), _ci, _ci, _ci, _ci]),
    ("eaf_cg_create_mesh", _ci, [ctypes.POINTER(_vp), _ci, _ci, _ci, _ci, _ci]),
    ("eaf_cg_destroy", _ci, [_vp]),
    ("eaf_cg_solve_f64", _ci, [_vp] + _A8 + [_vp, _ci, _cd, _pd, _pi]),
    ("eaf_cg_solve_f64_device", _ci, [_vp] + _A8 + [_vp, _ci, _cd, _pd, _pi]),
    ("eaf_tdma_3d_f64", _ci, [_vp] + _A8 + [_vp, _ci]),
    ("eaf_tdma_3d_f64_device", _ci, [_vp] + _A8 + [_vp, _ci]),
    ("eaf_residual_3d_f64", _ci, [_vp] + _A8 + [_vp, _pd]),
    ("eaf_pressure_correct_f64", _ci, [_vp, _vp]),
    ("eaf_mr_grid", _ci, [_ci, _ci, _ci, _ci, _pi]),
    ("eaf_mr_block", _ci, [_ci, _ci, _ci, _pi, _pi, _pi, _pi]),
    ("eaf_mr_pack_count", ctypes.c_longlong, [_pi, _pi, _pi]),
    ("eaf_mr_unpack_count", ctypes.c_longlong, [_ci, _ci, _pi, _pi]),
    ("eaf_mr_pack", _ci, [_vp, _pi, _pi, _pi, _vp]),
    ("eaf_mr_place", _ci, [_vp, _ci, _ci, _ci, _pi, _pi, _pi, _pi, _vp]),
    ("eaf_mr_extract", _ci, [_vp, _ci, _ci, _ci, _pi, _pi, _vp]),
    ("eaf_mr_unpack", _ci, [_vp, _ci, _ci, _pi, _pi, _vp]),
    ("eaf_pressure_correct_f64_device", _ci, [_vp, _vp]),
    ("eaf_pressure_assemble_f64", _ci, [_vp, _vp, _pd]),
    ("eaf_pressure_assemble_f64_device", _ci, [_vp, _vp, _pd]),
    ("eaf_cg_set_form", _ci, [_vp, _ci]),
    ("eaf_cg_get_form", _ci, [_vp, _pi]),
    ("eaf_pressure_step_f64", _ci, [_vp, _vp, _cd, _ci, _cd, _pd, _pd, _pi]),
    ("eaf_pressure_step_f64_device", _ci, [_vp, _vp, _cd, _ci, _cd, _pd, _pd, _pi]),
    ("eaf_residual_3d_f64_device", _ci, [_vp] + _A8 + [_vp, _pd]),
    ("eaf_cg_solve_mixed", _ci,
     [_vp] + _A8 + [_vp, _ci, _ci, _cd, _cd, _pd, _pi, _pi]),
    ("eaf_cg_solve_mixed_device", _ci,
     [_vp] + _A8 + [_vp, _ci, _ci, _cd, _cd, _pd, _pi, _pi]),
    ("eaf_cg_set_launch", _ci, [_vp, _ci, _ci]),
    ("eaf_cg_get_launch", _ci, [_vp, _pi, _pi]),
    ("eaf_cg_set_timeout_ms", _ci, [_vp, _cd]),
    ("eaf_cg_last_launch", _ci, [_vp, _pi, _pi]),
    ("eaf_cg_set_cluster", _ci, [_vp, _ci]),
    ("eaf_cg_get_cluster", _ci, [_vp, _pi]),
    ("eaf_cg_last_cluster", _ci, [_vp, _pi]),
    ("eaf_cg_set_resident", _ci, [_vp, _ci]),
    ("eaf_cg_set_kernel", _ci, [_vp, _ci]),
    ("eaf_cg_mixed_trace", _ci, [_vp, _vp, _ci, _pi]),
    ("eaf_cg_last_kernel", _ci, [_vp, _pi]),
    ("eaf_cg_last_timing", _ci, [_vp, _pd, _pd, _pi, _pi]),
    ("eaf_cg_last_e2e_ms", _cd, [_vp]),
    ("eaf_cg_stream", _vp, [_vp]),
    ("eaf_host_alloc", _ci, [ctypes.POINTER(_vp), _sz]),
    ("eaf_host_free", _ci, [_vp]),
    ("eaf_host_register", _ci, [_vp, _sz]),
    ("eaf_host_unregister", _ci, [_vp]),
    ("eaf_selftest_barrier_timeout", _ci, [_ci, _cd]),
    ("eaf_selftest_allreduce_timeout", _ci, [_ci, _cd, _ci]),
    ("eaf_diag_allreduce_us", _ci, [_ci, _ci, _ci, _ci, _ci, _pd]),
    ("eaf_diag_div_check", _ci, [_ci, ctypes.c_longlong, ctypes.c_ulonglong,
                                 ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_longlong)]),
    ("eaf_batch_create", _ci, [ctypes.POINTER(_vp), _ci, _pi, _ci]),
    ("eaf_batch_destroy", _ci, [_vp]),
    ("eaf_batch_set_width", _ci, [_vp, _ci, _ci]),
    ("eaf_batch_lane_width", _ci, [_vp, _ci, _pi]),
    ("eaf_batch_plan", _ci, [_vp, _pi, _pi, _pi]),
    ("eaf_batch_system_plan", _ci, [_vp, _ci, _pi, _pi, _pi]),
    ("eaf_batch_set_system", _ci, [_vp, _ci] + [_vp] * 9),
    ("eaf_batch_set_system_device", _ci, [_vp, _ci] + [_vp] * 9),
    ("eaf_batch_solve", _ci, [_vp, _ci, _ci, _cd, _ci, _cd]),
    ("eaf_batch_result", _ci, [_vp, _ci, _pd, _pi, _pi, _pi]),
    ("eaf_batch_get_phi", _ci, [_vp, _ci, _vp]),
    ("eaf_batch_last_ms", _cd, [_vp]),
    ("eaf_batch_stream", _vp, [_vp]),
    ("eaf_srv_create", _ci, [ctypes.POINTER(_vp), _ci, _cd, _ci, _ci, _cd, _ci, _cd, _ci]),
    ("eaf_srv_destroy", _ci, [_vp]),
    ("eaf_srv_open_run", _ci, [_vp, _ci, _ci, _ci, _pi]),
    ("eaf_srv_close_run", _ci, [_vp, _ci]),
    ("eaf_srv_submit", _ci, [_vp, _ci] + _A8 + [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    ("eaf_srv_poll", _ci, [_vp, ctypes.c_longlong, _pd, _pi, _pi, _pi]),
    ("eaf_srv_wait", _ci, [_vp, ctypes.c_longlong, _cd, _pd, _pi, _pi, _pi]),
    ("eaf_srv_stats", _ci, [_vp, _vp]),
    ("eaf_srv_reset_stats", _ci, [_vp]),
    ("eaf_srv_inject_fault", _ci, [_vp, _ci]),
    ("eaf_cg_solve_f64_noalloc", _ci,
     [_ci, _ci, _ci, _ci, _vp] + _A8 + [_vp, _ci, _cd, _pd, _pi]),
]

_lib = None


class EafError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, f"status {status}")
        detail = ""
        if status == EAF_ECUDA and _lib is not None:
            detail = " (" + (_lib.eaf_last_error() or b"").decode() + ")"
        super().__init__(f"{what}: {name}{detail}" if what else name + detail)


def load() -> ctypes.CDLL:
    """The loaded library; raises if it was never built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libeafcg.so is missing at {LIB_PATH}; build it with "
            "`python hornofusion-full3d_b200/build.py` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str = "", allow=(EAF_OK,)) -> int:
    if status not in allow:
        raise EafError(status, what)
    return status
