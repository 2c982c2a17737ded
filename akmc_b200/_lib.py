"""ctypes binding of ``libakmc_b200.so`` (the C ABI declared in include/akmc.h).

The library must exist: there is no CPU fallback.  ``load()`` raises if the shared
object is missing and ``akmc_b200.build`` has not been run.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
# AKMC_LIB selects another build of the same C ABI, e.g. the self-checking
# libakmc_b200_checks.so (python -m akmc_b200.build --checks)
LIB_PATH = os.environ.get("AKMC_LIB") or os.path.join(PKG, "libakmc_b200.so")
CHECKS_LIB_PATH = os.path.join(PKG, "libakmc_b200_checks.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Energy(C.Structure):
    """akmc_energy: the Energy fields Field::calculateForces writes (metal/Energy.h:13-108)."""
    _fields_ = [("total", C.c_double), ("rcp", C.c_double), ("real", C.c_double),
                ("vdw", C.c_double), ("many", C.c_double)]

    def getTotalEnergy(self):
        return self.rcp + self.real + self.vdw + self.many

    def as_dict(self):
        return dict(total=self.total, rcp=self.rcp, real=self.real, vdw=self.vdw, many=self.many)


class FireParams(C.Structure):
    """akmc_fire_params: RelaxCntrl (Common/RelaxCntrl.h:15-38)."""
    _fields_ = [("max_iter", C.c_int), ("n_min", C.c_int), ("norm_tol", C.c_double),
                ("force_tol", C.c_double), ("dt0", C.c_double), ("dt_max", C.c_double),
                ("alpha0", C.c_double), ("alpha_dec", C.c_double), ("step_inc", C.c_double),
                ("step_dec", C.c_double), ("max_move", C.c_double)]


class DimerParams(C.Structure):
    """akmc_dimer_params: DimerCntrl (Common/DimerCntrl.h:18-88) names where one exists."""
    _fields_ = [("max_iter", C.c_int), ("max_rotations", C.c_int), ("n_min", C.c_int),
                ("patience", C.c_int), ("delta", C.c_double), ("rot_tol", C.c_double),
                ("force_tol", C.c_double), ("max_eigenvalue", C.c_double),
                ("min_trial", C.c_double), ("max_move", C.c_double), ("max_rise", C.c_double),
                ("dt0", C.c_double), ("dt_max", C.c_double), ("alpha0", C.c_double),
                ("alpha_dec", C.c_double), ("step_inc", C.c_double), ("step_dec", C.c_double),
                ("translation", C.c_int), ("lbfgs_memory", C.c_int), ("max_step", C.c_double),
                ("convex_step", C.c_double)]


class WalkerResult(C.Structure):
    """akmc_walker_result."""
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("force_calls", C.c_int),
                ("reserved", C.c_int), ("energy", C.c_double), ("curvature", C.c_double),
                ("fmax", C.c_double), ("fnorm", C.c_double)]


class KmcStep(C.Structure):
    """akmc_kmc_step: the outcome of one KMC selection."""
    _fields_ = [("chosen", C.c_int), ("n_usable", C.c_int), ("total_rate", C.c_double),
                ("dt", C.c_double), ("barrier", C.c_double), ("rate", C.c_double),
                ("u1", C.c_double), ("u2", C.c_double)]


class ProposalParams(C.Structure):
    """akmc_proposal_params: how model predictions become walker starting displacements."""
    _fields_ = [("threshold", C.c_double), ("min_score", C.c_double), ("scale", C.c_double),
                ("noise", C.c_double), ("radius", C.c_double), ("min_disp", C.c_double),
                ("region", C.c_double), ("group", C.c_int)]


# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("akmc_field_create", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    ("akmc_field_create_from_text", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    ("akmc_field_setup", C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
    ("akmc_field_destroy", C.c_int, [C.c_void_p]),
    ("akmc_forces", C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp,
                              C.POINTER(Energy)]),
    ("akmc_batch_create", C.c_int, [C.c_void_p, C.c_int, _ip, _dp, _ip, _dp,
                                    C.POINTER(C.c_void_p)]),
    ("akmc_batch_create_skin", C.c_int, [C.c_void_p, C.c_int, _ip, _dp, _ip, _dp, C.c_double,
                                         C.POINTER(C.c_void_p)]),
    ("akmc_batch_destroy", C.c_int, [C.c_void_p]),
    ("akmc_batch_list_modes", C.c_int, [C.c_void_p, _ip]),
    ("akmc_batch_forces", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]),
    ("akmc_batch_forces_host", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    ("akmc_batch_launches", C.c_int, [C.c_void_p]),
    ("akmc_batch_neighbours", C.c_int, [C.c_void_p, _ip, _ip, C.c_int]),
    ("akmc_batch_set_home_chunk", C.c_int, [C.c_void_p, C.c_int]),
    ("akmc_batch_home_chunk", C.c_int, [C.c_void_p]),
    ("akmc_batch_autotune", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, _ip]),
    ("akmc_batch_profile", C.c_int, [C.c_void_p, C.c_int]),
    ("akmc_batch_kernel_times", C.c_int, [C.c_void_p, _dp, _ip, C.POINTER(C.c_char_p), C.c_int]),
    ("akmc_eam_forces_noalloc", C.c_int, [C.c_void_p, C.c_int, _dp, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("akmc_field_set_precision", C.c_int, [C.c_void_p, C.c_int]),
    ("akmc_field_family", C.c_int, [C.c_void_p]),
    ("akmc_field_num_species", C.c_int, [C.c_void_p]),
    ("akmc_field_species", C.c_int, [C.c_void_p, C.c_int, C.c_char_p, _dp, _dp]),
    ("akmc_field_cutoff", C.c_double, [C.c_void_p]),
    ("akmc_field_ewald", C.c_int, [C.c_void_p, _dp, _ip, _ip]),
    ("akmc_fire_defaults", None, [C.POINTER(FireParams)]),
    ("akmc_dimer_defaults", None, [C.POINTER(DimerParams)]),
    ("akmc_walkers_create", C.c_int, [C.c_void_p, C.c_int, _ip, _dp, _ip, _dp, _ip,
                                      C.POINTER(C.c_void_p)]),
    ("akmc_walkers_destroy", C.c_int, [C.c_void_p]),
    ("akmc_walkers_count", C.c_int, [C.c_void_p]),
    ("akmc_walkers_set_skin", C.c_int, [C.c_void_p, C.c_double]),
    ("akmc_walkers_skin", C.c_double, [C.c_void_p]),
    ("akmc_walkers_relax", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(FireParams),
                                     C.POINTER(WalkerResult), C.c_void_p]),
    ("akmc_walkers_dimer", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(DimerParams),
                                     C.POINTER(WalkerResult), C.c_void_p]),
    ("akmc_kmc_uniforms", C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, C.c_void_p,
                                    C.c_void_p]),
    ("akmc_events_dedup", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                    C.c_void_p, C.c_void_p]),
    ("akmc_kmc_select", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                  C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    ("akmc_mlp_num_params", C.c_int, []),
    ("akmc_batch_descriptors", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("akmc_batch_descriptors_rows", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("akmc_mlp_forward", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    ("akmc_mlp_forward_fp32pipe", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p]),
    ("akmc_mlp_check", C.c_int, []),
    ("akmc_mlp_train_step", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                      C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("akmc_mlp_train_step_fp32pipe", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                      C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("akmc_walkers_relax_subset", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(FireParams), C.c_void_p,
                                            C.POINTER(WalkerResult), C.c_void_p]),
    ("akmc_walkers_dimer_subset", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(DimerParams),
                                            C.c_void_p, C.POINTER(WalkerResult), C.c_void_p]),
    ("akmc_walkers_descriptors", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("akmc_walkers_descriptors_rows", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                                C.c_void_p, C.c_void_p]),
    ("akmc_proposal_seeds", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int, C.POINTER(ProposalParams), C.c_uint64, C.c_uint64,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("akmc_last_error", C.c_char_p, []),
    ("akmc_version", C.c_char_p, []),
    ("akmc_checks_enabled", C.c_int, []),
    ("akmc_field_set_list_density", C.c_int, [C.c_void_p, C.c_double]),
    ("akmc_batch_set_system_chunks", C.c_int, [C.c_void_p, _ip]),
    ("akmc_batch_autotune_classes", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, _ip, _ip, _ip, C.POINTER(C.c_float), C.c_int]),
    ("akmc_batch_total_items", C.c_int, [C.c_void_p]),
    ("akmc_walkers_tuning", C.c_int, [C.c_void_p, C.c_int, _ip, _ip, C.POINTER(C.c_float), C.c_int]),
    ("akmc_walkers_skip_tuning", C.c_int, [C.c_void_p]),
    ("akmc_checks_read", C.c_int, [_ip, _ip, C.c_int]),
]

_lib = None


def load():
    """Load the shared library (once) and declare every signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m akmc_b200.build` "
                               "(the force path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class AkmcError(RuntimeError):
    def __init__(self, code, where):
        msg = load().akmc_last_error().decode(errors="replace")
        super().__init__(f"{where}: status {code} ({STATUS_NAMES.get(code, '?')}): {msg}")
        self.code = code


STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_EMBED_RANGE", 3: "ERR_TABLE_RANGE",
                4: "ERR_CUTOFF", 5: "ERR_IO", 6: "ERR_PARSE", 7: "ERR_UNSUPPORTED",
                8: "ERR_CUDA", 9: "ERR_NONFINITE", 10: "ERR_STATE", 11: "ERR_CAPACITY"}
STATUS = {v: k for k, v in STATUS_NAMES.items()}


def check(code, where):
    if code != 0:
        raise AkmcError(code, where)
