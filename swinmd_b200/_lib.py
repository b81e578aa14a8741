"""ctypes binding of the C ABI in ``include/swinmd_b200.h``.

The CUDA library is the only compute path: if ``libswinmd_b200.so`` is
missing or cannot be loaded this module raises instead of falling back to
anything else.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libswinmd_b200.so")

SMD_OK = 0
ERRORS = {1: "SMD_ERR_ARG", 2: "SMD_ERR_CUDA", 3: "SMD_ERR_LIST_OVERFLOW", 4: "SMD_ERR_NH_ITER",
          5: "SMD_ERR_SHAKE", 6: "SMD_ERR_NAN", 7: "SMD_ERR_CG", 8: "SMD_ERR_NO_DEVICE",
          9: "SMD_ERR_TIMEOUT", 10: "SMD_ERR_BOX"}
SMD_ERR_ARG, SMD_ERR_CUDA, SMD_ERR_LIST_OVERFLOW, SMD_ERR_NH_ITER = 1, 2, 3, 4
SMD_ERR_SHAKE, SMD_ERR_NAN, SMD_ERR_CG, SMD_ERR_NO_DEVICE, SMD_ERR_TIMEOUT, SMD_ERR_BOX = 5, 6, 7, 8, 9, 10
PREC_FP64, PREC_MIXED = 0, 1
TERM_VDW, TERM_EWALD_REAL, TERM_EWALD_LONG, TERM_ALL = 1, 2, 4, 0xFFFF
TERM_MP_SHORT, TERM_MP_LONG, TERM_IND_SHORT, TERM_IND_LONG = 8, 16, 32, 64
TERM_BOND, TERM_ANGLE, TERM_UB, TERM_WOLF = 128, 256, 512, 1024
# fields of Ensemble::myLustig in declaration order (SMD_LUS_*)
LUSTIG_FIELDS = ("ljUlus", "ljdUlus", "ljd2Ulus", "virialcorrect", "intravirCorrect", "longDeriv",
                 "realDeriv", "realSecDeriv", "longSecDeriv", "surfDeriv", "surfSecDeriv", "inducEn",
                 "inducDeriv", "molDeriv", "molSecDeriv", "BondDeriv", "BondSecDeriv", "intravirPolCorrect",
                 "longPolDeriv", "realPolDeriv", "realSecPolDeriv", "longSecPolDeriv", "surfPolDeriv",
                 "surfSecPolDeriv", "molPolDeriv", "molSecPolDeriv", "selfPolDeriv", "ubDeriv", "ubSecDeriv")
E_VDW, E_REAL, E_LONG, E_CORRECT, E_MOLCORRECT, E_SURF = 0, 1, 2, 3, 4, 5
E_POL_REAL, E_POL_LONG, E_POL_SELF, E_POL_INTRA = 6, 7, 8, 9
E_POL_SURF, E_BOND, E_ANGLE, E_UB, E_TERMS, E_COUNT = 10, 11, 12, 13, 14, 16
VDW_NONE, VDW_LJ, VDW_MIE, VDW_BMH, VDW_BUFF = 0, 1, 2, 3, 4
GUESS_DIRECT, GUESS_PREVIOUS, GUESS_LEARNED, GUESS_FIRST_ORDER, GUESS_EXTRAP2, GUESS_EXTRAP3 = 0, 1, 2, 3, 4, 5
PRECOND_SITE, PRECOND_MOLECULE = 0, 1
THERMO_NONE, THERMO_NOSE_HOOVER, THERMO_NH_CHAIN = 0, 1, 2


class SmdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class IntegratorParams(ctypes.Structure):
    _fields_ = [("timestep", ctypes.c_double), ("temperature", ctypes.c_double),
                ("coupl_const", ctypes.c_double), ("thermostat", ctypes.c_int),
                ("atom_thermo", ctypes.c_int), ("constraint", ctypes.c_int),
                ("long_steps", ctypes.c_int), ("shake_tol", ctypes.c_double),
                ("shake_max_iter", ctypes.c_int), ("atom_ndf", ctypes.c_int),
                ("mol_ndf", ctypes.c_int), ("strain_rate", ctypes.c_double)]


class Observables(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int64), ("list_updates", ctypes.c_int64),
                ("energy", ctypes.c_double * E_COUNT), ("e_potential", ctypes.c_double),
                ("ke_atom", ctypes.c_double), ("ke_mol", ctypes.c_double),
                ("t_atom", ctypes.c_double), ("t_mol", ctypes.c_double),
                ("zeta", ctypes.c_double), ("virial", ctypes.c_double * 9),
                ("atom_pressure", ctypes.c_double * 9), ("mol_pressure", ctypes.c_double * 9),
                ("volume", ctypes.c_double), ("pairs_in_cutoff", ctypes.c_int64),
                ("status", ctypes.c_uint32), ("pad", ctypes.c_uint32),
                ("shear_offset", ctypes.c_double)]


class Averages(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_int64)] + \
               [(k, ctypes.c_double) for k in ("e_potential", "e_potential_sq", "e_total", "e_total_sq",
                                               "ke_atom", "ke_atom_sq", "ke_mol", "ke_mol_sq", "inv_ke_mol",
                                               "volume", "volume_sq")] + \
               [("atom_stress", ctypes.c_double * 5), ("mol_stress", ctypes.c_double * 5),
                ("atom_pressure", ctypes.c_double * 9), ("mol_pressure", ctypes.c_double * 9)]


_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int32)
_F = ctypes.POINTER(ctypes.c_float)

# name: (restype, argtypes)
SIGNATURES = {
    "smd_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    "smd_compute_forces_noalloc": (ctypes.c_int, [_P, ctypes.c_uint32, _D, _D, _D]),
    "smd_batch_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.POINTER(_P)]),
    "smd_batch_destroy": (None, [_P]),
    "smd_batch_last_error": (ctypes.c_char_p, [_P]),
    "smd_batch_autotune": (ctypes.c_int, [_P, ctypes.c_int, _I]),
    "smd_batch_run": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "smd_destroy": (None, [_P]),
    "smd_last_error": (ctypes.c_char_p, [_P]),
    "smd_set_topology": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _I, _I, _D, _D]),
    "smd_set_exclusions": (ctypes.c_int, [_P, _I, _I]),
    "smd_set_box": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "smd_set_pairlist": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "smd_set_vdw": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double]),
    "smd_set_ewald": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "smd_set_precision": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_set_tuning": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_set_reference_forms": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_upload_positions": (ctypes.c_int, [_P, _D]),
    "smd_upload_velocities": (ctypes.c_int, [_P, _D, _D]),
    "smd_download_state": (ctypes.c_int, [_P, _D, _D, _D]),
    "smd_download_real_positions": (ctypes.c_int, [_P, _D]),
    "smd_upload_real_positions": (ctypes.c_int, [_P, _D]),
    "smd_get_integrator_state": (ctypes.c_int, [_P, _D]),
    "smd_set_integrator_state": (ctypes.c_int, [_P, _D]),
    "smd_compute_forces": (ctypes.c_int, [_P, ctypes.c_uint32, _D, _D, _D]),
    "smd_get_pairs": (ctypes.c_int, [_P, _I, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "smd_ewald_nk": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "smd_set_integrator": (ctypes.c_int, [_P, ctypes.POINTER(IntegratorParams)]),
    "smd_lustig_lj": (ctypes.c_int, [_P, _D]),
    "smd_lustig": (ctypes.c_int, [_P, _D]),
    "smd_set_solver_pipelined": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_mlp_set_tensor_path": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_set_induction_damping": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_set_saap": (ctypes.c_int, [_P, _D, ctypes.c_int, ctypes.c_double]),
    "smd_set_wolf": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _I, ctypes.c_double]),
    "smd_set_barostat": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "smd_get_box": (ctypes.c_int, [_P, _D]),
    "smd_set_constraints": (ctypes.c_int, [_P, _D]),
    "smd_integrator_start": (ctypes.c_int, [_P]),
    "smd_integrator_resume": (ctypes.c_int, [_P]),
    "smd_run": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_get_observables": (ctypes.c_int, [_P, ctypes.POINTER(Observables)]),
    "smd_set_series_capacity": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_get_series": (ctypes.c_int, [_P, _D, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "smd_profile_stages": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "smd_step_kernel_count": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "smd_run_timed": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "smd_set_buff": (ctypes.c_int, [_P, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                    _D, ctypes.c_double, ctypes.c_double]),
    "smd_set_bonded": (ctypes.c_int, [_P, ctypes.c_int, _I, ctypes.c_int, _D, ctypes.c_int, _I, ctypes.c_int, _D,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    "smd_set_surface_correct": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_rdf_setup": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_averages_reset": (ctypes.c_int, [_P]),
    "smd_get_averages": (ctypes.c_int, [_P, ctypes.POINTER(Averages)]),
    "smd_rdf_sample": (ctypes.c_int, [_P]),
    "smd_rdf_get": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), _D, _D, ctypes.POINTER(ctypes.c_int64)]),
    "smd_set_multipole": (ctypes.c_int, [_P, _D, _D, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double]),
    "smd_set_solver": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "smd_set_preconditioner": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_solver_stats": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), _D]),
    "smd_solver_trace": (ctypes.c_int, [_P, _D, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "smd_set_wait_limit": (ctypes.c_int, [_P, ctypes.c_double]),
    "smd_test_skip_arrival": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_get_polarization": (ctypes.c_int, [_P, _D, _D, _D, _D]),
    "smd_set_induced": (ctypes.c_int, [_P, _D]),
    "smd_mlp_init": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_uint]),
    "smd_mlp_dims": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "smd_mlp_set_base": (ctypes.c_int, [_P, ctypes.c_int]),
    "smd_mlp_collect": (ctypes.c_int, [_P]),
    "smd_mlp_train": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_uint, _D]),
    "smd_mlp_params": (ctypes.c_int, [_P, _F, _F, ctypes.POINTER(ctypes.c_int)]),
    "smd_mlp_eval": (ctypes.c_int, [_P, _F, ctypes.c_int, _F]),
    "smd_mlp_gradient": (ctypes.c_int, [_P, _F, ctypes.c_int, _F]),
    "smd_mlp_features": (ctypes.c_int, [_P, _F]),
}

_lib = None


def load():
    """Loads the CUDA library once; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built: run `python -m swinmd_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def dptr(a):
    return a.ctypes.data_as(_D) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_I) if a is not None else None


def fptr(a):
    return a.ctypes.data_as(_F) if a is not None else None


def check(ctx, code):
    if code != SMD_OK:
        msg = load().smd_last_error(ctx) if ctx else b""
        raise SmdError(code, (msg or b"").decode())
