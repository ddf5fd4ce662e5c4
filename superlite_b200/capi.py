"""ctypes binding of libslg (include/slg.h).

This is the reference-facing Python layer: it loads the in-tree CUDA library
``superlite_b200/_lib/libslg.so`` and fails loudly when it is missing or when
no CUDA device is present -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libslg.so")

SLG_OK = 0
ERRORS = {-1: "SLG_ERR_CUDA", -2: "SLG_ERR_ARG", -3: "SLG_ERR_STATE", -4: "SLG_ERR_UNSORTED",
          -5: "SLG_ERR_OOM", -6: "SLG_ERR_NOT_BUILT", -7: "SLG_ERR_TOO_LARGE"}

vp = C.c_void_p


class SlgGas(C.Structure):
    _fields_ = [("temp", vp), ("natom", vp), ("nelec", vp), ("vol", vp), ("mass", vp), ("natomfr", vp),
                ("oc", vp), ("ginv", vp)]


class SlgOpacityFlags(C.Structure):
    _fields_ = [("nobb", C.c_int32), ("nobf", C.c_int32), ("noff", C.c_int32), ("nothmson", C.c_int32),
                ("ngs", C.c_int32), ("opacmixrossel", C.c_double)]


class SlgTransportIn(C.Structure):
    _fields_ = [("tempinv", vp), ("sig", vp), ("capgrey", vp), ("emitprob", vp), ("opaclump", vp), ("cap", vp),
                ("tauddmc", C.c_double), ("taulump", C.c_double), ("puretran", C.c_int32),
                ("noampfact", C.c_int32), ("errorfatal", C.c_int32), ("thm_aniso", C.c_int32),
                ("dogrdtally", C.c_int32), ("precision", C.c_int32), ("max_steps", C.c_int64)]


class SlgTransportOut(C.Structure):
    _fields_ = [("tally", vp), ("jrad", vp), ("eamp", vp), ("methodswap", vp), ("tot_evelo", C.c_double),
                ("tot_eout", C.c_double), ("tot_sflux", C.c_double), ("npckt", C.c_int64), ("nflux", C.c_int64),
                ("nstepimc", C.c_int64), ("nstepddmc", C.c_int64), ("nmethodswap", C.c_int64),
                ("nstepmax", C.c_int64), ("ndist", C.c_int64 * 11), ("nposwarn", C.c_int64),
                ("ierr", C.c_int32), ("ierr_part", C.c_int32)]


class SlgGridDev(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ng", C.c_int32), ("xarr", vp), ("vxarr", vp), ("divv", vp), ("wl", vp),
                ("wlinv", vp)]


# name -> (restype, argtypes); every symbol declared in include/slg.h
SIGNATURES = {
    "slg_create": (vp, [C.c_int]),
    "slg_destroy": (None, [vp]),
    "slg_last_error": (C.c_char_p, [vp]),
    "slg_version": (C.c_char_p, []),
    "slg_set_groups": (C.c_int, [vp, C.c_int32, vp]),
    "slg_set_grid": (C.c_int, [vp, C.c_int32, vp, vp, vp, vp]),
    "slg_set_models": (C.c_int, [vp, C.c_int32, vp, vp, vp, vp, vp, vp]),
    "slg_set_atomic_data": (C.c_int, [vp, C.c_int32, C.c_int32, vp, C.c_int64, vp, vp, vp, vp]),
    "slg_physical_opacity": (C.c_int, [vp, C.POINTER(SlgGas), C.POINTER(SlgOpacityFlags), vp, vp, vp, vp, vp]),
    "slg_analytic_opacity": (C.c_int, [vp, vp, vp, C.c_int32] + [C.c_double] * 8 + [vp, vp]),
    "slg_dev_analytic_opacity": (C.c_int, [vp, vp, vp, C.c_int32] + [C.c_double] * 8 + [vp, vp]),
    "slg_opacity_means": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "slg_leakage_opacity11": (C.c_int, [vp, vp, vp, vp, vp, C.c_double, C.c_double, vp]),
    "slg_emission_probability": (C.c_int, [vp, vp, vp, vp, vp]),
    "slg_particle_advance": (C.c_int, [vp, C.POINTER(SlgTransportIn), vp, vp, C.c_int64, C.c_uint64,
                                       C.POINTER(SlgTransportOut)]),
    "slg_set_trace": (C.c_int, [vp, vp, vp]),
    "slg_fluxtally": (C.c_int, [vp, C.c_int64, vp, vp, C.c_int32, vp, vp, vp, vp]),
    "slg_sourcetally": (C.c_int, [vp, C.c_int64, vp, vp, vp, vp]),
    "slg_dev_physical_opacity": (C.c_int, [vp, C.POINTER(SlgGas), C.POINTER(SlgOpacityFlags), vp, vp, vp, vp]),
    "slg_dev_opacity_means": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "slg_dev_leakage_opacity11": (C.c_int, [vp, vp, vp, vp, vp, C.c_double, C.c_double, vp]),
    "slg_dev_emission_probability": (C.c_int, [vp, vp, vp, vp, vp]),
    "slg_dev_particle_advance": (C.c_int, [vp, C.POINTER(SlgTransportIn), vp, vp, C.c_int64, C.c_uint64,
                                           C.POINTER(SlgTransportOut)]),
    "slg_dev_fluxtally": (C.c_int, [vp, C.c_int64, vp, vp, C.c_int32, vp, vp, vp, vp]),
    "slg_dev_sourcetally": (C.c_int, [vp, C.c_int64, vp, vp, vp, vp]),
    "slg_sourceenergy": (C.c_int, [vp, vp, C.c_double, vp, vp]),
    "slg_sourcenumbers": (C.c_int64, [vp, vp, C.c_double, C.c_int64, C.c_int64, vp]),
    "slg_models_sourcenumbers": (C.c_int64, [vp, vp, C.c_double, vp, vp, vp]),
    "slg_interior_source": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_int64, C.c_uint64, vp]),
    "slg_dev_interior_source": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_int64, C.c_uint64, vp]),
    "slg_particle_advance_static": (C.c_int, [C.POINTER(SlgGridDev), C.POINTER(SlgTransportIn), vp, vp, C.c_int64,
                                              C.c_uint64, C.POINTER(SlgTransportOut), vp]),
    "slg_autotune_transport": (C.c_int, [vp, C.POINTER(SlgTransportIn), vp, vp, C.c_int64, C.c_uint64, C.c_int64,
                                         vp, vp]),
    "slg_set_transport_variant": (C.c_int, [vp, C.c_int32]),
    "slg_sync": (C.c_int, [vp]),
    "slg_set_element_masses": (C.c_int, [vp, C.c_int32, vp]),
    "slg_dev_opacity_grad_forward": (C.c_int, [vp, vp, vp, vp, C.c_double, C.c_double, C.c_double] + [vp] * 6),
    "slg_dev_opacity_grad_backward": (C.c_int, [vp, vp, vp, vp, C.c_double, C.c_double, C.c_double] + [vp] * 14),
    "slg_partition_functions": (None, [C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, C.c_double, vp]),
    "slg_set_ions": (C.c_int, [vp, C.c_int32, C.c_int32, vp, vp, vp, vp]),
    "slg_saha_eos": (C.c_int, [vp, vp, vp, vp, vp, C.c_double, vp, C.c_int32, vp, vp, vp]),
    "slg_dev_saha_eos": (C.c_int, [vp, vp, vp, vp, vp, C.c_double, vp, C.c_int32, vp, vp, vp]),
    "slg_graph_begin": (C.c_int, [vp]),
    "slg_graph_end": (C.c_int, [vp]),
    "slg_graph_launch": (C.c_int, [vp, C.c_int32]),
    "slg_transport_totals": (C.c_int, [vp, vp, C.c_int32]),
    "slg_stream": (vp, [vp]),
    "slg_pipe_throughput": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    "slg_exp_eval": (C.c_int, [C.c_int, C.c_int64, C.c_void_p, C.c_void_p]),
}

_LIB = None


def load(path: str = LIB_PATH):
    """Load libslg.so and declare every entry point; raises if the library is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"libslg.so not built ({path}); run python -m superlite_b200.build")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class SlgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def ptr(a):
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch.Tensor
