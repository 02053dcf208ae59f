"""ctypes binding of the in-tree CUDA library (``include/ibis_b200.h``).

The product path has no CPU fallback: :func:`load` raises when the library is
missing or a symbol is absent, and the callers in this package never fall back
to a host implementation.
"""
from __future__ import annotations

import ctypes
import os
import re

from .params import IbisDayParamsC, IbisParamsC

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "_lib", "libibis_b200.so")



class IbisEnsembleC(ctypes.Structure):
    """ctypes mirror of ``IbisEnsemble`` (include/ibis_b200.h)."""
    _fields_ = [("prog", ctypes.c_void_p), ("acc", ctypes.c_void_p), ("stat", ctypes.c_void_p),
                ("forc", ctypes.c_void_p), ("run_params", ctypes.c_void_p), ("run_site", ctypes.c_void_p),
                ("run_forc", ctypes.c_void_p), ("run_nstep", ctypes.c_void_p), ("run_pos", ctypes.c_void_p),
                ("order", ctypes.c_void_p), ("yearly", ctypes.c_void_p), ("forc_len", ctypes.c_longlong),
                ("nrun", ctypes.c_int), ("ld_run", ctypes.c_int), ("nsite", ctypes.c_int),
                ("ld_site", ctypes.c_int), ("nyear", ctypes.c_int), ("year_steps", ctypes.c_int),
                ("norder", ctypes.c_int), ("queue", ctypes.c_void_p),
                ("status", ctypes.c_void_p)]


class IbisEnsembleDailyC(ctypes.Structure):
    """ctypes mirror of ``IbisEnsembleDaily`` (include/ibis_b200.h)."""
    _fields_ = [("records", ctypes.c_void_p), ("site_lat", ctypes.c_void_p), ("len", ctypes.c_longlong),
                ("seed", ctypes.c_uint), ("flags", ctypes.c_uint)]


class IbisWetlandBuilderC(ctypes.Structure):
    """ctypes mirror of ``IbisWetlandBuilder`` (include/ibis_b200.h)."""
    _fields_ = [("npoi", ctypes.c_int), ("ld", ctypes.c_int), ("nlat", ctypes.c_int), ("nlon", ctypes.c_int),
                ("cell_i", ctypes.c_void_p), ("cell_j", ctypes.c_void_p), ("poros", ctypes.c_void_p),
                ("hsoi", ctypes.c_double * 4), ("lf", ctypes.c_void_p), ("buf", ctypes.c_void_p),
                ("work", ctypes.c_void_p), ("nmonth", ctypes.c_int)]


class IbisForestC(ctypes.Structure):
    """ctypes mirror of ``IbisForest`` (include/ibis_b200.h)."""
    _fields_ = [("nband", ctypes.c_int), ("nfeat", ctypes.c_int), ("tree_first", ctypes.c_void_p),
                ("node_first", ctypes.c_void_p), ("left", ctypes.c_void_p), ("right", ctypes.c_void_p),
                ("feature", ctypes.c_void_p), ("value", ctypes.c_void_p), ("default_left", ctypes.c_void_p),
                ("base_margin", ctypes.c_void_p), ("transform", ctypes.c_void_p)]


_c_int_p = ctypes.POINTER(ctypes.c_int)
_P = ctypes.POINTER(IbisParamsC)
_E = ctypes.POINTER(IbisEnsembleC)
_DP = ctypes.POINTER(IbisDayParamsC)
_V = ctypes.c_void_p

# name -> (restype, argtypes); every function declared in include/*.h
SIGNATURES = {
    "ibis_step_f32": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.c_int] * 3 + [_P, ctypes.c_void_p, ctypes.c_void_p]),
    "ibis_step_f64": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.c_int] * 3 + [_P, ctypes.c_void_p, ctypes.c_void_p]),
    "ibis_step_split_f32": (ctypes.c_int, [ctypes.c_void_p] * 6 + [ctypes.c_int] * 3
                            + [_P, ctypes.c_void_p, ctypes.c_void_p]),
    "ibis_mid_planes": (ctypes.c_int, []),
    "ibis_step_config_f32": (ctypes.c_int, [ctypes.c_void_p] * 6 + [ctypes.c_int] * 3
                             + [_P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "ibis_num_configs": (ctypes.c_int, []),
    "ibis_step_split_noalloc_f32": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.c_int] * 3
                                    + [_P, ctypes.c_void_p, ctypes.c_void_p]),
    "ibis_config_info": (ctypes.c_int, [ctypes.c_int] + [_c_int_p] * 5),
    "ibis_wetland_dynamic_f32": (ctypes.c_int, [_V] * 4 + [ctypes.c_int] * 2 + [_P, _V]),
    "ibis_wetland_grid": (ctypes.c_int, [ctypes.POINTER(IbisWetlandBuilderC), _V]),
    "ibis_wetland_features": (ctypes.c_int, [ctypes.POINTER(IbisWetlandBuilderC)] + [_V] * 4),
    "ibis_wetland_learned": (ctypes.c_int, [ctypes.POINTER(IbisForestC), _V] + [ctypes.c_int] * 2 + [_V] * 7
                             + [ctypes.c_int] + [_V] * 3),
    "ibis_day_host_f32": (ctypes.c_int, [_V] * 9 + [ctypes.c_int] * 5 + [ctypes.c_uint] * 2 + [_P, _V]
                          + [ctypes.c_int] * 2 + [_V]),
    "ibis_step_host_f32": (ctypes.c_int, [_V] * 7 + [ctypes.c_int] * 3 + [_P, _V] + [ctypes.c_int] * 3 + [_V]),
    "ibis_ensemble_f32": (ctypes.c_int, [_E, _P, ctypes.c_int, ctypes.c_void_p]),
    "ibis_ensemble_hours_f32": (ctypes.c_int, [_E, _P, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "ibis_ensemble_occupancy": (ctypes.c_int, [_P, ctypes.c_int]),
    "ibis_ensemble_daily_f32": (ctypes.c_int, [_E, ctypes.POINTER(IbisEnsembleDailyC), _P, ctypes.c_int,
                                               ctypes.c_void_p]),
    "ibis_diurnal_f32": (ctypes.c_int, [ctypes.c_void_p] * 3 + [ctypes.c_int] * 5
                         + [ctypes.c_float, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p]),
    "ibis_diurnal_sw_f32": (ctypes.c_int, [_V] * 5 + [ctypes.c_int] * 5
                            + [ctypes.c_float, ctypes.c_uint, ctypes.c_uint, _V]),
    "ibis_day_begin_f32": (ctypes.c_int, [_V] * 4 + [ctypes.c_int] * 2 + [_P, _DP, _V]),
    "ibis_day_begin_f64": (ctypes.c_int, [_V] * 4 + [ctypes.c_int] * 2 + [_P, _DP, _V]),
    "ibis_day_end_f32": (ctypes.c_int, [_V] * 5 + [ctypes.c_int] * 2 + [_P, _DP, _V]),
    "ibis_day_end_f64": (ctypes.c_int, [_V] * 5 + [ctypes.c_int] * 2 + [_P, _DP, _V]),
    "ibis_month_begin_f32": (ctypes.c_int, [_V] * 3 + [ctypes.c_int] * 2 + [ctypes.c_uint, _V]),
    "ibis_month_begin_f64": (ctypes.c_int, [_V] * 3 + [ctypes.c_int] * 2 + [ctypes.c_uint, _V]),
    "ibis_month_end_f32": (ctypes.c_int, [_V] * 6 + [ctypes.c_int] * 3 + [_P, ctypes.c_uint, _V]),
    "ibis_month_end_f64": (ctypes.c_int, [_V] * 6 + [ctypes.c_int] * 3 + [_P, ctypes.c_uint, _V]),
}


_configs = None


def configs():
    """List of dicts describing the launch configurations of the FP32 kernels
    (read from the library once; the table is compiled in).  ``staged`` marks
    the fused configuration whose hourly forcing tiles are brought into shared
    memory by bulk copies."""
    global _configs
    if _configs is not None:
        return [dict(c) for c in _configs]
    L = load()
    out = []
    for i in range(L.ibis_num_configs()):
        v = [ctypes.c_int() for _ in range(5)]
        check(L.ibis_config_info(i, *[ctypes.byref(x) for x in v]), "ibis_config_info")
        f, b, m, b2, m2 = (x.value for x in v)
        out.append(dict(id=i, form="split" if f == 1 else "fused", staged=f == 2, block=b, min_blocks=m,
                        block2=b2, min_blocks2=m2))
    _configs = out
    return [dict(c) for c in out]


_lib = None


class IbisError(RuntimeError):
    pass


def declared_symbols():
    """Function names declared in the public headers."""
    names = []
    inc = os.path.join(REPO, "include")
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        with open(os.path.join(inc, f)) as fh:
            txt = fh.read()
        names += re.findall(r"^\s*(?:int|void|size_t|const char\s*\*)\s+(ibis_\w+)\s*\(", txt, flags=re.M)
    return names


def load(path: str = LIB_PATH):
    """Load the CUDA library (build it first with ``python -m ibis_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise IbisError(f"{path} is missing: build it with `python -m ibis_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            raise IbisError(f"{path} does not export {name}")
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str):
    if rc != 0:
        if rc == -22:
            raise IbisError(f"{what}: invalid argument (EINVAL)")
        if rc <= -1000:
            raise IbisError(f"{what}: CUDA launch error {-rc - 1000}")
        raise IbisError(f"{what}: error {rc}")
