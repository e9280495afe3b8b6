"""The freestream_input parameter block in pure Python (no library load).

`Params` has the field order and types of `fsm_params` in include/fsm.h, which
are those of the reference's `struct parameters` (src/Parameter.h:2-33), so a
`Params` instance passes straight to the C ABI.  `default_params` and `derive`
restate fsm_params_default / fsm_params_derive (the reference's defaults,
src/FreestreamMilne.cpp:149-171, and DIM / TAU, :177-178) with float32
arithmetic, so that code which only builds workloads -- the synthetic event
generators, the CPU reference timing -- never loads libfsm.so.
"""
import ctypes

import numpy as np

PARAM_FIELDS = [
    ("OUTPUTFORMAT", ctypes.c_int), ("BARYON", ctypes.c_int), ("IC_ENERGY", ctypes.c_int),
    ("IC_BARYON", ctypes.c_int), ("ETA_WIDTH", ctypes.c_float), ("ETA_FLAT", ctypes.c_float),
    ("SIGMA", ctypes.c_float), ("SIGMA_B", ctypes.c_float), ("DIM_X", ctypes.c_int),
    ("DIM_Y", ctypes.c_int), ("DIM_ETA", ctypes.c_int), ("DIM_RAP", ctypes.c_int),
    ("DIM_PHIP", ctypes.c_int), ("DX", ctypes.c_float), ("DY", ctypes.c_float),
    ("DETA", ctypes.c_float), ("DRAP", ctypes.c_float), ("DTAU", ctypes.c_float),
    ("TAU0", ctypes.c_float), ("EOS_TYPE", ctypes.c_int), ("E_FREEZE", ctypes.c_float),
    ("VISCOUS_MATCHING", ctypes.c_int), ("E_DEP_FS", ctypes.c_int), ("E_R", ctypes.c_float),
    ("TAU_R", ctypes.c_float), ("ALPHA", ctypes.c_float), ("DIM", ctypes.c_int),
    ("TAU", ctypes.c_float),
]

# src/FreestreamMilne.cpp:149-171 (E_R, TAU_R, ALPHA have no default there:
# 1, 1, 0 here, as in fsm_params_default)
DEFAULTS = dict(OUTPUTFORMAT=2, BARYON=0, IC_ENERGY=5, IC_BARYON=1, ETA_WIDTH=0.5, ETA_FLAT=0.5,
                SIGMA=1.0, SIGMA_B=1.0, DIM_X=101, DIM_Y=101, DIM_ETA=1, DIM_RAP=1, DIM_PHIP=51,
                DX=0.1, DY=0.1, DETA=0.1, DRAP=0.2, DTAU=0.5, TAU0=0.1, EOS_TYPE=1,
                E_FREEZE=1.7, VISCOUS_MATCHING=1, E_DEP_FS=0, E_R=1.0, TAU_R=1.0, ALPHA=0.0)


class Params(ctypes.Structure):
    _fields_ = PARAM_FIELDS

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in PARAM_FIELDS}


def derive(p):
    """DIM = DIM_X*DIM_Y*DIM_ETA and TAU = TAU0 + DTAU in float32."""
    p.DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA
    p.TAU = float(np.float32(p.TAU0) + np.float32(p.DTAU))
    return p


def default_params(**kw):
    """The reference's defaults, overridden by `kw`, with DIM and TAU derived."""
    p = Params(**DEFAULTS)
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return derive(p)
