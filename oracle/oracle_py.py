"""TEST INFRASTRUCTURE: ctypes access to the CPU oracle.

Loads ``oracle/_build/liboracle.so`` (the project's CPU restatement of the
freestream-milne hot path) and, where it was built, ``oracle/_ref/libfsm_ref.so``
(the reference's own sources compiled against the project's GSL-API stand-in).
Only tests, the smoke check and bench.py's CPU-baseline leg import this module.
"""
import ctypes
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libfsm_ref.so"

# Field order of `struct parameters` (reference src/Parameter.h:2-33).
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

# Defaults set by the reference before reading freestream_input
# (src/FreestreamMilne.cpp:149-171); E_R/TAU_R/ALPHA have no default there.
DEFAULTS = dict(OUTPUTFORMAT=2, BARYON=0, IC_ENERGY=5, IC_BARYON=1, ETA_WIDTH=0.5, ETA_FLAT=0.5,
                SIGMA=1.0, SIGMA_B=1.0, DIM_X=101, DIM_Y=101, DIM_ETA=1, DIM_RAP=1, DIM_PHIP=51,
                DX=0.1, DY=0.1, DETA=0.1, DRAP=0.2, DTAU=0.5, TAU0=0.1, EOS_TYPE=1,
                E_FREEZE=1.7, VISCOUS_MATCHING=1, E_DEP_FS=0, E_R=1.0, TAU_R=1.0, ALPHA=0.0,
                DIM=0, TAU=0.0)


class Params(ctypes.Structure):
    _fields_ = PARAM_FIELDS


def make_params(**kw):
    d = dict(DEFAULTS)
    d.update(kw)
    unknown = set(d) - {f for f, _ in PARAM_FIELDS}
    if unknown:
        raise KeyError(f"unknown parameters {sorted(unknown)}")
    p = Params(**d)
    p.DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA
    p.TAU = np.float32(p.TAU0) + np.float32(p.DTAU)
    return p


_DP = ctypes.POINTER(ctypes.c_double)


class Out(ctypes.Structure):
    _fields_ = [("T", _DP), ("J", _DP), ("e", _DP), ("P", _DP), ("Pi", _DP), ("u", _DP),
                ("pi", _DP), ("nB", _DP), ("V", _DP), ("dim_phip", ctypes.c_int),
                ("dtau", ctypes.c_float), ("tau", ctypes.c_float), ("n_fallback", ctypes.c_int)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"oracle not built: {ORACLE_SO} (run `make -C oracle`)")
        _lib = ctypes.CDLL(str(ORACLE_SO))
        _lib.oracle_run.argtypes = [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.POINTER(Out), ctypes.c_int]
        _lib.oracle_run.restype = ctypes.c_int
        _lib.oracle_run_fm4.argtypes = _lib.oracle_run.argtypes
        _lib.oracle_run_fm4.restype = ctypes.c_int
        _lib.oracle_spline_derivs.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int, ctypes.c_void_p]
        _lib.oracle_bicubic_eval.argtypes = ([ctypes.c_void_p] * 3 + [ctypes.c_int] * 2 +
                                             [ctypes.c_void_p] * 2 + [ctypes.c_int, ctypes.c_void_p])
        _lib.oracle_eig.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4
        _lib.oracle_eig.restype = ctypes.c_int
        _lib.oracle_landau_cell.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p,
                                            ctypes.c_void_p]
        _lib.oracle_landau_cell.restype = ctypes.c_int
    return _lib


def ref_available():
    return REF_SO.exists()


def ref():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise RuntimeError(f"reference build not present: {REF_SO}")
        _ref = ctypes.CDLL(str(REF_SO))
        _ref.ref_run.argtypes = [ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.POINTER(Out)]
        _ref.ref_run.restype = ctypes.c_int
        _ref.ref_run_fm4.argtypes = _ref.ref_run.argtypes
        _ref.ref_run_fm4.restype = ctypes.c_int
        _ref.ref_run_full.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p]
        _ref.ref_run_full.restype = ctypes.c_int
        _ref.ref_write_outputs.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params)] + [ctypes.c_void_p] * 8
        _ref.ref_write_outputs.restype = ctypes.c_int
        _ref.ref_initial.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params), ctypes.c_int, ctypes.c_void_p]
        _ref.ref_initial.restype = ctypes.c_int
    return _ref


def ref_initial(workdir, params, which):
    """The reference's own initial-condition function `which` (see
    ref_harness.cpp) run inside workdir; returns the float32 profile."""
    out = np.zeros(params.DIM_X * params.DIM_Y * params.DIM_ETA, np.float32)
    rc = ref().ref_initial(str(workdir).encode(), ctypes.byref(params), int(which), out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ref_initial failed with code {rc}")
    return out


def ref_write_outputs(workdir, params, res, diag17):
    """The reference's own writers on host fields (float32 arrays) inside
    workdir/output; diag17 as oracle_diagnostics lays it out."""
    keep = []

    def ptr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float32).ravel()
        keep.append(a)
        return a.ctypes.data

    rc = ref().ref_write_outputs(str(workdir).encode(), ctypes.byref(params), ptr(res["e"]),
                                 ptr(res["P"]), ptr(res["Pi"]), ptr(res["u"]), ptr(res["pi"]),
                                 ptr(res.get("nB")), ptr(res.get("V")), ptr(diag17))
    if rc != 0:
        raise RuntimeError(f"ref_write_outputs failed with code {rc}")


OUT_SHAPES = dict(T=10, J=4, e=1, P=1, Pi=1, u=4, pi=10, nB=1, V=4)


def _alloc_out(dim, baryon):
    arrs = {}
    o = Out()
    for k, ncomp in OUT_SHAPES.items():
        if k in ("J", "nB", "V") and not baryon:
            setattr(o, k, _DP())
            continue
        a = np.zeros((ncomp, dim) if ncomp > 1 else (dim,), dtype=np.float64)
        arrs[k] = a
        setattr(o, k, a.ctypes.data_as(_DP))
    return o, arrs


def run(params, e_gev, nB=None, fp64=False, impl="oracle", nthreads=0, fm4=False):
    """Run the hot path on the CPU.  impl: 'oracle' (restatement) or 'ref'
    (reference sources); fm4: the profile is already in fm^-4 (the reference's
    initial conditions other than the vector).  Returns a dict of float64
    arrays plus metadata."""
    e_gev = np.ascontiguousarray(e_gev, dtype=np.float32).ravel()
    dim = params.DIM_X * params.DIM_Y * params.DIM_ETA
    if e_gev.size != dim:
        raise ValueError(f"input has {e_gev.size} cells, grid has {dim}")
    baryon = bool(params.BARYON)
    nb_ptr = None
    if baryon:
        if nB is None:
            raise ValueError("BARYON=1 needs an nB profile")
        nB = np.ascontiguousarray(nB, dtype=np.float32).ravel()
        nb_ptr = nB.ctypes.data
    o, arrs = _alloc_out(dim, baryon)
    if impl == "oracle":
        fn = lib().oracle_run_fm4 if fm4 else lib().oracle_run
        rc = fn(ctypes.byref(params), int(fp64), e_gev.ctypes.data, nb_ptr, ctypes.byref(o), int(nthreads))
    elif impl == "ref":
        if fp64:
            raise ValueError("the reference build is float only")
        if nthreads:
            os.environ["OMP_NUM_THREADS"] = str(nthreads)
        fn = ref().ref_run_fm4 if fm4 else ref().ref_run
        rc = fn(ctypes.byref(params), e_gev.ctypes.data, nb_ptr, ctypes.byref(o))
    else:
        raise ValueError(impl)
    if rc != 0:
        raise RuntimeError(f"{impl} run failed with code {rc}")
    arrs.update(dim_phip=o.dim_phip, dtau=o.dtau, tau=o.tau, n_fallback=o.n_fallback)
    return arrs


def spline_derivs(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    d = np.zeros_like(y)
    lib().oracle_spline_derivs(x.ctypes.data, y.ctypes.data, len(x), d.ctypes.data)
    return d


def bicubic_eval(x, y, z, px, py):
    x, y = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y))
    z = np.ascontiguousarray(z, dtype=np.float64)  # z[j, i] = f(x[i], y[j])
    px, py = (np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (px, py))
    out = np.zeros(px.size)
    lib().oracle_bicubic_eval(x.ctypes.data, y.ctypes.data, z.ctypes.data, len(x), len(y),
                              px.ctypes.data, py.ctypes.data, px.size, out.ctypes.data)
    return out


def eig(A):
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    wr, wi = np.zeros(n), np.zeros(n)
    vr = np.zeros((n, n))
    rc = lib().oracle_eig(n, A.ctypes.data, wr.ctypes.data, wi.ctypes.data, vr.ctypes.data)
    return rc, wr + 1j * wi, vr


def landau_cell(T10, tau):
    T10 = np.ascontiguousarray(T10, dtype=np.float32)
    e = np.zeros(1, np.float32)
    u = np.zeros(4, np.float32)
    ok = lib().oracle_landau_cell(T10.ctypes.data, ctypes.c_float(tau), e.ctypes.data,
                                  u.ctypes.data)
    return ok, float(e[0]), u


DIAG_NAMES = ["R_Pi_Inv", "R_pimunu_Inv", "pi_dot_u", "pi_mu_mu", "beta", "omega"]
DIAG_COMPS = {"R_Pi_Inv": 1, "R_pimunu_Inv": 1, "pi_dot_u": 4, "pi_mu_mu": 1, "beta": 4, "omega": 6}


def diagnostics(p, tau, e, P, Pi, u, pi, impl="oracle"):
    """Hydro-validity and vorticity diagnostics (17 x DIM floats) of the
    oracle's restatement or of the reference's own functions."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32).ravel() for a in (e, P, Pi, u, pi)]
    n = arrs[0].size
    out = np.zeros(17 * n, np.float32)
    fn = (lib().oracle_diagnostics if impl == "oracle" else ref().ref_diagnostics)
    fn.argtypes = [ctypes.POINTER(Params), ctypes.c_float] + [ctypes.c_void_p] * 6
    fn.restype = None
    fn(ctypes.byref(p), ctypes.c_float(tau), *[a.ctypes.data for a in arrs], out.ctypes.data)
    return out.reshape(17, n)
