"""Shared helpers for the parity tests: fixtures, parameter conversion and the
tolerance checks (each tolerance is stated where it is checked)."""
import ctypes
import pathlib

import numpy as np

import oracle_py as O

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

# Parity tolerances against the reference's float path (and the FP64 oracle):
#   T^{mu nu}, J^mu : 1e-5, relative to the cell's T^{tau tau} (J^tau for J)
#   e               : 1e-4 relative against the FP64 precision oracle; against
#                     the reference's float output 1e-4 of the cell's T^{tau tau}
#                     (the Landau eigenvalue amplifies the float rounding of T by
#                     ~gamma^2 in boosted cells, and the reference's own float e
#                     is up to ~1e-4 relative away from FP64 there)
#   u^mu            : 1e-4, relative to u^tau
#   Pi, pi^{mu nu}  : 1e-4, relative to the cell's T^{tau tau} (norm-wise: pi is
#                     T minus its ideal part, so in a cell boosted to gamma its
#                     components carry errors of e and u amplified by gamma^2)
#   n_B, V^mu       : 1e-4, relative to the cell's |J^tau|
# evaluated in cells with e > 1e-6 * max e and T^{tau tau} > 1e-6 * max T^{tau tau}.  Components with eta indices are
# scaled by tau per eta index so that all components share the units of
# T^{tau tau} (u^eta -> tau u^eta, T^{tau eta} -> tau T^{tau eta}, ...).
TOL_T = 1e-5
TOL_E = 1e-4
TOL_U = 1e-4
TOL_VISC = 1e-4
TOL_B = 1e-4
ETA_POW_T = np.array([0, 0, 0, 1, 0, 0, 1, 0, 1, 2])  # eta indices per T / pi component
ETA_POW_V = np.array([0, 0, 0, 1])


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith("full_"))


def load_golden(name):
    z = np.load(GOLDEN / f"{name}.npz")
    ints = [k for k, t in O.PARAM_FIELDS if t is ctypes.c_int]
    flts = [k for k, t in O.PARAM_FIELDS if t is ctypes.c_float]
    d = {}
    for k, v in zip(ints, z["params_int"]):
        d[k] = int(v)
    for k, v in zip(flts, z["params_float"]):
        d[k] = float(v)
    out = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    nB = z["nB_in"] if "nB_in" in z.files else None
    meta = z["meta"]
    return d, z["e_gev"], nB, out, meta


def oracle_params(d):
    p = O.Params(**d)
    return p


def fsm_params(d):
    import fsm_b200 as F
    p = F.Params(**d)
    F.lib().fsm_params_derive(ctypes.byref(p))
    return p


def mask_of(ref):
    """Cells with e > 1e-6 max e and a non-empty moment sum (cells that no
    momentum sample reaches keep T = 0 and take the Landau fallback e = 1e-3)."""
    e = np.asarray(ref["e"], dtype=np.float64)
    ttt = np.asarray(ref["T"], dtype=np.float64)[0]
    return (e > 1e-6 * e.max()) & (ttt > 1e-6 * ttt.max())


def scale_eta(a, pow_, tau):
    a = np.asarray(a, dtype=np.float64)
    return a * (float(tau) ** pow_)[:, None]


def compare(got, ref, tau, what=("T", "e", "u", "Pi", "pi"), baryon=False, tolT=TOL_T,
            e_normwise=False):
    """Returns {name: worst scaled error} and raises AssertionError on failure.
    e_normwise: measure e against T^{tau tau} (for comparisons with the
    reference's float output) instead of relative to e (FP64 oracle)."""
    m = mask_of(ref)
    errs = {}
    Tref = np.asarray(ref["T"], np.float64)
    ttt = Tref[0][m]
    if "T" in what:
        d = np.abs(scale_eta(got["T"], ETA_POW_T, tau) - scale_eta(Tref, ETA_POW_T, tau))[:, m]
        errs["T"] = float(np.max(d / ttt))
    if "e" in what:
        e_r = np.asarray(ref["e"], np.float64)[m]
        den = ttt if e_normwise else e_r
        errs["e"] = float(np.max(np.abs(np.asarray(got["e"], np.float64)[m] - e_r) / den))
    if "u" in what:
        ur = scale_eta(ref["u"], ETA_POW_V, tau)[:, m]
        ug = scale_eta(got["u"], ETA_POW_V, tau)[:, m]
        errs["u"] = float(np.max(np.abs(ug - ur) / ur[0]))
    ep = ttt
    if "Pi" in what:
        errs["Pi"] = float(np.max(np.abs(np.asarray(got["Pi"], np.float64)[m] -
                                         np.asarray(ref["Pi"], np.float64)[m]) / ep))
    if "pi" in what:
        d = np.abs(scale_eta(got["pi"], ETA_POW_T, tau) - scale_eta(ref["pi"], ETA_POW_T, tau))[:, m]
        errs["pi"] = float(np.max(d / ep))
    if baryon:
        Jr = np.asarray(ref["J"], np.float64)
        jt = np.abs(Jr[0][m])
        jm = jt > 1e-6 * jt.max()
        dJ = np.abs(scale_eta(got["J"], ETA_POW_V, tau) - scale_eta(Jr, ETA_POW_V, tau))[:, m]
        errs["J"] = float(np.max(dJ[:, jm] / jt[jm]))
        dn = np.abs(np.asarray(got["nB"], np.float64)[m] - np.asarray(ref["nB"], np.float64)[m])
        errs["nB"] = float(np.max(dn[jm] / jt[jm]))
        dV = np.abs(scale_eta(got["V"], ETA_POW_V, tau) - scale_eta(ref["V"], ETA_POW_V, tau))[:, m]
        errs["V"] = float(np.max(dV[:, jm] / jt[jm]))
    limits = dict(T=tolT, e=TOL_E, u=TOL_U, Pi=TOL_VISC, pi=TOL_VISC, J=tolT, nB=TOL_B, V=TOL_B)
    bad = {k: v for k, v in errs.items() if not v <= limits[k]}
    assert not bad, f"tolerance exceeded: {bad} (all: {errs})"
    return errs


def _per_cell_errors(got, ref, tau, m, ttt, baryon):
    """Per-cell scaled errors (same scales as compare(), e norm-wise), as
    {name: array over masked cells}."""
    out = {}
    Tref = np.asarray(ref["T"], np.float64)
    out["T"] = np.max(np.abs(scale_eta(got["T"], ETA_POW_T, tau) -
                             scale_eta(Tref, ETA_POW_T, tau))[:, m], axis=0) / ttt
    out["e"] = np.abs(np.asarray(got["e"], np.float64)[m] - np.asarray(ref["e"], np.float64)[m]) / ttt
    ur = scale_eta(ref["u"], ETA_POW_V, tau)[:, m]
    out["u"] = np.max(np.abs(scale_eta(got["u"], ETA_POW_V, tau)[:, m] - ur), axis=0) / ur[0]
    out["Pi"] = np.abs(np.asarray(got["Pi"], np.float64)[m] - np.asarray(ref["Pi"], np.float64)[m]) / ttt
    out["pi"] = np.max(np.abs(scale_eta(got["pi"], ETA_POW_T, tau) -
                              scale_eta(ref["pi"], ETA_POW_T, tau))[:, m], axis=0) / ttt
    if baryon:
        jt = np.maximum(np.abs(np.asarray(ref["J"], np.float64)[0][m]), 1e-300)
        out["J"] = np.max(np.abs(scale_eta(got["J"], ETA_POW_V, tau) -
                                 scale_eta(ref["J"], ETA_POW_V, tau))[:, m], axis=0) / jt
        out["nB"] = np.abs(np.asarray(got["nB"], np.float64)[m] - np.asarray(ref["nB"], np.float64)[m]) / jt
        out["V"] = np.max(np.abs(scale_eta(got["V"], ETA_POW_V, tau) -
                                 scale_eta(ref["V"], ETA_POW_V, tau))[:, m], axis=0) / jt
    return out


# Landau-matched quantities of cells whose T^{mu nu} is nearly light-like
# (e << T^{tau tau}: streaming-dominated fringes of the profile) amplify the
# FP32 rounding of the moments by ~(T^{tau tau}/e)^2; there neither FP32 path
# (the reference's nor this one) can hold 1e-4 on u and pi against FP64.
# Such cells, outside the tolerance of both the reference's float output and
# FP64, are allowed at a fraction RESIDUAL_FRAC of the masked cells at most,
# each within RESIDUAL_FACTOR x the tolerance of FP64 and no further from FP64
# than the reference's own float output is anywhere on the same event.
RESIDUAL_FRAC = 1e-3
RESIDUAL_FACTOR = 2.0


def compare_parity(got, ref_float, ref64, tau, baryon=False):
    """Parity with the reference's float output, per cell and quantity: the GPU
    result is within the tolerance of the reference's value, or -- in a cell
    where the reference's own float value is more than a quarter of the
    tolerance away from the FP64 precision oracle (its rounding noise,
    amplified in the Landau-matched quantities of boosted or nearly light-like
    cells) -- within the tolerance of the FP64 value ("rescued").  Cells that
    pass neither are the bounded residual described above.  The strict
    contract, every masked cell within tolerance of FP64 (e relative to e), is
    compare(got, ref64, ...), run beside this check for T, e, Pi.
    Returns ({name: worst error vs reference}, {name: rescued cells},
    {name: masked cells}, {name: (residual cells, worst residual vs FP64)})."""
    m = mask_of(ref64)
    ttt = np.asarray(ref64["T"], np.float64)[0][m]
    if baryon:
        jt = np.abs(np.asarray(ref64["J"], np.float64)[0][m])
        keep = jt > 1e-6 * jt.max()
    g_ref = _per_cell_errors(got, ref_float, tau, m, ttt, baryon)
    g_64 = _per_cell_errors(got, ref64, tau, m, ttt, baryon)
    r_64 = _per_cell_errors(ref_float, ref64, tau, m, ttt, baryon)
    limits = dict(T=TOL_T, e=TOL_E, u=TOL_U, Pi=TOL_VISC, pi=TOL_VISC, J=TOL_T, nB=TOL_B, V=TOL_B)
    worst, rescued, cells, residual, bad = {}, {}, {}, {}, {}
    for k, a in g_ref.items():
        sel = keep if k in ("J", "nB", "V") else np.ones(a.size, bool)
        a, b, c = a[sel], g_64[k][sel], r_64[k][sel]
        lim = limits[k]
        over = a > lim
        ok_by_64 = (b <= lim) & (c > 0.25 * lim)
        worst[k] = float(a.max()) if a.size else 0.0
        rescued[k] = int(np.count_nonzero(over & ok_by_64))
        cells[k] = int(a.size)
        rest = over & ~ok_by_64
        nres = int(np.count_nonzero(rest))
        wres = float(b[rest].max()) if nres else 0.0
        residual[k] = (nres, wres)
        if nres:
            cap = min(RESIDUAL_FACTOR * lim, float(c.max()))
            if k in ("T", "e", "Pi", "J", "nB") or nres > RESIDUAL_FRAC * a.size or wres > cap:
                bad[k] = (nres, wres, cap)
    assert not bad, f"parity violated: {bad} (worst vs reference {worst})"
    return worst, rescued, cells, residual
