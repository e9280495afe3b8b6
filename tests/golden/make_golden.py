"""Generates the golden fixtures in tests/golden/ from the reference's own sources.

Run from the repository root in a checkout where the reference is available:

    make -C oracle            # builds oracle/_ref/libfsm_ref.so from <reference>/src
    python tests/golden/make_golden.py [fixture names]

Each fixture holds a seeded synthetic input, its parameters and the outputs of
the reference pipeline (src/FreestreamMilne.cpp:251-506) compiled from the
reference sources against the project's GSL-API stand-in.  Inputs are
synthetic (no dataset); outputs are stored as float32, exactly the reference's
float results.  The `full_*` fixture runs the reference's public entry point
FREESTREAMMILNE::run_freestream_milne (with a freestream_input file) and stores
its 17 output vectors and two of its text output files.
"""
import os
import pathlib
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle_py as O  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent


def axis(n, d):
    d = np.float32(d)
    lo = np.float32(-1.0 * (np.float32(n - 1) / 2.0) * d)
    return np.arange(n, dtype=np.float32) * d + lo


def hotspots(rng, x, y, n=40, sigma=0.4, amp=5.0, radius=2.0):
    a = rng.exponential(amp, n)
    r = radius * np.sqrt(rng.random(n))
    t = 2 * np.pi * rng.random(n)
    X = x.astype(np.float64)[:, None]
    Y = y.astype(np.float64)[None, :]
    out = np.zeros((x.size, y.size))
    for k in range(n):
        out += a[k] * np.exp(-((X - r[k] * np.cos(t[k])) ** 2 + (Y - r[k] * np.sin(t[k])) ** 2)
                             / (2 * sigma * sigma))
    return out


def cases():
    rng = np.random.default_rng(20261203)
    cs = []
    # 2D smooth Gaussian (the CPU-runnable configuration, grid reduced)
    p = O.make_params(DIM_X=41, DIM_Y=41, DX=0.1, DY=0.1, DIM_PHIP=51, TAU0=0.1, DTAU=0.5,
                      EOS_TYPE=1)
    x, y = axis(41, 0.1), axis(41, 0.1)
    X, Y = np.meshgrid(x.astype(np.float64), y.astype(np.float64), indexing="ij")
    e = (10 * np.exp(-(X ** 2 + Y ** 2) / (2 * 1.0 ** 2))).astype(np.float32)
    cs.append(("gauss2d_41", p, e, None))
    # 2D lumpy event, Wuppertal-Budapest EoS, axis-aligned shifts land on nodes
    p = O.make_params(DIM_X=61, DIM_Y=53, DX=0.1, DY=0.1, DIM_PHIP=64, TAU0=0.2, DTAU=1.0,
                      EOS_TYPE=2)
    x, y = axis(61, 0.1), axis(53, 0.1)
    e = hotspots(rng, x, y).astype(np.float32)
    cs.append(("lumpy2d_wb_61x53", p, e, None))
    # 2D lumpy, anisotropic spacing, phi_p raised by the arc-length rule
    p = O.make_params(DIM_X=48, DIM_Y=57, DX=0.07, DY=0.09, DIM_PHIP=20, TAU0=0.3, DTAU=0.9,
                      EOS_TYPE=1, DIM_RAP=3)
    x, y = axis(48, 0.07), axis(57, 0.09)
    e = hotspots(rng, x, y, radius=1.2, sigma=0.3).astype(np.float32)
    cs.append(("lumpy2d_aniso_48x57_rap3", p, e, None))
    # 2D with the energy-dependent free-streaming time
    p = O.make_params(DIM_X=45, DIM_Y=45, DX=0.1, DY=0.1, DIM_PHIP=40, TAU0=0.1, DTAU=0.5,
                      EOS_TYPE=1, E_DEP_FS=1, E_R=4.0, TAU_R=0.6, ALPHA=0.25)
    x, y = axis(45, 0.1), axis(45, 0.1)
    e = hotspots(rng, x, y, radius=1.5).astype(np.float32)
    cs.append(("edepfs2d_45", p, e, None))
    # 3D with baryon charge (tan-map rapidity nodes)
    p = O.make_params(DIM_X=25, DIM_Y=23, DIM_ETA=15, DX=0.15, DY=0.15, DETA=0.25, DIM_RAP=9,
                      DIM_PHIP=24, TAU0=0.2, DTAU=0.6, EOS_TYPE=1, BARYON=1, IC_BARYON=3,
                      SIGMA=1.0, SIGMA_B=1.0, DRAP=0.2)
    x, y, eta = axis(25, 0.15), axis(23, 0.15), axis(15, 0.25)
    tp = hotspots(rng, x, y, n=20, radius=1.2)
    a = np.abs(eta.astype(np.float64)) - 1.0
    H = np.exp(-(a ** 2) / 2 * (a > 0))
    e = (tp[:, :, None] * H[None, None, :]).astype(np.float32)
    Hb = np.exp(-((eta.astype(np.float64) - 0.5) ** 2) / 2)
    nB = (0.1 * (tp / tp.max())[:, :, None] * Hb[None, None, :]).astype(np.float32)
    cs.append(("baryon3d_25x23x15", p, e, nB))
    # 3D Wuppertal-Budapest EoS without baryons, wider rapidity grid
    p = O.make_params(DIM_X=21, DIM_Y=21, DIM_ETA=11, DX=0.2, DY=0.2, DETA=0.3, DIM_RAP=13,
                      DIM_PHIP=16, TAU0=0.3, DTAU=0.5, EOS_TYPE=2, SIGMA=0.8)
    x, y, eta = axis(21, 0.2), axis(21, 0.2), axis(11, 0.3)
    tp = hotspots(rng, x, y, n=15, radius=1.5)
    e = (tp[:, :, None] * np.exp(-eta.astype(np.float64) ** 2 / 4)[None, None, :]).astype(np.float32)
    cs.append(("wb3d_21x21x11", p, e, None))
    # 2D with baryon charge: five uniform rapidity nodes for the charge density
    p = O.make_params(DIM_X=45, DIM_Y=41, DX=0.1, DY=0.1, DIM_PHIP=40, TAU0=0.2, DTAU=0.7,
                      EOS_TYPE=1, BARYON=1, IC_BARYON=3, DIM_RAP=5, DRAP=0.3, SIGMA_B=0.8)
    x, y = axis(45, 0.1), axis(41, 0.1)
    tp = hotspots(rng, x, y, n=20, radius=1.4)
    e = tp.astype(np.float32)
    nB = (0.1 * tp / tp.max()).astype(np.float32)
    cs.append(("baryon2d_45x41_rap5", p, e, nB))
    return cs


FIELDS = ["T", "J", "e", "P", "Pi", "u", "pi", "nB", "V"]


def params_dict(p):
    return {k: getattr(p, k) for k, _ in O.PARAM_FIELDS}


def main(only=None):
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libfsm_ref.so missing: build it with `make -C oracle`")
    for name, p, e, nB in cases():
        if only and name not in only:
            continue
        r = O.run(p, e.ravel(), nB=None if nB is None else nB.ravel(), impl="ref")
        arrays = {"e_gev": e.ravel().astype(np.float32)}
        if nB is not None:
            arrays["nB_in"] = nB.ravel().astype(np.float32)
        for k in FIELDS:
            if k in r:
                arrays["out_" + k] = r[k].astype(np.float32)
        pd = params_dict(p)
        arrays["params_int"] = np.array([pd[k] for k, t in O.PARAM_FIELDS if t is O.ctypes.c_int],
                                        dtype=np.int64)
        arrays["params_float"] = np.array([pd[k] for k, t in O.PARAM_FIELDS
                                           if t is O.ctypes.c_float], dtype=np.float32)
        arrays["meta"] = np.array([r["dim_phip"], r["dtau"], r["tau"], r["n_fallback"]],
                                  dtype=np.float64)
        np.savez_compressed(OUT / f"{name}.npz", **arrays)
        print(name, "cells", e.size, "phi_p", r["dim_phip"], "fallback", r["n_fallback"])
    # the public entry point end to end, with its parameter file
    if not only or "full_entry_31x29" in only:
        full_case()


FULL_INPUT = """OUTPUTFORMAT 2
BARYON 0
IC_ENERGY 5
IC_BARYON 1
ETA_WIDTH 0.5
ETA_FLAT 0.5
SIGMA 1.0
SIGMA_B 1.0
DIM_X 31
DIM_Y 29
DIM_ETA 1
DIM_RAP 1
DIM_PHIP 40
DX 0.12
DY 0.12
DETA 0.1
DRAP 0.2
DTAU 0.6
TAU0 0.2
EOS_TYPE 2
E_FREEZE 1.7
VISCOUS_MATCHING 1
E_DEP_FS 0
E_R 1.0
TAU_R 1.0
ALPHA 0.0
"""


def full_case():
    rng = np.random.default_rng(7)
    x, y = axis(31, 0.12), axis(29, 0.12)
    e = hotspots(rng, x, y, n=12, radius=1.0).astype(np.float32).ravel()
    with tempfile.TemporaryDirectory() as d:
        pathlib.Path(d, "freestream_input").write_text(FULL_INPUT)
        os.mkdir(os.path.join(d, "output"))
        out = np.zeros(17 * e.size)
        O.ref().ref_run_full(d.encode(), e.ctypes.data, e.size, out.ctypes.data)
        files = {}
        for fn in ("e.dat", "ux.dat", "e_projection.dat", "pixy.dat"):
            files[fn] = pathlib.Path(d, "output", fn).read_text()
    np.savez_compressed(OUT / "full_entry_31x29.npz", e_gev=e, vectors=out.reshape(17, e.size),
                        freestream_input=np.array(FULL_INPUT),
                        **{"file_" + k.replace(".", "_"): np.array(v) for k, v in files.items()})
    print("full_entry_31x29 written")


if __name__ == "__main__":
    main(set(sys.argv[1:]) or None)  # optional fixture names: regenerate only those
