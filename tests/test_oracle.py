"""CPU tests of the oracle: pinned against the reference's own sources (golden
fixtures and, where the reference checkout exists, a live build), and against
independent numerics (scipy, numpy) and closed-form free-streaming results."""
import numpy as np
import pytest

import oracle_py as O
from fsm_testutil import golden_names, load_golden, oracle_params

FIELDS = ["T", "J", "e", "P", "Pi", "u", "pi", "nB", "V"]


@pytest.mark.parametrize("name", golden_names())
def test_oracle_bit_exact_against_reference_fixture(name):
    """The float restatement reproduces the reference pipeline bit for bit."""
    d, e, nB, ref, meta = load_golden(name)
    r = O.run(oracle_params(d), e, nB=nB)
    assert r["dim_phip"] == int(meta[0])
    for k in FIELDS:
        if k in ref:
            assert np.array_equal(r[k].astype(np.float32), ref[k]), k


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("seed", [11, 12])
def test_oracle_matches_live_reference_build(seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(20, 40)), int(rng.integers(20, 40))
    p = O.make_params(DIM_X=nx, DIM_Y=ny, DX=float(rng.uniform(0.05, 0.15)),
                      DY=float(rng.uniform(0.05, 0.15)), DIM_PHIP=int(rng.integers(8, 60)),
                      TAU0=0.2, DTAU=float(rng.uniform(0.1, 1.2)), EOS_TYPE=int(rng.integers(1, 4)),
                      VISCOUS_MATCHING=int(rng.integers(0, 2)))
    e = (rng.random(nx * ny) * 5).astype(np.float32)
    a = O.run(p, e, impl="oracle")
    b = O.run(p, e, impl="ref")
    for k in ["T", "e", "P", "Pi", "u", "pi"]:
        assert np.array_equal(a[k], b[k]), k


def test_natural_spline_derivatives_match_scipy():
    from scipy.interpolate import CubicSpline
    rng = np.random.default_rng(0)
    for n in (4, 5, 17, 101):
        x = np.cumsum(rng.uniform(0.5, 1.5, n))
        y = rng.normal(size=n)
        d = O.spline_derivs(x, y)
        ref = CubicSpline(x, y, bc_type="natural")(x, 1)
        assert np.allclose(d, ref, rtol=1e-12, atol=1e-12)


def test_bicubic_reproduces_linear_and_converges():
    x = np.linspace(-2, 2, 21)
    y = np.linspace(-1.5, 1.5, 17)
    X, Y = np.meshgrid(x, y, indexing="xy")  # z[j, i] = f(x[i], y[j])
    lin = 0.3 + 1.7 * X - 0.4 * Y + 0.25 * X * Y
    rng = np.random.default_rng(1)
    px, py = rng.uniform(-1.99, 1.99, 500), rng.uniform(-1.49, 1.49, 500)
    got = O.bicubic_eval(x, y, lin, px, py)
    assert np.allclose(got, 0.3 + 1.7 * px - 0.4 * py + 0.25 * px * py, atol=1e-12)
    f = lambda a, b: np.exp(-(a ** 2 + b ** 2))
    got = O.bicubic_eval(x, y, f(X, Y), px, py)
    assert np.max(np.abs(got - f(px, py))) < 2e-3


def test_eigensolver_matches_numpy():
    rng = np.random.default_rng(2)
    for _ in range(200):
        n = int(rng.integers(2, 5))
        A = rng.normal(size=(n, n))
        rc, w, V = O.eig(A)
        assert rc == 0
        ref = np.linalg.eigvals(A)
        assert np.allclose(np.sort_complex(w), np.sort_complex(ref), atol=1e-9)
        for k in range(n):
            if w[k].imag == 0:
                v = V[:, k]
                assert abs(np.linalg.norm(v) - 1) < 1e-12
                assert np.allclose(A @ v, w[k].real * v, atol=1e-8)


def _axis(n, d):
    d = np.float32(d)
    lo = np.float32(-1.0 * (np.float32(n - 1) / 2.0) * d)
    return np.arange(n, dtype=np.float32) * d + lo


def test_known_answer_2d_gaussian_free_streaming():
    """Boost-invariant free streaming of e0 exp(-r^2/2R^2) with the reference's
    normalisation (F = e/2pi, T = sum F p p dphi / tau) gives
    T^tt = (e0/tau) exp(-(r^2+D^2)/2R^2) I0(rD/R^2) and
    T^tr = (e0/tau) exp(-(r^2+D^2)/2R^2) I1(rD/R^2), D = DTAU."""
    from scipy.special import i0e, i1e
    n, dx, R, D, tau0 = 121, 0.1, 1.5, 0.5, 0.1
    p = O.make_params(DIM_X=n, DIM_Y=n, DX=dx, DY=dx, DIM_PHIP=400, TAU0=tau0, DTAU=D)
    x = _axis(n, dx).astype(np.float64)
    X, Y = np.meshgrid(x, x, indexing="ij")
    e_gev = 10.0 * np.exp(-(X ** 2 + Y ** 2) / (2 * R * R))
    r = O.run(p, e_gev.astype(np.float32).ravel(), fp64=True)
    e0 = 10.0 / 0.197326938
    tau = tau0 + D
    rr = np.sqrt(X ** 2 + Y ** 2).ravel()
    z = rr * D / R ** 2
    env = (e0 / tau) * np.exp(-(rr ** 2 + D ** 2) / (2 * R * R) + z)
    ttt = env * i0e(z) + 1e-7 / tau  # plus the 1e-7 fm^-4 floor of the input conversion
    inner = rr < 3.0
    assert np.max(np.abs(r["T"][0][inner] / ttt[inner] - 1)) < 2e-4
    ttr = env * i1e(z)
    tr = (r["T"][1] * X.ravel() + r["T"][2] * Y.ravel()) / np.maximum(rr, 1e-12)
    sel = inner & (rr > 0.5)
    assert np.max(np.abs(tr[sel] - ttr[sel]) / ttt[sel]) < 2e-4


def test_2d_conformal_trace_and_energy():
    """2D free streaming of massless particles is traceless in (tau, x, y), so the
    conformal bulk pressure vanishes; tau * T^tt integrates to the initial energy
    while the profile stays inside the grid (src/FreestreamMilne.cpp:349-354,531-535)."""
    n, dx = 81, 0.1
    p = O.make_params(DIM_X=n, DIM_Y=n, DX=dx, DY=dx, DIM_PHIP=64, TAU0=0.2, DTAU=0.8)
    x = _axis(n, dx).astype(np.float64)
    X, Y = np.meshgrid(x, x, indexing="ij")
    e = (8 * np.exp(-((X - 0.4) ** 2 + (Y + 0.3) ** 2) / 0.8)).astype(np.float32).ravel()
    r = O.run(p, e, fp64=True)
    T = r["T"]
    m = r["e"] > 1e-3 * r["e"].max()
    assert np.max(np.abs(T[0] - T[4] - T[7])[m] / T[0][m]) < 1e-12
    assert np.max(np.abs(r["Pi"][m]) / r["e"][m]) < 1e-10
    e_fm = e / 0.197326938 + 1e-7
    before = e_fm.sum() * dx * dx
    after = r["tau"] * T[0].sum() * dx * dx
    assert abs(after / before - 1) < 2e-3


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("name", ["lumpy2d_wb_61x53", "baryon3d_25x23x15"])
def test_diagnostics_match_reference(name):
    """The diagnostics restatement (hydro validity, thermal vorticity) against
    the reference's own functions on the reference's Landau-matched fields:
    bit for bit."""
    d, e, nB, ref, meta = load_golden(name)
    p = oracle_params(d)
    p.DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA
    args = (p, float(np.float32(meta[2])), ref["e"], ref["P"], ref["Pi"], ref["u"], ref["pi"])
    a = O.diagnostics(*args, impl="oracle")
    b = O.diagnostics(*args, impl="ref")
    np.testing.assert_array_equal(a, b)
    assert np.isfinite(a).all() and np.abs(a[1]).max() > 0
