"""Seeded synthetic initial profiles for the freestream-milne workloads.

No dataset is involved: every profile is generated here from a seed, with the
shapes and value distributions of the five workload configurations:

  gaussian2d   smooth Gaussian T^00 = 10 GeV/fm^3 exp(-r^2/(2*1.5^2)), 101^2,
               DX=0.1, DIM_PHIP=51, TAU0=0.1, DTAU=0.5, conformal EoS
  lumpy2d      200 Gaussian hotspots (sigma 0.4 fm, amplitude ~ Exp(mean 5
               GeV/fm^3), centres uniform in a 6 fm disk) on 261^2, DX=0.06,
               DIM_PHIP=200, TAU0=0.2, DTAU=1.0, Wuppertal-Budapest EoS
  baryon3d     lumpy transverse profile x plateau-plus-Gaussian in eta
               (ETA_FLAT=4, ETA_WIDTH=1) on 131^2 x 51 (DX=0.1, DETA=0.2),
               n_B = 0.1 * normalised T^00 with its eta profile shifted by
               +-1.5; DIM_RAP=21 (tan-map nodes), DIM_PHIP=100, TAU0=0.1,
               DTAU=0.8, BARYON=1, SIGMA=SIGMA_B=1
  uneven_batch 512 lumpy 2D events, side in {101,151,201,261,301}, DX in
               [0.05,0.1], DIM_PHIP in {64,100,200}, DTAU in [0.3,1.5],
               conformal or WB EoS 50:50
  stream       Poisson arrivals, 80% 2D (side 101-301) and 20% 3D (C2 shape,
               DIM_ETA in {25,51}, DIM_RAP in {21,31,41})

Grid coordinates follow the reference's float formula
x = ix*DX + xmin, xmin = -((DIM_X-1)/2)*DX (src/FreeStream.cpp:16-31).
"""
import numpy as np

from fsm_params import default_params, derive  # noqa: F401 (derive: re-exported)


def axis(n, d):
    d = np.float32(d)
    lo = np.float32(-1.0 * (np.float32(n - 1) / 2.0) * d)
    return (np.arange(n, dtype=np.float32) * d + lo).astype(np.float32)


def hotspots(rng, x, y, n_spots=200, sigma=0.4, mean_amp=5.0, radius=6.0):
    """Sum of Gaussian hotspots in GeV/fm^3 on the (x, y) grid, shape (NX, NY)."""
    amp = rng.exponential(mean_amp, n_spots)  # Gamma(k=1, theta=mean_amp)
    r = radius * np.sqrt(rng.random(n_spots))
    th = 2 * np.pi * rng.random(n_spots)
    cx, cy = r * np.cos(th), r * np.sin(th)
    inv = 1.0 / (2 * sigma * sigma)
    # separable Gaussians: sum_k a_k gx_k(x) gy_k(y) as one matrix product
    gx = np.exp(-(x.astype(np.float64)[None, :] - cx[:, None]) ** 2 * inv)
    gy = np.exp(-(y.astype(np.float64)[None, :] - cy[:, None]) ** 2 * inv)
    return (gx * amp[:, None]).T @ gy


def plateau(eta, flat, width):
    """exp(-(|eta|-flat)^2/(2 width^2)) for |eta| > flat, 1 inside
    (the eta profile form of src/InitialConditions.cpp:175-176)."""
    a = np.abs(eta) - flat
    return np.exp(-(a ** 2) / (2 * width ** 2) * (a > 0))


def gaussian2d(**over):
    p = default_params(DIM_X=101, DIM_Y=101, DX=0.1, DY=0.1, DIM_ETA=1, DIM_RAP=1, DIM_PHIP=51,
                       TAU0=0.1, DTAU=0.5, EOS_TYPE=1, BARYON=0, VISCOUS_MATCHING=1,
                       E_DEP_FS=0, OUTPUTFORMAT=2)
    for k, v in over.items():
        setattr(p, k, v)
    derive(p)
    x, y = axis(p.DIM_X, p.DX), axis(p.DIM_Y, p.DY)
    X, Y = np.meshgrid(x.astype(np.float64), y.astype(np.float64), indexing="ij")
    e = 10.0 * np.exp(-(X ** 2 + Y ** 2) / (2 * 1.5 ** 2))
    return p, e.astype(np.float32).ravel(), None


def lumpy2d(seed=1, side=261, dx=0.06, nphip=200, tau0=0.2, dtau=1.0, eos=2, radius=6.0, **over):
    rng = np.random.default_rng(seed)
    p = default_params(DIM_X=side, DIM_Y=side, DX=dx, DY=dx, DIM_ETA=1, DIM_RAP=1,
                       DIM_PHIP=nphip, TAU0=tau0, DTAU=dtau, EOS_TYPE=eos, BARYON=0,
                       VISCOUS_MATCHING=1, E_DEP_FS=0, OUTPUTFORMAT=2)
    for k, v in over.items():
        setattr(p, k, v)
    derive(p)
    x, y = axis(p.DIM_X, p.DX), axis(p.DIM_Y, p.DY)
    e = hotspots(rng, x, y, radius=radius)
    return p, e.astype(np.float32).ravel(), None


def lumpy2d_baryon(seed=1, side=101, dx=0.08, nphip=64, dtau=0.8, nrap=5, drap=0.3, sigma_b=0.8,
                   eos=1, radius=3.0, **over):
    """Boost-invariant event with baryon charge: lumpy T^00 and n_B = 0.1 x the
    normalised profile, DIM_RAP uniform rapidity nodes for the charge."""
    p, e, _ = lumpy2d(seed=seed, side=side, dx=dx, nphip=nphip, dtau=dtau, eos=eos, radius=radius,
                      BARYON=1, IC_BARYON=3, DIM_RAP=nrap, DRAP=drap, SIGMA_B=sigma_b, **over)
    nB = (0.1 * e / max(float(e.max()), 1e-30)).astype(np.float32)
    return p, e, nB


def baryon3d(seed=2, side=131, dx=0.1, neta=51, deta=0.2, nrap=21, nphip=100, tau0=0.1,
             dtau=0.8, eta_flat=4.0, eta_width=1.0, **over):
    rng = np.random.default_rng(seed)
    p = default_params(DIM_X=side, DIM_Y=side, DX=dx, DY=dx, DIM_ETA=neta, DETA=deta,
                       DIM_RAP=nrap, DRAP=0.2, DIM_PHIP=nphip, TAU0=tau0, DTAU=dtau,
                       EOS_TYPE=1, BARYON=1, IC_BARYON=3, SIGMA=1.0, SIGMA_B=1.0,
                       ETA_FLAT=eta_flat, ETA_WIDTH=eta_width, VISCOUS_MATCHING=1,
                       E_DEP_FS=0, OUTPUTFORMAT=2)
    for k, v in over.items():
        setattr(p, k, v)
    derive(p)
    x, y, eta = axis(p.DIM_X, p.DX), axis(p.DIM_Y, p.DY), axis(p.DIM_ETA, p.DETA)
    radius = min(6.0, 0.45 * side * dx)
    tp = hotspots(rng, x, y, radius=radius)
    H = plateau(eta.astype(np.float64), eta_flat, eta_width)
    e = tp[:, :, None] * H[None, None, :]
    Hb = 0.5 * (plateau(eta - 1.5, eta_flat, eta_width) + plateau(eta + 1.5, eta_flat, eta_width))
    nB = 0.1 * (tp / tp.max())[:, :, None] * Hb[None, None, :]
    return p, e.astype(np.float32).ravel(), nB.astype(np.float32).ravel()


def uneven_batch(n=512, seed=3):
    """Event list of the batched configuration: [(params, e_gev, None)]."""
    rng = np.random.default_rng(seed)
    events = []
    for k in range(n):
        side = int(rng.choice([101, 151, 201, 261, 301]))
        dx = float(np.float32(rng.uniform(0.05, 0.1)))
        nphip = int(rng.choice([64, 100, 200]))
        dtau = float(np.float32(rng.uniform(0.3, 1.5)))
        eos = 1 if rng.random() < 0.5 else 2
        half = 0.5 * (side - 1) * dx
        radius = min(6.0, 0.6 * half)
        events.append(lumpy2d(seed=int(rng.integers(1 << 30)), side=side, dx=dx, nphip=nphip,
                              tau0=0.2, dtau=dtau, eos=eos, radius=radius))
    return events


def stream_requests(n, rate_hz, seed=4, frac3d=0.2, small3d=False):
    """Poisson request stream: list of (arrival_s, (params, e, nB))."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate_hz)
        if rng.random() < frac3d:
            neta = int(rng.choice([25, 51]))
            nrap = int(rng.choice([21, 31, 41]))
            side = 131 if not small3d else 41
            ev = baryon3d(seed=int(rng.integers(1 << 30)), side=side, neta=neta, nrap=nrap,
                          deta=0.2 * 51 / neta if neta != 51 else 0.2)
        else:
            side = int(rng.choice([101, 151, 201, 261, 301]))
            dx = float(np.float32(rng.uniform(0.05, 0.1)))
            ev = lumpy2d(seed=int(rng.integers(1 << 30)), side=side, dx=dx,
                         nphip=int(rng.choice([64, 100, 200])),
                         dtau=float(np.float32(rng.uniform(0.3, 1.5))),
                         eos=1 if rng.random() < 0.5 else 2,
                         radius=min(6.0, 0.3 * (side - 1) * dx))
        out.append((t, ev))
    return out
