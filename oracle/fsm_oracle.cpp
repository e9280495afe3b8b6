// fsm_oracle.cpp -- TEST INFRASTRUCTURE: CPU restatement of the freestream-milne
// reference hot path.  Only tests/, the smoke check and bench.py's CPU-baseline
// leg may load it; the product never does.
//
// Each function names the reference lines it follows.  The loops of the
// reference are fused per cell (the reference's ten passes of
// calculateStressTensor each accumulate one component in (irap, iphip) order;
// interleaving the components per cell keeps every component's order, so the
// float sums are unchanged) and no momentum-resolved array is stored.
//
// Template parameters: R is the value type (interpolation, weights, sums,
// Landau matching) and FG selects float geometry.  <float, *> reproduces the
// reference's float/double mixing operation by operation; <double, false> runs
// the whole algorithm in FP64; <double, true> keeps the reference's float
// geometry (sample angles, shifted positions, index floors and therefore the
// set of in-grid samples) and does every value computation in FP64 -- the
// precision oracle for the float paths, which would otherwise be dominated by
// samples that land exactly on the grid boundary and flip in or out with the
// rounding of their position.
#include "fsm_oracle.h"

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fsm_numerics.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// The profile passed to oracle_run is already in fm^-4 (oracle_run_fm4).
static thread_local bool g_raw_input = false;

// hbar*c as the reference stores it: `float hbarc = 0.197326938;`
// (src/FreestreamMilne.cpp:141)
const float kHbarcF = 0.197326938f;

template <class R>
struct Grid {
  int DIM_X, DIM_Y, DIM_ETA, DIM_RAP, DIM_PHIP, DIM;
  R DX, DY, DETA, DRAP, DTAU, TAU0, TAU;
  R xmin, ymin, etamin;
};

// (src/FreeStream.cpp:113-115)
template <class R>
Grid<R> make_grid(const oracle_params& p) {
  Grid<R> g;
  g.DIM_X = p.DIM_X;
  g.DIM_Y = p.DIM_Y;
  g.DIM_ETA = p.DIM_ETA;
  g.DIM_RAP = p.DIM_RAP;
  g.DIM_PHIP = p.DIM_PHIP;
  g.DIM = p.DIM;
  g.DX = p.DX;
  g.DY = p.DY;
  g.DETA = p.DETA;
  g.DRAP = p.DRAP;
  g.DTAU = p.DTAU;
  g.TAU0 = p.TAU0;
  g.TAU = p.TAU;
  g.xmin = (R)((-1.0) * ((R)(g.DIM_X - 1) / 2.0) * g.DX);
  g.ymin = (R)((-1.0) * ((R)(g.DIM_Y - 1) / 2.0) * g.DY);
  g.etamin = (R)((-1.0) * ((R)(g.DIM_ETA - 1) / 2.0) * g.DETA);
  return g;
}

// tan-map rapidity node (src/FreeStream.cpp:174, LandauMatch.cpp:40,92)
template <class R>
R tanmap_w(int irap, int DIM_RAP) {
  return (R)(-.9975 + (R)irap * (1.995 / (R)(DIM_RAP - 1)));
}

// phi_p node (src/FreeStream.cpp:179, LandauMatch.cpp:32)
template <class R>
R phip_of(int iphip, int DIM_PHIP) {
  return (R)(R(iphip) * (2.0 * M_PI) / R(DIM_PHIP));
}

// (src/FreeStream.cpp:84-94)
template <class R>
R lin2(R x0, R x1, R a00, R a10, R a01, R a11) {
  R result = ((1 - x0) * (1 - x1) * a00) + ((x0) * (1 - x1) * a10) + ((1 - x0) * (x1) * a01) +
             ((x0) * (x1) * a11);
  return result;
}

// (src/FreeStream.cpp:67-82)
template <class R>
R lin3(R x0, R x1, R x2, R a000, R a100, R a010, R a001, R a110, R a101, R a011, R a111) {
  R result = ((1 - x0) * (1 - x1) * (1 - x2) * a000) + ((x0) * (1 - x1) * (1 - x2) * a100) +
             ((1 - x0) * (x1) * (1 - x2) * a010) + ((1 - x0) * (1 - x1) * (x2) * a001) +
             ((x0) * (x1) * (1 - x2) * a110) + ((x0) * (1 - x1) * (x2) * a101) +
             ((1 - x0) * (x1) * (x2) * a011) + ((x0) * (x1) * (x2) * a111);
  return result;
}

// Landau matching of one cell (src/LandauMatch.cpp:173-291).  Tm holds the ten
// components in the reference's row order; returns 1 if accepted.
template <class R>
int landau_cell(const R* Tm, R TAU, R* e_out, R* u_out) {
  double M[16];
  const int idx[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      double g = (c == 0) ? 1.0 : (c == 3 ? -1.0 * TAU * TAU : -1.0);
      M[r * 4 + c] = (double)Tm[idx[r][c]] * g;
    }
  double wr[4], wi[4], vr[16];
  fsm_num::eig_nonsym(4, M, wr, wi, vr);
  const R gamma_max = 100.0;
  int exists = 0;
  for (int i = 0; i < 4; ++i) {
    double re = wr[i], im = wi[i];
    if (re > 0.0 && std::fabs(im) < (std::fabs(re) * 1.0e-30)) {
      double v0 = vr[0 * 4 + i], v1 = vr[1 * 4 + i], v2 = vr[2 * 4 + i], v3 = vr[3 * 4 + i];
      if ((2.0 * v0 * v0 - 1.0 - (v3 * v3 * (TAU * TAU - 1.0))) > 0) {
        double mink = v0 * v0 - (v1 * v1 + v2 * v2 + TAU * TAU * v3 * v3);
        double factor = 1.0 / std::sqrt(mink);
        if (v0 < 0) factor = -factor;
        if ((v0 * factor) < gamma_max) {
          exists = 1;
          *e_out = (R)re;
          u_out[0] = (R)(v0 * factor);
          u_out[1] = (R)(v1 * factor);
          u_out[2] = (R)(v2 * factor);
          u_out[3] = (R)(v3 * factor);
        }
      }
    }
  }
  if (!exists) {  // (src/LandauMatch.cpp:283-291)
    *e_out = (R)1.0e-3;
    u_out[0] = 1.0;
    u_out[1] = 0.0;
    u_out[2] = 0.0;
    u_out[3] = 0.0;
  }
  return exists;
}

// Equation of state (src/EquationOfState.cpp:5-80)
template <class R>
R pressure_of(R e, int eos) {
  if (eos == 1) return (R)(e / 3.0);
  if (eos == 2) {
    const R a0 = -0.25181736420168666, a1 = 9737.845799644809, a2 = 1.077580993288114e6,
            a3 = 3.1729694865420084e6, a4 = 1.6357487344679043e6, a5 = 334334.4309240126,
            a6 = 41913.439282708554, a7 = 6340.448389300905, a8 = 141.5073484468774,
            a9 = 0.7158279081255019, a10 = 0.0009417586777847889, a11 = 3.1188455176941583e-7,
            a12 = 1.9531729608963267e-11;
    const R b0 = 45829.44617893836, b1 = 4.0574329080826794e6, b2 = 2.0931169138134286e7,
            b3 = 1.3512402226067686e7, b4 = 1.7851642641834426e6, b5 = 278581.2989342773,
            b6 = 26452.34905933697, b7 = 499.04919730607065, b8 = 2.3405487982094204,
            b9 = 0.002962497695527404, b10 = 9.601103399348206e-7, b11 = 5.928138360995685e-11,
            b12 = 3.2581066229887368e-18;
    R e1 = e, e2 = e * e, e3 = e2 * e, e4 = e3 * e, e5 = e4 * e, e6 = e5 * e, e7 = e6 * e,
      e8 = e7 * e, e9 = e8 * e, e10 = e9 * e, e11 = e10 * e, e12 = e11 * e;
    using std::fma;
    R a = fma(a12, e12, fma(a11, e11, fma(a10, e10, fma(a9, e9, fma(a8, e8, fma(a7, e7,
          fma(a6, e6, fma(a5, e5, fma(a4, e4, fma(a3, e3, fma(a2, e2, fma(a1, e1, a0))))))))))));
    R b = fma(b12, e12, fma(b11, e11, fma(b10, e10, fma(b9, e9, fma(b8, e8, fma(b7, e7,
          fma(b6, e6, fma(b5, e5, fma(b4, e4, fma(b3, e3, fma(b2, e2, fma(b1, e1, b0))))))))))));
    return a / b;
  }
  return (R)0.0;  // EOS_TYPE 3 placeholder (src/EquationOfState.cpp:72-79)
}

template <class R, bool FG>
int run(const oracle_params& pin, const float* e_gev, const float* nB_in, oracle_out* out) {
  using G = typename std::conditional<FG, float, R>::type;  // geometry type
  oracle_params p = pin;
  if (p.DIM_X < 4 || p.DIM_Y < 4 || p.DIM_ETA < 1 || p.DIM_RAP < 1 || p.DIM_PHIP < 1) return 1;
  if (p.DIM_ETA > 1 && (p.DIM_ETA < 3 || p.DIM_RAP < 2)) return 1;
  p.DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA;  // (src/FreestreamMilne.cpp:177-178)
  p.TAU = p.TAU0 + p.DTAU;
  const int DIM = p.DIM;

  // initial energy density in fm^-4 (src/FreestreamMilne.cpp:266-267), or
  // as given when the profile already is in fm^-4 (the reference's other
  // initial conditions, :231-281)
  std::vector<R> e0(DIM);
  const R lower_tolerance = 1.0e-7;
  for (int i = 0; i < DIM; ++i) {
    if (g_raw_input) {
      e0[i] = (R)e_gev[i];
    } else if (sizeof(R) == 4) {
      float rescale = 1.0f;
      e0[i] = (R)(e_gev[i] * rescale / (float)kHbarcF + (float)lower_tolerance);
    } else {
      e0[i] = (R)((double)e_gev[i] / 0.197326938 + 1.0e-7);
    }
  }

  // energy-dependent free-streaming time (src/FreeStream.cpp:389-417)
  if (p.E_DEP_FS == 1) {  // the free-streaming time is geometry: G arithmetic
    G num = 0.0, den = 0.0;
    for (int i = 0; i < DIM; ++i) {
      G eps = g_raw_input ? (G)e_gev[i]
              : (sizeof(G) == 4) ? (G)(e_gev[i] * 1.0f / kHbarcF + 1.0e-7f)
                                 : (G)((double)e_gev[i] / 0.197326938 + 1.0e-7);
      num += (eps * eps);
      den += eps;
    }
    G e_T = (G)(num / (den + 1.0e-7));
    e_T = e_T * (sizeof(G) == 4 ? (G)kHbarcF : (G)0.197326938);
    G tau_fs = (G)p.TAU_R * std::pow((e_T / (G)p.E_R), (G)p.ALPHA);
    p.DTAU = (float)tau_fs;
    p.TAU = p.TAU0 + p.DTAU;
  }
  // phi_p refinement by arc length (src/FreestreamMilne.cpp:329-332)
  {
    float min_dx_dy = std::min(p.DX, p.DY);
    int nphip = int(std::ceil((2.0 * M_PI * p.DTAU) / min_dx_dy));
    p.DIM_PHIP = std::max(p.DIM_PHIP, nphip);
  }
  out->dim_phip = p.DIM_PHIP;
  out->dtau = p.DTAU;
  out->tau = p.TAU;

  const Grid<G> g = make_grid<G>(p);
  const int NX = g.DIM_X, NY = g.DIM_Y, NE = g.DIM_ETA, NR = g.DIM_RAP, NP = g.DIM_PHIP;
  const bool is3d = NE > 1;

  // ---- initial densities (src/FreeStream.cpp:289-387) as per-(ieta, irap) factors
  // density[is][irap] = e0[is] * norm * rapf[ieta][irap]  (3D), e0/(2 pi) (2D)
  R norm_factor = 0;
  std::vector<R> rapf((size_t)NE * NR, (R)0);
  if (is3d) {
    R SIGMA = p.SIGMA;
    R n = (R)(std::sqrt(M_PI / 2.0) * SIGMA * (1.0 + std::exp(2.0 * SIGMA * SIGMA)));
    norm_factor = (R)(1.0 / (2.0 * M_PI * n));
    for (int ieta = 0; ieta < NE; ++ieta) {
      G eta = (G)ieta * g.DETA + g.etamin;
      for (int irap = 0; irap < NR; ++irap) {
        G w = tanmap_w<G>(irap, NR);
        G rap = (G)(eta + std::tan((M_PI / 2.0) * w));
        R d = (R)(eta - rap);
        R rf = (R)(std::cosh(d) * std::cosh(d) *
                   std::exp((-1.0) * d * d / (2.0 * SIGMA * SIGMA)));
        rapf[(size_t)ieta * NR + irap] = rf;
      }
    }
  }
  std::vector<R> dens2d;  // 2D: F = e/(2 pi)
  if (!is3d) {
    dens2d.resize(DIM);
    for (int i = 0; i < DIM; ++i) dens2d[i] = (R)(e0[i] / (2.0 * M_PI));
  }
  // baryon J~ (src/FreeStream.cpp:353-387): per-(ieta, irap) factor on a uniform grid
  const bool baryon = p.BARYON != 0 && nB_in != nullptr;
  R normB = 0;
  std::vector<R> rapfB;
  if (baryon) {
    R SIGMA_B = p.SIGMA_B;
    R n = (R)(std::sqrt(2.0 * M_PI) * SIGMA_B * std::exp(SIGMA_B * SIGMA_B / 2.0));
    normB = (R)(1.0 / (2.0 * M_PI * n));
    G rapmin = (G)((-1.0) * ((G)(NR - 1) / 2.0) * g.DRAP);
    rapfB.resize((size_t)NE * NR);
    for (int ieta = 0; ieta < NE; ++ieta) {
      G eta = (G)ieta * g.DETA + g.etamin;
      for (int irap = 0; irap < NR; ++irap) {
        G rap = (G)irap * g.DRAP + rapmin;
        R d = (R)(eta - rap);
        rapfB[(size_t)ieta * NR + irap] =
            (R)(std::cosh(d) * std::exp((-1.0) * d * d / (SIGMA_B * SIGMA_B)));
      }
    }
  }
  auto Gval = [&](int is, int irap) -> R {  // density[is][irap]
    if (!is3d) return dens2d[is];
    int ieta = is % NE;
    return e0[is] * norm_factor * rapf[(size_t)ieta * NR + irap];
  };
  auto Jval = [&](int is, int irap) -> R {  // chargeDensity[is][irap]
    int ieta = is % NE;
    return (R)nB_in[is] * normB * rapfB[(size_t)ieta * NR + irap];
  };

  // ---- 2D bicubic spline of slice irap = 0 (src/FreeStream.cpp:121-154)
  fsm_num::Bicubic spl, splB;
  double x_min_i = 0, x_max_i = 0, y_min_i = 0, y_max_i = 0;
  if (!is3d) {
    std::vector<double> xv(NX), yv(NY), zv((size_t)NX * NY), zb;
    if (baryon) zb.resize((size_t)NX * NY);
    for (int ix = 0; ix < NX; ++ix)
      for (int iy = 0; iy < NY; ++iy) {
        int is = NY * ix + iy;
        xv[ix] = (G)((G)ix * g.DX + g.xmin);
        yv[iy] = (G)((G)iy * g.DY + g.ymin);
        zv[(size_t)NX * iy + ix] = Gval(is, 0);
        if (baryon) zb[(size_t)NX * iy + ix] = Jval(is, 0);
      }
    x_min_i = xv[0];
    y_min_i = yv[0];
    x_max_i = xv[NX - 1];
    y_max_i = yv[NY - 1];
    spl.init(xv.data(), yv.data(), zv.data(), NX, NY);
    if (baryon) splB.init(xv.data(), yv.data(), zb.data(), NX, NY);
  }

  // ---- hypertrig table [10][irap][iphip][ieta] (src/LandauMatch.cpp:14-59)
  std::vector<R> trig((size_t)10 * NR * NP * NE);
  auto TI = [&](int v, int irap, int iphip, int ieta) -> R& {
    return trig[(((size_t)v * NR + irap) * NP + iphip) * NE + ieta];
  };
  for (int irap = 0; irap < NR; ++irap)
    for (int iphip = 0; iphip < NP; ++iphip) {
      const R phip = (R)phip_of<G>(iphip, NP);
      for (int ieta = 0; ieta < NE; ++ieta) {
        G eta = (G)ieta * g.DETA + g.etamin;
        if (NE == 1) eta = 0.0;
        G w = tanmap_w<G>(irap, NR);
        G rap = (G)(eta + std::tan((M_PI / 2.0) * w));
        if (NE == 1) rap = 0.0;
        const R d = (R)(rap - eta);
        const R TAU = (R)g.TAU;
        TI(0, irap, iphip, ieta) = 1.0;
        TI(1, irap, iphip, ieta) = std::cos(phip) / std::cosh(d);
        TI(2, irap, iphip, ieta) = std::sin(phip) / std::cosh(d);
        TI(3, irap, iphip, ieta) = (R)((1.0 / TAU) * std::tanh(d));
        TI(4, irap, iphip, ieta) = (std::cos(phip) * std::cos(phip)) / (std::cosh(d) * std::cosh(d));
        TI(5, irap, iphip, ieta) = (std::cos(phip) * std::sin(phip)) / (std::cosh(d) * std::cosh(d));
        TI(6, irap, iphip, ieta) = (R)((1.0 / TAU) * (std::cos(phip) * std::tanh(d)) / std::cosh(d));
        TI(7, irap, iphip, ieta) = (std::sin(phip) * std::sin(phip)) / (std::cosh(d) * std::cosh(d));
        TI(8, irap, iphip, ieta) = (R)((1.0 / TAU) * (std::sin(phip) * std::tanh(d)) / std::cosh(d));
        TI(9, irap, iphip, ieta) = (R)((1.0 / (TAU * TAU)) * std::tanh(d) * std::tanh(d));
      }
    }
  std::vector<R> jac(NR);  // (src/LandauMatch.cpp:92-93)
  for (int irap = 0; irap < NR; ++irap) {
    R w = (R)tanmap_w<G>(irap, NR);
    jac[irap] = (R)((M_PI / 2.0) / std::cos((M_PI / 2.0) * w) / std::cos((M_PI / 2.0) * w) *
                    (1.995 / R(NR - 1)));
  }
  std::vector<G> cphi(NP), sphi(NP);
  for (int iphip = 0; iphip < NP; ++iphip) {
    G phip = phip_of<G>(iphip, NP);
    cphi[iphip] = std::cos(phip);
    sphi[iphip] = std::sin(phip);
  }
  const R d_phip = (R)((2.0 * M_PI) / R(NP));

  // ---- free streaming + moments + Landau matching, per cell
  int n_fallback = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : n_fallback)
  for (int is = 0; is < DIM; ++is) {
    int ix = is / (NY * NE);
    int iy = (is - (NY * NE * ix)) / NE;
    int ieta = is - (NY * NE * ix) - (NE * iy);
    G x = (G)ix * g.DX + g.xmin;
    G y = (G)iy * g.DY + g.ymin;
    G eta = (G)ieta * g.DETA + g.etamin;
    R T[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    R J[4] = {0, 0, 0, 0};
    for (int irap = 0; irap < NR; ++irap) {
      G w = tanmap_w<G>(irap, NR);
      G rap = (G)(eta + std::tan((M_PI / 2.0) * w));
      // (src/FreeStream.cpp:192-194) pieces independent of phi_p
      G eta_new3 = 0, D3 = 0;
      if (is3d) {
        eta_new3 = std::asinh((g.TAU / g.TAU0) * std::sinh(eta - rap)) + rap;
        D3 = (g.TAU * std::cosh(rap - eta_new3) - g.TAU0 * std::cosh(rap - eta));
      }
      for (int iphip = 0; iphip < NP; ++iphip) {
        G eta_new, x_new, y_new;
        if (NE == 1) {
          eta_new = 0.0;
          x_new = x - cphi[iphip] * g.DTAU;
          y_new = y - sphi[iphip] * g.DTAU;
        } else {
          eta_new = eta_new3;
          x_new = x - cphi[iphip] * D3;
          y_new = y - sphi[iphip] * D3;
        }
        G ix_new = (x_new - g.xmin) / g.DX;
        G iy_new = (y_new - g.ymin) / g.DY;
        G ieta_new;
        if (NE > 1) ieta_new = (eta_new - g.etamin) / g.DETA;
        else ieta_new = 0;
        G ix_f = std::floor(ix_new), iy_f = std::floor(iy_new), ie_f = std::floor(ieta_new);
        R xf = (R)(ix_new - ix_f), yf = (R)(iy_new - iy_f), ef = (R)(ieta_new - ie_f);
        if (!((ix_f >= 1) && (ix_f < NX - 1) && (iy_f >= 1) && (iy_f < NY - 1))) continue;
        R interp = 0.0, interpB = 0.0;
        bool have = false;
        if (NE == 1) {
          int i11 = (NY * NE * (int)ix_f) + (NE * (int)iy_f) + (int)ie_f;
          int i21 = (NY * NE * ((int)ix_f + 1)) + (NE * (int)iy_f) + (int)ie_f;
          int i12 = (NY * NE * (int)ix_f) + (NE * ((int)iy_f + 1)) + (int)ie_f;
          int i22 = (NY * NE * ((int)ix_f + 1)) + (NE * ((int)iy_f + 1)) + (int)ie_f;
          bool inside = (x_min_i < (double)x_new) && ((double)x_new < x_max_i) &&
                        (y_min_i < (double)y_new) && ((double)y_new < y_max_i);
          R l = lin2<R>(xf, yf, Gval(i11, irap), Gval(i21, irap), Gval(i12, irap), Gval(i22, irap));
          R c = inside ? (R)spl.eval((double)x_new, (double)y_new) : (R)0.0;
          interp = (c > 0.0) ? c : l;
          if (baryon) {
            R lb = lin2<R>(xf, yf, Jval(i11, irap), Jval(i21, irap), Jval(i12, irap), Jval(i22, irap));
            R cb = inside ? (R)splB.eval((double)x_new, (double)y_new) : (R)0.0;
            interpB = (cb > 0.0) ? cb : lb;
          }
          have = true;
        } else if ((ie_f >= 1) && (ie_f < NE - 1)) {
          int ixf = (int)ix_f, iyf = (int)iy_f, ief = (int)ie_f;
          int i000 = (NY * NE * ixf) + (NE * iyf) + ief;
          int i100 = (NY * NE * (ixf + 1)) + (NE * iyf) + ief;
          int i010 = (NY * NE * ixf) + (NE * (iyf + 1)) + ief;
          int i110 = (NY * NE * (ixf + 1)) + (NE * (iyf + 1)) + ief;
          int i001 = i000 + 1, i101 = i100 + 1, i011 = i010 + 1, i111 = i110 + 1;
          interp = lin3<R>(xf, yf, ef, Gval(i000, irap), Gval(i100, irap), Gval(i010, irap),
                           Gval(i001, irap), Gval(i110, irap), Gval(i101, irap), Gval(i011, irap),
                           Gval(i111, irap));
          if (baryon)
            interpB = lin3<R>(xf, yf, ef, Jval(i000, irap), Jval(i100, irap), Jval(i010, irap),
                              Jval(i001, irap), Jval(i110, irap), Jval(i101, irap),
                              Jval(i011, irap), Jval(i111, irap));
          have = true;
        }
        if (!have) continue;
        // (src/LandauMatch.cpp:100-101, 137)
        for (int v = 0; v < 10; ++v) {
          if (NE == 1) T[v] += interp * TI(v, irap, iphip, ieta);
          else T[v] += interp * TI(v, irap, iphip, ieta) * jac[irap];
        }
        if (baryon)
          for (int v = 0; v < 4; ++v) J[v] += interpB * TI(v, irap, iphip, ieta);
      }
    }
    for (int v = 0; v < 10; ++v) {  // (src/LandauMatch.cpp:104-105)
      if (NE == 1) T[v] = T[v] * d_phip / (R)g.TAU;
      else T[v] = T[v] * d_phip;
    }
    if (baryon)
      for (int v = 0; v < 4; ++v) J[v] = J[v] * g.DRAP * d_phip;  // (LandauMatch.cpp:140)

    R e, u[4];
    int ok = landau_cell<R>(T, (R)g.TAU, &e, u);
    if (!ok) ++n_fallback;
    R nBc = 0, V[4] = {0, 0, 0, 0};
    if (baryon) {  // (src/LandauMatch.cpp:370-392)
      nBc = (u[0] * J[0]) - (u[1] * J[1]) - (u[2] * J[2]) - ((R)g.TAU * (R)g.TAU * u[3] * J[3]);
      for (int v = 0; v < 4; ++v) V[v] = J[v] - (nBc * u[v]);
    }
    R P = pressure_of<R>(e, p.EOS_TYPE);
    R Pi = 0, pi[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (p.VISCOUS_MATCHING) {  // (src/LandauMatch.cpp:332-367)
      R TAU = (R)g.TAU;
      R a = T[0] - T[4] - T[7] - TAU * TAU * T[9];
      Pi = (R)((-1.0 / 3.0) * (a - e) - P);
      R b = e + P + Pi;
      R c = P + Pi;
      pi[0] = T[0] - u[0] * u[0] * b + c;
      pi[1] = T[1] - u[0] * u[1] * b;
      pi[2] = T[2] - u[0] * u[2] * b;
      pi[3] = T[3] - u[0] * u[3] * b;
      pi[4] = T[4] - u[1] * u[1] * b - c;
      pi[5] = T[5] - u[1] * u[2] * b;
      pi[6] = T[6] - u[1] * u[3] * b;
      pi[7] = T[7] - u[2] * u[2] * b - c;
      pi[8] = T[8] - u[2] * u[3] * b;
      pi[9] = (R)(T[9] - u[3] * u[3] * b - c * (1.0 / (TAU * TAU)));
    }
    if (out->T)
      for (int v = 0; v < 10; ++v) out->T[(size_t)v * DIM + is] = T[v];
    if (out->J && baryon)
      for (int v = 0; v < 4; ++v) out->J[(size_t)v * DIM + is] = J[v];
    if (out->e) out->e[is] = e;
    if (out->P) out->P[is] = P;
    if (out->Pi) out->Pi[is] = Pi;
    if (out->u)
      for (int v = 0; v < 4; ++v) out->u[(size_t)v * DIM + is] = u[v];
    if (out->pi)
      for (int v = 0; v < 10; ++v) out->pi[(size_t)v * DIM + is] = pi[v];
    if (out->nB && baryon) out->nB[is] = nBc;
    if (out->V && baryon)
      for (int v = 0; v < 4; ++v) out->V[(size_t)v * DIM + is] = V[v];
  }
  out->n_fallback = n_fallback;
  return 0;
}

}  // namespace

extern "C" int oracle_run(const oracle_params* p, int fp64, const float* e_gev, const float* nB,
                          oracle_out* out, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  if (fp64 == 1) return run<double, false>(*p, e_gev, nB, out);
  if (fp64 == 2) return run<double, true>(*p, e_gev, nB, out);
  return run<float, true>(*p, e_gev, nB, out);
}

// oracle_run for a profile already in fm^-4 (no GeV/fm^3 conversion).
extern "C" int oracle_run_fm4(const oracle_params* p, int fp64, const float* e_fm4, const float* nB,
                              oracle_out* out, int nthreads) {
  g_raw_input = true;
  const int rc = oracle_run(p, fp64, e_fm4, nB, out, nthreads);
  g_raw_input = false;
  return rc;
}

extern "C" void oracle_spline_derivs(const double* x, const double* y, int n, double* d) {
  fsm_num::natural_spline_node_derivs(x, y, 1, (size_t)n, d, 1);
}

extern "C" void oracle_bicubic_eval(const double* x, const double* y, const double* z, int nx,
                                    int ny, const double* px, const double* py, int npts,
                                    double* outv) {
  fsm_num::Bicubic b;
  b.init(x, y, z, (size_t)nx, (size_t)ny);
  for (int k = 0; k < npts; ++k) outv[k] = b.eval(px[k], py[k]);
}

extern "C" int oracle_eig(int n, const double* A, double* wr, double* wi, double* vr) {
  return fsm_num::eig_nonsym(n, A, wr, wi, vr);
}

extern "C" int oracle_landau_cell(const float* T10, float tau, float* e, float* u4) {
  return landau_cell<float>(T10, tau, e, u4);
}

// ---- diagnostics: restated from src/HydroValidity.cpp:8-101 and
// src/LandauMatch.cpp:395-489 with the reference's float/double mixing.
extern "C" void oracle_diagnostics(const oracle_params* p, float tau, const float* e,
                                   const float* P, const float* Pi, const float* u,
                                   const float* pi, float* out) {
  const int NX = p->DIM_X, NY = p->DIM_Y, NE = p->DIM_ETA;
  const size_t n = (size_t)NX * NY * NE;
  for (size_t k = 0; k < 17 * n; ++k) out[k] = 0.0f;
  float* rpi = out;
  float* rsh = out + n;
  float* pdu = out + 2 * n;
  float* pmm = out + 6 * n;
  float* beta = out + 7 * n;
  float* om = out + 11 * n;
  const float tau2 = tau * tau;
  for (size_t is = 0; is < n; ++is) {
    // bulk inverse Reynolds number (HydroValidity.cpp:8-19)
    float pp = (P[is] < 1.0e-5) ? 1.0e-5 : P[is];
    rpi[is] = Pi[is] / pp;
    // shear inverse Reynolds number (HydroValidity.cpp:21-38)
    const float* s = pi;
    auto S = [&](int m) { return s[m * n + is]; };
    float num = S(0) * S(0) - 2.0 * (S(1) * S(1) + S(2) * S(2) + tau2 * S(3) * S(3)) +
                (S(4) * S(4) + S(7) * S(7) + tau2 * tau2 * S(9) * S(9)) +
                2.0 * (S(5) * S(5) + tau2 * S(6) * S(6) + tau2 * S(8) * S(8));
    float den;
    if (e[is] < 1.0e-5) den = 1.0e-5;
    else den = e[is] * e[is] + 3.0 * P[is] * P[is];
    rsh[is] = std::sqrt(std::fabs(num)) / std::sqrt(std::fabs(den));
    // pi^{mu nu} u_nu (HydroValidity.cpp:40-79)
    float ut = u[is], ux = -u[n + is], uy = -u[2 * n + is], un = -tau * tau * u[3 * n + is];
    pdu[is] = S(0) * ut + S(1) * ux + S(2) * uy + S(3) * un;
    pdu[n + is] = S(1) * ut + S(4) * ux + S(5) * uy + S(6) * un;
    pdu[2 * n + is] = S(2) * ut + S(5) * ux + S(7) * uy + S(8) * un;
    pdu[3 * n + is] = S(3) * ut + S(6) * ux + S(8) * uy + S(9) * un;
    // pi^mu_mu (HydroValidity.cpp:81-101)
    float pxx = -S(4), pyy = -S(7), pnn = -tau * tau * S(9);
    pmm[is] = S(0) + pxx + pyy + pnn;
  }
  // thermal velocity and vorticity (LandauMatch.cpp:395-489): interior (ix, iy),
  // cell index DIM_Y * ix + iy as in the reference
  auto T = [&](size_t k) { return std::pow((e[k] / 13.8997f), 0.25f); };
  for (int ix = 1; ix < NX - 1; ++ix)
    for (int iy = 1; iy < NY - 1; ++iy) {
      const size_t is = (size_t)NY * ix + iy, px = (size_t)NY * (ix + 1) + iy,
                   mx = (size_t)NY * (ix - 1) + iy, py = (size_t)NY * ix + (iy + 1),
                   my = (size_t)NY * ix + (iy - 1);
      float Tc = T(is), Tpx = T(px), Tmx = T(mx), Tpy = T(py), Tmy = T(my);
      beta[is] = u[is] / Tc;
      beta[n + is] = -u[n + is] / Tc;
      beta[2 * n + is] = -u[2 * n + is] / Tc;
      beta[3 * n + is] = 0.0f / Tc;
      float bx_py = -u[n + py] / Tpy, bx_my = -u[n + my] / Tmy;
      float by_px = -u[2 * n + px] / Tpx, by_mx = -u[2 * n + mx] / Tmx;
      om[3 * n + is] = 0.5 * ((bx_py - bx_my) / 2.0 / p->DY - (by_px - by_mx) / 2.0 / p->DX);
    }
}
