// fsm_hosttest.cpp -- TEST-ONLY build of the Landau-matching algorithm of
// fsm_landau.cuh and the windowed spline slopes of fsm_spline.cuh for the CPU,
// so unit tests can exercise their logic against the oracle without a GPU.
// Not part of libfsm.so; the product runs the same headers only inside its
// kernels.
#include <string>
#include <vector>

#include "fsm_landau.cuh"
#include "fsm_plan.h"
#include "fsm_spline.cuh"

// Slopes dy/dx * d of the natural spline through y[0..n) on the float grid
// i*d + lo, segment by segment as the prep kernels compute them.
extern "C" void fsm_hosttest_line_slopes(const float* y, int n, float d, float lo, float* out) {
  std::vector<fsm::AxisNode> ax;
  fsm::build_axis(n, d, lo, ax);
  const fsm::AxisNode* A = ax.data() + fsm::kPadLo;
  std::vector<double> yp((size_t)n + fsm::kPadLo + fsm::kPadHi, 0.0);
  for (int i = 0; i < n; ++i) yp[(size_t)fsm::kPadLo + i] = y[i];
  const double* Y = yp.data() + fsm::kPadLo;
  for (int a = 0; a < n; a += fsm::kSegP) {
    float s[fsm::kSegP];
    fsm::seg_slopes([&](int k) -> const fsm::AxisNode& { return A[k]; }, n, (double)d, a,
                    [&](int i) { return Y[i]; }, s);
    for (int t = 0; t < fsm::kSegP && a + t < n; ++t) out[a + t] = s[t];
  }
}

extern "C" int fsm_hosttest_landau_cell(const float* T10, const float* J4, int is3d, int baryon,
                                        int eos, int viscous, float tau, float* out24) {
  fsm::CellOut o;
  fsm::landau_cell(T10, J4, is3d, baryon, eos, viscous, tau, &o);
  // e P Pi u[4] pi[10] nB V[4] fallback
  out24[0] = o.e;
  out24[1] = o.P;
  out24[2] = o.Pi;
  for (int k = 0; k < 4; ++k) out24[3 + k] = o.u[k];
  for (int k = 0; k < 10; ++k) out24[7 + k] = o.pi[k];
  out24[17] = o.nB;
  for (int k = 0; k < 4; ++k) out24[18 + k] = o.V[k];
  out24[22] = (float)o.fallback;
  return o.fallback ? 0 : 1;
}

// FNV-1a digest of the tables plan_event builds for *p, planned on the worker
// pool (serial = 0) or on the calling thread only (serial = 1).  Returns the
// plan status.
extern "C" int fsm_hosttest_plan_digest(const fsm_params* p, int serial, unsigned long long* digest) {
  fsm::EventPlan E;
  std::string why;
  if (serial) ++fsm::parallel_depth();
  const fsm_status s = fsm::plan_event(*p, nullptr, &E, &why);
  if (serial) --fsm::parallel_depth();
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](const void* data, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  };
  mix(E.cs.data(), E.cs.size() * sizeof(E.cs[0]));
  mix(E.tab2.data(), E.tab2.size() * sizeof(E.tab2[0]));
  mix(E.chunks2.data(), E.chunks2.size() * sizeof(E.chunks2[0]));
  mix(E.re.data(), E.re.size() * sizeof(E.re[0]));
  mix(E.rapf.data(), E.rapf.size() * 4);
  mix(E.rapfB.data(), E.rapfB.size() * 4);
  if (E.tab3) mix(E.tab3->data(), E.tab3->size() * sizeof(fsm::PhiEntry3D));
  mix(E.live_eta.data(), E.live_eta.size() * sizeof(E.live_eta[0]));
  mix(E.plane_of.data(), E.plane_of.size() * sizeof(int));
  mix(E.cw_start.data(), E.cw_start.size() * sizeof(int));
  mix(E.cw.data(), E.cw.size() * sizeof(fsm::CombW));
  mix(&E.r_lo, sizeof(E.r_lo));
  mix(&E.r_hi, sizeof(E.r_hi));
  *digest = h;
  return (int)s;
}

// The 2D output tiles of one event as (x0, y0, shape, x1, y1), with the runs
// planned per shape (nch[7]) and the largest staged window in nodes; returns
// the number of tiles (at most cap written) or -1 when planning fails.
extern "C" int fsm_hosttest_tiles(const fsm_params* p, int tail_tiles, int window_budget, int* out,
                                  int cap, int* nch, int* box_elems) {
  fsm::EventPlan E;
  std::string why;
  if (fsm::plan_event(*p, nullptr, &E, &why, window_budget, false, tail_tiles != 0) != FSM_OK) return -1;
  std::vector<fsm::Tile2D> t;
  fsm::tiles_2d(E, 0, t);
  for (int k = 0; k < (int)t.size() && k < cap; ++k) {
    out[5 * k + 0] = t[k].x0;
    out[5 * k + 1] = t[k].y0;
    out[5 * k + 2] = t[k].shape;
    out[5 * k + 3] = t[k].x1;
    out[5 * k + 4] = t[k].y1;
  }
  for (int s = 0; s < fsm::kShapes2D; ++s) nch[s] = E.nch[s];
  *box_elems = E.box_elems;
  return (int)t.size();
}

// The combined-plane tables of a 3D event: plane_of[NE*NR], cw_start[NE],
// cw as (plane, w0, w1, b0, b1) float rows [cap], and per (ieta, irap) pair
// (efl, efrac, D) [NE*NR] and the rapidity weights rapf, rapfB [NE*NR], with
// r_lo, r_hi.  Returns the number of planes (at most cap written) or -1.
extern "C" int fsm_hosttest_comb_planes(const fsm_params* p, int* plane_of, int* cw_start, float* cw,
                                        int cap, float* pair3, float* rapf, float* rapfB, int* r_lohi) {
  fsm::EventPlan E;
  std::string why;
  if (fsm::plan_event(*p, nullptr, &E, &why) != FSM_OK || !E.is3d) return -1;
  const size_t np = E.re.size();
  for (size_t i = 0; i < np; ++i) {
    plane_of[i] = E.plane_of[i];
    pair3[3 * i + 0] = (float)E.re[i].efl;
    pair3[3 * i + 1] = E.re[i].efrac;
    pair3[3 * i + 2] = E.re[i].D;
    rapf[i] = E.rapf[i];
    rapfB[i] = E.rapfB[i];
  }
  for (size_t e = 0; e < E.cw_start.size(); ++e) cw_start[e] = E.cw_start[e];
  for (int k = 0; k < (int)E.cw.size() && k < cap; ++k) {
    cw[5 * k + 0] = (float)E.cw[k].plane;
    cw[5 * k + 1] = E.cw[k].w0;
    cw[5 * k + 2] = E.cw[k].w1;
    cw[5 * k + 3] = E.cw[k].b0;
    cw[5 * k + 4] = E.cw[k].b1;
  }
  r_lohi[0] = E.r_lo;
  r_lohi[1] = E.r_hi;
  return (int)E.cw.size();
}
