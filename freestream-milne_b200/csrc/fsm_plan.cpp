// fsm_plan.cpp -- parameters, status strings and per-event planning (host).
//
// Compiled with the host compiler and -ffp-contract=off: every float table
// entry below repeats the reference's own expression with its float/double
// mixing, so the kernels see the same shift lengths, node angles and index
// floors the reference computes (a one-ulp difference in a shift can move a
// sample across the in-grid test at src/FreeStream.cpp:213).
#include "fsm_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <mutex>
#include <functional>
#include <condition_variable>
#include <atomic>
#include <unistd.h>

namespace fsm {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

namespace {

// Worker threads started on first use and kept for the life of the process
// (blocked on a condition variable between jobs).  A child created by fork()
// inherits the pool object but none of its threads: it runs loops serially.
struct WorkerPool {
  const pid_t owner = getpid();
  std::mutex busy;  // one job at a time
  std::mutex m;
  std::condition_variable cv, cv_done;
  const std::function<void(int)>* f = nullptr;
  int n = 0, want = 0, running = 0;
  std::atomic<int> next{0};
  unsigned long long gen = 0;
  std::vector<std::thread> th;

  explicit WorkerPool(int workers) {
    for (int t = 0; t < workers; ++t) th.emplace_back([this, t] { loop(t); });
  }
  void drain() {
    for (int i; (i = next.fetch_add(1)) < n;) (*f)(i);
  }
  void loop(int t) {
    unsigned long long seen = 0;
    std::unique_lock<std::mutex> lk(m);
    for (;;) {
      cv.wait(lk, [&] { return gen != seen; });
      seen = gen;
      if (t >= want) continue;  // this job uses fewer threads
      lk.unlock();
      ++parallel_depth();
      drain();
      --parallel_depth();
      lk.lock();
      if (--running == 0) cv_done.notify_all();
    }
  }
};

WorkerPool& worker_pool() {
  static WorkerPool* pool = new WorkerPool(host_threads() - 1);  // kept until exit
  return *pool;
}

}  // namespace

int host_threads() {
  static const int n = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
  return n;
}

int& parallel_depth() {
  static thread_local int d = 0;
  return d;
}

void run_parallel(int n, int threads, const std::function<void(int)>& f) {
  threads = std::min(std::min(threads, n), host_threads());
  if (threads <= 1 || parallel_depth() > 0) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  WorkerPool& P = worker_pool();
  std::unique_lock<std::mutex> job(P.busy, std::try_to_lock);
  if (!job.owns_lock() || P.owner != getpid()) {  // in use by another host thread, or forked
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  {
    std::lock_guard<std::mutex> g(P.m);
    P.f = &f;
    P.n = n;
    P.next = 0;
    P.want = threads - 1;
    P.running = threads - 1;
    ++P.gen;
  }
  P.cv.notify_all();
  ++parallel_depth();
  P.drain();
  --parallel_depth();
  std::unique_lock<std::mutex> lk(P.m);
  P.cv_done.wait(lk, [&] { return P.running == 0; });
  P.f = nullptr;
}

void parallel_copy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kPiece = (size_t)1 << 20;
  const int pieces = (int)((bytes + kPiece - 1) / kPiece);
  parallel_for(pieces, bytes >= 2 * kPiece ? host_threads() : 1, [&](int k) {
    const size_t o = (size_t)k * kPiece;
    std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o,
                std::min(kPiece, bytes - o));
  });
}

int output_components(bool baryon) { return baryon ? 36 : 27; }

static inline float tanmap_w(int irap, int NR) {  // src/FreeStream.cpp:174
  return (float)(-.9975 + (float)irap * (1.995 / (float)(NR - 1)));
}

// Natural-spline axis table on the float grid coordinates x_i = i*d + lo
// (src/FreeStream.cpp:129-140): interval widths and the elimination factors of
// the tridiagonal system, padded with zero entries (see AxisNode).
void build_axis(int n, float d, float lo, std::vector<AxisNode>& ax) {
  std::vector<double> xv(n);
  for (int i = 0; i < n; ++i) {
    float xf = (float)i * d + lo;
    xv[i] = xf;
  }
  ax.assign((size_t)n + kPadLo + kPadHi, AxisNode{0.0, 0.0, 0.0, 0.0});
  AxisNode* A = ax.data() + kPadLo;
  for (int i = 0; i + 1 < n; ++i) {
    A[i].h = xv[i + 1] - xv[i];
    A[i].g = 6.0 / A[i].h;
  }
  const int m = n - 2;
  double dgp = 0.0;
  for (int k = 0; k < m; ++k) {
    double dg = 2.0 * (A[k].h + A[k + 1].h);
    if (k > 0) {
      A[k].f = A[k].h / dgp;
      dg -= A[k].f * A[k].h;
    }
    A[k].idg = 1.0 / dg;
    dgp = dg;
  }
}

float edep_dtau(const fsm_params& p, float numerator, float denominator) {
  const float hbarc = 0.197326938;
  float e_T = numerator / (denominator + 1.0e-7);  // src/FreeStream.cpp:411-415
  e_T = e_T * hbarc;
  return p.TAU_R * std::pow((e_T / p.E_R), p.ALPHA);
}

int y_tail_shape(int NY) {
  const int r = NY % kTileY;
  return r == 0 ? -1 : r <= 4 ? 6 : r <= 8 ? 2 : r <= 16 ? 1 : -1;
}

int x_tail_shape(int NX) {
  const int r = NX % kTileX;
  return r == 0 ? -1 : r <= 4 ? 5 : r <= 8 ? 4 : r <= 16 ? 3 : -1;
}

void grid_tiles(int NX, int NY, int ys, int xs, std::vector<TileXY>& out) {
  // the 32 x 32 region: whole tiles up to the narrow last strips, or over the
  // whole grid (rounded up) where a last strip keeps 32 x 32 tiles
  const int NXm = xs >= 0 ? NX - NX % kTileX : (NX + kTileX - 1) / kTileX * kTileX;
  const int NYm = ys >= 0 ? NY - NY % kTileY : (NY + kTileY - 1) / kTileY * kTileY;
  for (int x0 = 0; x0 < NXm; x0 += kTileX)
    for (int y0 = 0; y0 < NYm; y0 += kTileY) out.push_back(TileXY{x0, y0, 0, NX, NY});
  // the last y strip, x < NXr (up to the last x strip, when that has its own
  // tiles): its last tile stores no cell of the x strip
  const int NXr = xs >= 0 ? NXm : NX;
  if (ys >= 0)
    for (int x0 = 0; x0 < NXr; x0 += shape_tx(ys)) out.push_back(TileXY{x0, NYm, ys, NXr, NY});
  // the last x strip over the whole y range (its corner with the y strip included)
  if (xs >= 0)
    for (int y0 = 0; y0 < NY; y0 += shape_ty(xs)) out.push_back(TileXY{NXm, y0, xs, NX, NY});
}

void tiles_2d(const EventPlan& P, int ev, std::vector<Tile2D>& out, bool square) {
  std::vector<TileXY> t;
  grid_tiles(P.p.DIM_X, P.p.DIM_Y, square ? -1 : P.y_shape, square ? -1 : P.x_shape, t);
  for (const TileXY& q : t) out.push_back(Tile2D{ev, q.x0, q.y0, q.shape, q.x1, q.y1});
}

fsm_status plan_event(const fsm_params& in, const float* host_e_gev, EventPlan* out,
                      std::string* why, int window_budget, bool input_fm4, bool tail_tiles) {
  EventPlan& E = *out;
  E = EventPlan();
  E.input_fm4 = input_fm4;
  fsm_params p = in;
  auto fail = [&](fsm_status s, const char* msg) {
    if (why) *why = msg;
    return s;
  };
  if (p.DIM_X < 4 || p.DIM_Y < 4)
    return fail(FSM_ERR_INVALID_ARG, "DIM_X and DIM_Y must be >= 4 (bicubic spline minimum)");
  if (p.DIM_ETA < 1 || p.DIM_RAP < 1 || p.DIM_PHIP < 1)
    return fail(FSM_ERR_INVALID_ARG, "DIM_ETA, DIM_RAP and DIM_PHIP must be >= 1");
  if (!(p.DX > 0) || !(p.DY > 0)) return fail(FSM_ERR_INVALID_ARG, "DX and DY must be > 0");
  if (!(p.DTAU >= 0)) return fail(FSM_ERR_INVALID_ARG, "DTAU must be >= 0");
  E.is3d = p.DIM_ETA > 1;
  if (E.is3d) {
    if (p.DIM_RAP < 2)
      return fail(FSM_ERR_UNSUPPORTED,
                  "3D needs DIM_RAP >= 2 (the reference's tan-map node is NaN for DIM_RAP = 1)");
    if (!(p.DETA > 0) || !(p.TAU0 > 0))
      return fail(FSM_ERR_INVALID_ARG, "3D needs DETA > 0 and TAU0 > 0");
  }
  if (!E.is3d && p.DIM_Y > kMaxNY2D)
    return fail(FSM_ERR_TOO_LARGE, "DIM_Y above 5120 on the 2D path");
  E.baryon = p.BARYON != 0;
  long long dim = (long long)p.DIM_X * p.DIM_Y * p.DIM_ETA;
  if (dim > (1ll << 30)) return fail(FSM_ERR_TOO_LARGE, "grid too large");
  p.DIM = (int)dim;
  p.TAU = p.TAU0 + p.DTAU;  // src/FreestreamMilne.cpp:177-178

  const float hbarc = 0.197326938;
  if (p.E_DEP_FS == 1) {  // src/FreeStream.cpp:389-417 on the converted profile
    if (!host_e_gev)
      return fail(FSM_ERR_UNSUPPORTED, "E_DEP_FS=1 needs the profile on the host (fsm_run_event)");
    float numerator = 0.0, denominator = 0.0;
    float rescale = 1.0, lower_tolerance = 1.0e-7;
    for (int i = 0; i < p.DIM; i++) {
      // the sums run over the profile in fm^-4 (converted from GeV/fm^3 unless
      // it already is, src/FreestreamMilne.cpp:266-267)
      float eps = input_fm4 ? host_e_gev[i] : host_e_gev[i] * rescale / (float)hbarc + lower_tolerance;
      numerator += (eps * eps);
      denominator += eps;
    }
    p.DTAU = edep_dtau(p, numerator, denominator);
    p.TAU = p.TAU0 + p.DTAU;
  }
  if (!(p.TAU > 0)) return fail(FSM_ERR_INVALID_ARG, "TAU0 + DTAU must be > 0");
  {  // phi_p arc-length rule, src/FreestreamMilne.cpp:329-332
    float min_dx_dy = std::min(p.DX, p.DY);
    int nphip = int(std::ceil((2.0 * M_PI * p.DTAU) / min_dx_dy));
    p.DIM_PHIP = std::max(p.DIM_PHIP, nphip);
  }
  if (p.DIM_PHIP > 16384) return fail(FSM_ERR_TOO_LARGE, "DIM_PHIP above 16384");
  E.p = p;
  E.DIM = p.DIM;
  const int NX = p.DIM_X, NY = p.DIM_Y, NE = p.DIM_ETA, NR = p.DIM_RAP, NP = p.DIM_PHIP;

  // grid origin (src/FreeStream.cpp:113-115) and spline domain (:142-146)
  E.xmin = (-1.0) * ((float)(NX - 1) / 2.0) * p.DX;
  E.ymin = (-1.0) * ((float)(NY - 1) / 2.0) * p.DY;
  E.etamin = (-1.0) * ((float)(NE - 1) / 2.0) * p.DETA;
  E.xmax_i = (float)(NX - 1) * p.DX + E.xmin;
  E.ymax_i = (float)(NY - 1) * p.DY + E.ymin;
  E.d_phip = (2.0 * M_PI) / float(NP);  // src/LandauMatch.cpp:74

  // phi_p nodes (src/FreeStream.cpp:179, cos/sin of a float)
  E.cs.resize(NP);
  for (int k = 0; k < NP; ++k) {
    float phip = float(k) * (2.0 * M_PI) / float(NP);
    E.cs[k].x = std::cos(phip);
    E.cs[k].y = std::sin(phip);
  }

  if (!E.is3d) {
    // natural-spline axes on the float grid coordinates (src/FreeStream.cpp:129-140)
    build_axis(NX, p.DX, E.xmin, E.axx);
    build_axis(NY, p.DY, E.ymin, E.axy);
    // per-phi_p stream table (see PhiEntry2D)
    E.tab2.resize(NP);
    for (int k = 0; k < NP; ++k) {
      PhiEntry2D& w = E.tab2[k];
      const float c = E.cs[k].x, s = E.cs[k].y;
      const float shx = c * p.DTAU, shy = s * p.DTAU;  // reference float products
      const double sx = -(double)shx / (double)p.DX, sy = -(double)shy / (double)p.DY;
      const double ox = std::floor(sx), oy = std::floor(sy);
      const double t = sx - ox, u = sy - oy;
      auto herm = [](double a, float* H0, float* H1, float* G0, float* G1, float* dH0, float* dH1,
                     float* dG0, float* dG1) {
        *H0 = 1.0 - 3.0 * a * a + 2.0 * a * a * a;
        *H1 = 3.0 * a * a - 2.0 * a * a * a;
        *G0 = a - 2.0 * a * a + a * a * a;
        *G1 = a * a * a - a * a;
        *dH0 = -6.0 * a + 6.0 * a * a;
        *dH1 = -*dH0;
        *dG0 = 1.0 - 4.0 * a + 3.0 * a * a;
        *dG1 = 3.0 * a * a - 2.0 * a;
      };
      herm(t, &w.H0, &w.H1, &w.G0, &w.G1, &w.dH0, &w.dH1, &w.dG0, &w.dG1);
      herm(u, &w.K0, &w.K1, &w.L0, &w.L1, &w.dK0, &w.dK1, &w.dL0, &w.dL1);
      w.t = (float)t;
      w.u = (float)u;
      w.c = c;
      w.s = s;
      w.cc = c * c;
      w.cs = c * s;
      w.ox = (int)ox;
      const int nearx = (t < 1e-3 || t > 1.0 - 1e-3) ? 1 : 0;
      const int neary = (u < 1e-3 || u > 1.0 - 1e-3) ? 1 : 0;
      w.oy_near = ((int)oy & 0xffff) | (nearx << 16) | (neary << 17);
    }
    // bit 18: the integer offset differs from the previous phi_p's (always at
    // phi_p 0, where every tile starts), so the stream kernel reloads the
    // nodes it keeps in registers exactly there
    for (int k = 0; k < NP; ++k) {
      PhiEntry2D& w = E.tab2[k];
      const bool moved = (k == 0) || w.ox != E.tab2[k - 1].ox ||
                         (w.oy_near & 0xffff) != (E.tab2[k - 1].oy_near & 0xffff);
      if (moved) w.oy_near |= 1 << 18;
    }
    // offset range over all phi_p
    auto oy_of = [&](int k) { return (int)(short)(E.tab2[k].oy_near & 0xffff); };
    E.ox_min = E.ox_max = E.tab2[0].ox;
    E.oy_min = E.oy_max = oy_of(0);
    for (int k = 1; k < NP; ++k) {
      E.ox_min = std::min(E.ox_min, E.tab2[k].ox);
      E.ox_max = std::max(E.ox_max, E.tab2[k].ox);
      E.oy_min = std::min(E.oy_min, oy_of(k));
      E.oy_max = std::max(E.oy_max, oy_of(k));
    }
    // phi_p runs, per tile shape the event uses, of at most kMaxRunPhi2D
    // nodes whose staged window (tile + offset spread + 1-node margins) fits
    // the window budget; consecutive nodes have neighbouring offsets.  A
    // budget that cuts the circle into more than kMaxChunks2D runs is raised
    // up to kMaxWindow2D (fewer, larger windows for long free-streaming
    // distances).
    const int min_runs = (NP + kMaxRunPhi2D - 1) / kMaxRunPhi2D;
    E.y_shape = tail_tiles ? y_tail_shape(E.p.DIM_Y) : -1;
    E.x_shape = tail_tiles ? x_tail_shape(E.p.DIM_X) : -1;
    E.chunks2.clear();
    E.box_elems = 0;
    // the narrow shapes plan at the budget the 32 x 32 shape ended with and
    // never raise it: a batch sizes its shared memory by its largest window,
    // so a narrow tile must not push every CTA of the launch past two per SM
    int budget0 = window_budget;
    for (int sh = 0; sh < kShapes2D; ++sh) {
      E.choff[sh] = (int)E.chunks2.size();
      E.nch[sh] = 0;
      if (sh != 0 && sh != E.y_shape && sh != E.x_shape) continue;
      const int TX = shape_tx(sh), TY = shape_ty(sh);
      std::vector<Chunk2D> runs;
      int box = 0;
      for (int budget = sh == 0 ? window_budget : budget0;; budget = budget * 3 / 2) {
        if (sh == 0) budget0 = budget;
        auto win_bytes = [&](int dox, int doy) {
          return (size_t)(TX + dox + 3) * (size_t)(TY + doy + 3) * 16;
        };
        runs.clear();
        box = 0;
        int p0 = 0;
        int lo_x = E.tab2[0].ox, hi_x = lo_x, lo_y = oy_of(0), hi_y = lo_y;
        for (int k = 1; k <= NP; ++k) {
          bool flush = (k == NP) || (k - p0 == kMaxRunPhi2D);
          if (!flush) {
            int nlx = std::min(lo_x, E.tab2[k].ox), nhx = std::max(hi_x, E.tab2[k].ox);
            int nly = std::min(lo_y, oy_of(k)), nhy = std::max(hi_y, oy_of(k));
            if (win_bytes(nhx - nlx, nhy - nly) > (size_t)budget) {
              flush = true;
            } else {
              lo_x = nlx; hi_x = nhx; lo_y = nly; hi_y = nhy;
            }
          }
          if (flush) {
            runs.push_back(Chunk2D{p0, k, lo_x, lo_y, hi_x, hi_y});
            box = std::max(box, (TX + (hi_x - lo_x) + 3) * (TY + (hi_y - lo_y) + 3));
            if (k < NP) {
              p0 = k;
              lo_x = hi_x = E.tab2[k].ox;
              lo_y = hi_y = oy_of(k);
            }
          }
        }
        const bool few = (int)runs.size() <= std::max(kMaxChunks2D, 2 * min_runs);
        if (sh != 0 || few || budget * 3 / 2 > kMaxWindow2D) break;
      }
      E.chunks2.insert(E.chunks2.end(), runs.begin(), runs.end());
      E.nch[sh] = (int)runs.size();
      E.box_elems = std::max(E.box_elems, box);
    }
    E.samples = (double)p.DIM * NP;
    E.ref_samples = (double)p.DIM * NR * NP;
    if (E.baryon) {
      // Charge pass.  The reference splines the irap = 0 slice of
      // J~ = n_B * normB * c_irap (src/FreeStream.cpp:137, 353-387) for every
      // rapidity and falls back to each slice's own bilinear value, so per
      // sample the rapidity sum is NR c_0 S(B) when the spline of B = n_B normB
      // is positive and (sum_irap c_irap) L(B) otherwise, c_irap the uniform-
      // grid rapidity weights at eta = 0.
      float SIGMA_B = p.SIGMA_B;
      float nb = std::sqrt(2.0 * M_PI) * SIGMA_B * std::exp(SIGMA_B * SIGMA_B / 2.0);
      E.normB = 1.0 / (2.0 * M_PI * nb);  // src/FreeStream.cpp:365-366
      const float rapmin = (-1.0) * ((float)(NR - 1) / 2.0) * p.DRAP;
      const float eta = 0.0f * p.DETA + E.etamin;
      double csum = 0.0;
      float c0 = 0.0f;
      for (int irap = 0; irap < NR; ++irap) {
        float rap = (float)irap * p.DRAP + rapmin;
        float c = std::cosh(eta - rap) * std::exp((-1.0) * (eta - rap) * (eta - rap) / (SIGMA_B * SIGMA_B));
        csum += c;
        if (irap == 0) c0 = c;
      }
      if (!(c0 > 0.0f) || !std::isfinite(csum))
        return fail(FSM_ERR_UNSUPPORTED,
                    "2D BARYON: the first rapidity weight underflows (DRAP * DIM_RAP too wide for SIGMA_B)");
      E.fb_scale2 = (float)(csum / ((double)NR * (double)c0));
      E.jscale2 = (float)NR * c0;
      E.samples *= 2.0;
      E.ref_samples *= 2.0;
    }
    return FSM_OK;
  }

  // ---------------------------------------------------------------- 3D tables
  const float TAU = p.TAU, TAU0 = p.TAU0, DETA = p.DETA;
  {
    float SIGMA = p.SIGMA;
    float n = std::sqrt(M_PI / 2.0) * SIGMA * (1.0 + std::exp(2.0 * SIGMA * SIGMA));
    E.norm = 1.0 / (2.0 * M_PI * n);  // src/FreeStream.cpp:302-303
    float SIGMA_B = p.SIGMA_B;
    float nb = std::sqrt(2.0 * M_PI) * SIGMA_B * std::exp(SIGMA_B * SIGMA_B / 2.0);
    E.normB = 1.0 / (2.0 * M_PI * nb);  // src/FreeStream.cpp:365-366
  }
  E.jac.resize(NR);
  for (int irap = 0; irap < NR; ++irap) {  // src/LandauMatch.cpp:92-93
    float w = tanmap_w(irap, NR);
    E.jac[irap] = (M_PI / 2.0) / std::cos((M_PI / 2.0) * w) / std::cos((M_PI / 2.0) * w) *
                  (1.995 / float(NR - 1));
  }
  E.re.resize((size_t)NE * NR);
  E.rapf.resize((size_t)NE * NR);
  E.rapfB.resize((size_t)NE * NR);
  const float rapmin = (-1.0) * ((float)(NR - 1) / 2.0) * p.DRAP;
  const float SIGMA = p.SIGMA, SIGMA_B = p.SIGMA_B;
  std::vector<int> live_cnt(NR, 0);
  std::vector<char> live_pair((size_t)NE * NR, 0);
  const int plan_threads = (double)NE * NR * NP > 1.0e5 ? host_threads() : 1;
  parallel_for(NE, plan_threads, [&](int ieta) {
    float eta = (float)ieta * DETA + E.etamin;
    for (int irap = 0; irap < NR; ++irap) {
      float w = tanmap_w(irap, NR);
      float rap = eta + std::tan((M_PI / 2.0) * w);
      // streaming step (src/FreeStream.cpp:192-201)
      float eta_new = std::asinh((TAU / TAU0) * std::sinh(eta - rap)) + rap;
      float D = (TAU * std::cosh(rap - eta_new) - TAU0 * std::cosh(rap - eta));
      float ieta_new = (eta_new - E.etamin) / DETA;
      float fl = std::floor(ieta_new);
      RapEta r;
      r.D = D;
      if (std::isfinite(ieta_new) && fl > -1.0e6f && fl < 1.0e6f) {
        r.efl = (int)fl;
        r.efrac = ieta_new - fl;
      } else {
        r.efl = -1;
        r.efrac = 0.0f;
      }
      // hypertrig factors (src/LandauMatch.cpp:46-55) with d = rap - eta
      float d = rap - eta;
      float ch = std::cosh(d), th = std::tanh(d);
      r.A = 1.0f / ch;
      r.B = 1.0f / (ch * ch);
      r.C = (1.0 / TAU) * ((double)th / (double)ch);
      r.Dt = (1.0 / TAU) * std::tanh(rap - eta);
      r.E = (1.0 / (TAU * TAU)) * std::tanh(rap - eta) * std::tanh(rap - eta);
      E.re[(size_t)ieta * NR + irap] = r;
      // rapidity weights of the initial densities (src/FreeStream.cpp:345, 381-382)
      float de = eta - rap;
      E.rapf[(size_t)ieta * NR + irap] =
          std::cosh(de) * std::cosh(de) * std::exp((-1.0) * de * de / (2.0 * SIGMA * SIGMA));
      float rapu = (float)irap * p.DRAP + rapmin;
      float du = eta - rapu;
      E.rapfB[(size_t)ieta * NR + irap] =
          std::cosh(du) * std::exp((-1.0) * du * du / (SIGMA_B * SIGMA_B));
      live_pair[(size_t)ieta * NR + irap] = (r.efl >= 1 && r.efl < NE - 1) && std::isfinite(D) &&
                                             std::fabs(D) <= (float)(NX + NY) * std::max(p.DX, p.DY);
    }
  });
  for (int ieta = 0; ieta < NE; ++ieta)
    for (int irap = 0; irap < NR; ++irap) live_cnt[irap] += live_pair[(size_t)ieta * NR + irap];
  E.r_lo = NR;
  E.r_hi = 0;
  double live_pairs = 0;
  for (int irap = 0; irap < NR; ++irap)
    if (live_cnt[irap] > 0) {
      E.r_lo = std::min(E.r_lo, irap);
      E.r_hi = std::max(E.r_hi, irap + 1);
    }
  if (E.r_lo >= E.r_hi) E.r_lo = E.r_hi = 0;
  for (int irap = E.r_lo; irap < E.r_hi; ++irap)
    for (int ieta = 0; ieta < NE; ++ieta) {
      const RapEta& r = E.re[(size_t)ieta * NR + irap];
      if (r.efl >= 1 && r.efl < NE - 1 && std::isfinite(r.D)) live_pairs += 1;
    }
  E.samples = live_pairs * (double)NX * NY * NP;
  E.ref_samples = (double)p.DIM * NR * NP;
  // 3D stream table: integer offsets and fractions of the shifted points
  // (src/FreeStream.cpp:193-212) for every live (ieta, irap) and phi_p
  E.tab3 = std::make_shared<std::vector<PhiEntry3D>>((size_t)NE * NR * NP, PhiEntry3D{0.0f, 0.0f, 0, 0});
  std::vector<PhiEntry3D>& tab3 = *E.tab3;
  E.live_eta.assign(NE, 0);
  parallel_for(NE, plan_threads, [&](int ieta) {
    for (int irap = E.r_lo; irap < E.r_hi; ++irap) {
      const RapEta& r = E.re[(size_t)ieta * NR + irap];
      if (!(r.efl >= 1 && r.efl < NE - 1 && std::isfinite(r.D))) continue;
      E.live_eta[ieta] += 1;
      for (int k = 0; k < NP; ++k) {
        const float shx = E.cs[k].x * r.D, shy = E.cs[k].y * r.D;  // reference float products
        const double sx = -(double)shx / (double)p.DX, sy = -(double)shy / (double)p.DY;
        const double ox = std::floor(sx), oy = std::floor(sy);
        PhiEntry3D& w = tab3[((size_t)ieta * NR + irap) * NP + k];
        const double t = sx - ox, u = sy - oy;
        w.t = (float)t;
        w.u = (float)u;
        if (!(std::fabs(ox) < 30000.0 && std::fabs(oy) < 30000.0)) {  // far outside any grid
          w.ox = 1 << 20;
          w.oy_near = 0;
          continue;
        }
        w.ox = (int)ox;
        const int nearx = (t < 1e-3 || t > 1.0 - 1e-3) ? 1 : 0;
        const int neary = (u < 1e-3 || u > 1.0 - 1e-3) ? 1 : 0;
        w.oy_near = ((int)oy & 0xffff) | (nearx << 16) | (neary << 17);
      }
    }
  });
  // combined node planes: one per sampled pair (a pair whose shift exceeds
  // the grid's extent has no sample inside and gets none), grouped by the
  // source eta pair they read; the weights are the float products the
  // stream kernel applied per sample before (1 - efrac) rf(efl), efrac rf(efl+1)
  E.plane_of.assign((size_t)NE * NR, -1);
  E.cw_start.assign(NE, 0);
  E.cw.clear();
  for (int efl = 0; efl < NE - 1; ++efl) {
    E.cw_start[efl] = (int)E.cw.size();
    for (int ieta = 0; ieta < NE; ++ieta)
      for (int irap = E.r_lo; irap < E.r_hi; ++irap) {
        const size_t pr = (size_t)ieta * NR + irap;
        const RapEta& r = E.re[pr];
        if (!live_pair[pr] || r.efl != efl) continue;
        const float et = r.efrac, omet = 1.0f - et;
        CombW c;
        c.plane = (int)E.cw.size();
        c.w0 = omet * E.rapf[(size_t)efl * NR + irap];
        c.w1 = et * E.rapf[(size_t)(efl + 1) * NR + irap];
        c.b0 = omet * E.rapfB[(size_t)efl * NR + irap];
        c.b1 = et * E.rapfB[(size_t)(efl + 1) * NR + irap];
        E.plane_of[pr] = c.plane;
        E.cw.push_back(c);
      }
  }
  E.cw_start[NE - 1] = (int)E.cw.size();
  return FSM_OK;
}

}  // namespace fsm

// ------------------------------------------------------------------ C ABI
using namespace fsm;

extern "C" const char* fsm_status_str(fsm_status s) {
  switch (s) {
    case FSM_OK: return "ok";
    case FSM_ERR_INVALID_ARG: return "invalid argument";
    case FSM_ERR_SIZE_MISMATCH: return "input size does not match the grid";
    case FSM_ERR_INVALID_IC: return "not a valid initial condition";
    case FSM_ERR_UNSUPPORTED: return "unsupported parameter combination";
    case FSM_ERR_CUDA: return "CUDA error";
    case FSM_ERR_NO_DEVICE: return "no CUDA device";
    case FSM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case FSM_ERR_FILE: return "file not found";
    case FSM_ERR_BUSY: return "busy";
    case FSM_ERR_TIMEOUT: return "timed out";
    case FSM_ERR_PENDING: return "pending";
    case FSM_ERR_TOO_LARGE: return "request too large";
    case FSM_ERR_CANCELLED: return "cancelled";
  }
  return "unknown status";
}

extern "C" const char* fsm_last_error(void) { return g_last_error.c_str(); }

extern "C" void fsm_params_default(fsm_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  // src/FreestreamMilne.cpp:149-171
  p->OUTPUTFORMAT = 2;
  p->BARYON = 0;
  p->IC_ENERGY = 5;
  p->IC_BARYON = 1;
  p->ETA_WIDTH = 0.5;
  p->ETA_FLAT = 0.5;
  p->SIGMA = 1.0;
  p->SIGMA_B = 1.0;
  p->DIM_X = 101;
  p->DIM_Y = 101;
  p->DIM_ETA = 1;
  p->DIM_RAP = 1;
  p->DIM_PHIP = 51;
  p->DX = 0.1;
  p->DY = 0.1;
  p->DETA = 0.1;
  p->DRAP = 0.2;
  p->DTAU = 0.5;
  p->TAU0 = 0.1;
  p->EOS_TYPE = 1;
  p->E_FREEZE = 1.7;
  p->VISCOUS_MATCHING = 1;
  p->E_DEP_FS = 0;
  p->E_R = 1.0;
  p->TAU_R = 1.0;
  p->ALPHA = 0.0;
  fsm_params_derive(p);
}

extern "C" void fsm_params_derive(fsm_params* p) {
  if (!p) return;
  p->DIM = p->DIM_X * p->DIM_Y * p->DIM_ETA;
  p->TAU = p->TAU0 + p->DTAU;
}

// Positional parse with the reference's own format strings (src/FileIO.cpp:166-245).
extern "C" fsm_status fsm_params_read_file(const char* path, fsm_params* p) {
  if (!path || !p) return FSM_ERR_INVALID_ARG;
  FILE* fileIn = std::fopen(path, "r");
  if (!fileIn) {
    set_last_error(std::string("cannot open parameter file ") + path);
    return FSM_ERR_FILE;
  }
  char dummyChar[255];
  int dummyInt = 0;
  float dummyFloat = 0;
  auto rdi = [&](int* dst) {
    if (std::fscanf(fileIn, "%254s\t%d\n", dummyChar, &dummyInt) == 2) *dst = dummyInt;
  };
  auto rdf = [&](float* dst) {
    if (std::fscanf(fileIn, "%254s\t%f\n", dummyChar, &dummyFloat) == 2) *dst = dummyFloat;
  };
  rdi(&p->OUTPUTFORMAT);
  rdi(&p->BARYON);
  rdi(&p->IC_ENERGY);
  rdi(&p->IC_BARYON);
  rdf(&p->ETA_WIDTH);
  rdf(&p->ETA_FLAT);
  rdf(&p->SIGMA);
  rdf(&p->SIGMA_B);
  rdi(&p->DIM_X);
  rdi(&p->DIM_Y);
  rdi(&p->DIM_ETA);
  rdi(&p->DIM_RAP);
  rdi(&p->DIM_PHIP);
  rdf(&p->DX);
  rdf(&p->DY);
  rdf(&p->DETA);
  rdf(&p->DRAP);
  rdf(&p->DTAU);
  rdf(&p->TAU0);
  rdi(&p->EOS_TYPE);
  rdf(&p->E_FREEZE);
  rdi(&p->VISCOUS_MATCHING);
  rdi(&p->E_DEP_FS);
  rdf(&p->E_R);
  rdf(&p->TAU_R);
  rdf(&p->ALPHA);
  std::fclose(fileIn);
  fsm_params_derive(p);
  return FSM_OK;
}
