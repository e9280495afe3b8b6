// fsm_io.cpp -- text output of per-cell fields in the reference's formats
// (src/FileIO.cpp:11-131), formatted by several host threads into one buffer
// per thread and written with one fwrite each.
//
//   full grid   "x y eta value\n" per cell in the reference cell order, the
//               coordinates rounded to multiples of the spacing
//               (src/FileIO.cpp:29-35 and 59-65);
//   projection  the eta-centre slice, one text row per y with the x values
//               as columns, each value followed by one space
//               (src/FileIO.cpp:86-101 and 115-130).
// Values print like an ostream with default settings (six significant
// digits, %g).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fsm.h"
#include "fsm_plan.h"

namespace fsm {
namespace {

// The reference's rounded coordinate of node i on an axis of n nodes
// (float/double mixing as src/FileIO.cpp:29-30).
float axis_coord(int i, int n, float d) {
  float x = (float)i * d - (((float)(n - 1)) / 2.0 * d);
  return d * roundf(x / d);
}

void append_g(std::string& s, float v) {
  char buf[48];
  int k = std::snprintf(buf, sizeof(buf), "%g", (double)v);
  s.append(buf, (size_t)k);
}

}  // namespace
}  // namespace fsm

namespace fsm {
namespace {

// Formats text rows [u0, u1) of one field: x rows of the full grid, or y rows
// of the eta-centre projection.
void format_rows(std::string& s, const float* var, const fsm_params* p, bool projection, int u0,
                 int u1) {
  const int NX = p->DIM_X, NY = p->DIM_Y, NE = p->DIM_ETA;
  if (projection) {
    const int ieta = (NE - 1) / 2;
    s.reserve(s.size() + (size_t)(u1 - u0) * NX * 12);
    for (int iy = u0; iy < u1; ++iy) {
      for (int ix = 0; ix < NX; ++ix) {
        const size_t is = (size_t)(NY * NE) * ix + (size_t)NE * iy + ieta;
        append_g(s, var[is]);
        s.push_back(' ');
      }
      s.push_back('\n');
    }
    return;
  }
  s.reserve(s.size() + (size_t)(u1 - u0) * NY * NE * 40);
  std::vector<std::string> ys(NY), es(NE);
  for (int iy = 0; iy < NY; ++iy) append_g(ys[iy], axis_coord(iy, NY, p->DY));
  for (int ie = 0; ie < NE; ++ie) append_g(es[ie], axis_coord(ie, NE, p->DETA));
  for (int ix = u0; ix < u1; ++ix) {
    std::string xs;
    append_g(xs, axis_coord(ix, NX, p->DX));
    for (int iy = 0; iy < NY; ++iy)
      for (int ie = 0; ie < NE; ++ie) {
        const size_t is = (size_t)(NY * NE) * ix + (size_t)NE * iy + ie;
        s += xs;
        s.push_back(' ');
        s += ys[iy];
        s.push_back(' ');
        s += es[ie];
        s.push_back(' ');
        append_g(s, var[is]);
        s.push_back('\n');
      }
  }
}

fsm_status write_chunks(const char* path, const std::vector<std::string>& parts) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {  // the reference's ofstream fails silently; report it instead
    set_last_error(std::string("cannot open ") + path);
    return FSM_ERR_FILE;
  }
  bool ok = true;
  for (auto& s : parts) ok = ok && (std::fwrite(s.data(), 1, s.size(), f) == s.size());
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    set_last_error(std::string("write failed for ") + path);
    return FSM_ERR_FILE;
  }
  return FSM_OK;
}

bool valid_grid(const fsm_params* p) { return p && p->DIM_X >= 1 && p->DIM_Y >= 1 && p->DIM_ETA >= 1; }

}  // namespace
}  // namespace fsm

extern "C" fsm_status fsm_write_field(const char* path, const float* var, const fsm_params* p,
                                      int projection, int nthreads) {
  using namespace fsm;
  if (!path || !var || !p) {
    set_last_error("fsm_write_field: null argument");
    return FSM_ERR_INVALID_ARG;
  }
  if (!valid_grid(p)) {
    set_last_error("fsm_write_field: empty grid");
    return FSM_ERR_INVALID_ARG;
  }
  // work unit: one x row (full grid) or one y row (projection)
  const int units = projection ? p->DIM_Y : p->DIM_X;
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, units));
  std::vector<std::string> out(nt);
  auto work = [&](int t) {
    const int u0 = (int)((long long)units * t / nt), u1 = (int)((long long)units * (t + 1) / nt);
    format_rows(out[t], var, p, projection != 0, u0, u1);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  return write_chunks(path, out);
}

// Every per-cell file the reference writes after Landau matching
// (src/FreestreamMilne.cpp:561-673), in its file names, as one job list: the
// files are formatted concurrently, each by one thread, largest first.
extern "C" fsm_status fsm_write_outputs(const char* dir, const fsm_params* p, const fsm_outputs* out,
                                        const fsm_diagnostics* diag, int nthreads) {
  using namespace fsm;
  if (!dir || !out || !valid_grid(p)) {
    set_last_error("fsm_write_outputs: null argument or empty grid");
    return FSM_ERR_INVALID_ARG;
  }
  const size_t n = (size_t)p->DIM_X * p->DIM_Y * p->DIM_ETA;
  struct Job {
    std::string name;
    const float* var;
    bool proj;
  };
  std::vector<Job> jobs;
  auto add = [&](const char* name, const float* base, int comp, bool proj) {
    if (base) jobs.push_back(Job{name, base + (size_t)comp * n, proj});
  };
  if (diag) {  // hydro validity (src/FreestreamMilne.cpp:561-600)
    add("R_Pi_Inv_projection", diag->R_Pi_Inv, 0, true);
    add("R_pimunu_Inv_projection", diag->R_pimunu_Inv, 0, true);
    static const char* pdu[4] = {"pi_dot_u_tau_projection", "pi_dot_u_x_projection",
                                 "pi_dot_u_y_projection", "pi_dot_u_eta_projection"};
    for (int m = 0; m < 4; ++m) add(pdu[m], diag->pi_dot_u, m, true);
    add("pi_mu_mu_projection", diag->pi_mu_mu, 0, true);
  }
  // hydro variables (src/FreestreamMilne.cpp:618-659)
  add("e", out->e, 0, false);
  add("p", out->P, 0, false);
  add("bulk_PI", out->Pi, 0, false);
  add("e_projection", out->e, 0, true);
  add("p_projection", out->P, 0, true);
  add("bulk_PI_projection", out->Pi, 0, true);
  static const char* un[4] = {"ut", "ux", "uy", "un"};
  static const char* unp[4] = {"ut_projection", "ux_projection", "uy_projection", "un_projection"};
  for (int m = 0; m < 4; ++m) add(un[m], out->u, m, false);
  for (int m = 0; m < 4; ++m) add(unp[m], out->u, m, true);
  static const char* pn[10] = {"pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn", "pinn"};
  for (int m = 0; m < 10; ++m) add(pn[m], out->pi, m, false);
  for (int m = 0; m < 10; ++m) add((std::string(pn[m]) + "_projection").c_str(), out->pi, m, true);
  if (diag) {  // thermal vorticity (src/FreestreamMilne.cpp:661-666)
    add("beta_x_projection", diag->beta, 1, true);
    add("beta_x", diag->beta, 1, false);
    add("beta_y_projection", diag->beta, 2, true);
    add("beta_y", diag->beta, 2, false);
    add("w_xy_projection", diag->omega, 3, true);
    add("w_xy", diag->omega, 3, false);
  }
  if (p->BARYON) {  // src/FreestreamMilne.cpp:668-673
    add("nB", out->nB, 0, false);
    add("nB_projection", out->nB, 0, true);
    add("V_x", out->V, 1, false);
    add("V_y", out->V, 2, false);
    add("V_eta", out->V, 3, false);
  }
  std::stable_sort(jobs.begin(), jobs.end(), [](const Job& a, const Job& b) { return !a.proj && b.proj; });
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, (int)jobs.size()));
  std::atomic<int> next{0};
  std::vector<fsm_status> st(jobs.size(), FSM_OK);
  std::vector<std::string> err(jobs.size());
  auto worker = [&]() {
    for (int j; (j = next.fetch_add(1)) < (int)jobs.size();) {
      const Job& J = jobs[j];
      std::vector<std::string> part(1);
      format_rows(part[0], J.var, p, J.proj, 0, J.proj ? p->DIM_Y : p->DIM_X);
      const std::string path = std::string(dir) + "/" + J.name + ".dat";
      st[j] = write_chunks(path.c_str(), part);
      if (st[j] != FSM_OK) err[j] = fsm_last_error();
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(worker);
  worker();
  for (auto& x : th) x.join();
  for (size_t j = 0; j < jobs.size(); ++j)
    if (st[j] != FSM_OK) {
      set_last_error("fsm_write_outputs: " + err[j]);
      return st[j];
    }
  return FSM_OK;
}
