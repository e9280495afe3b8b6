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

extern "C" fsm_status fsm_write_field(const char* path, const float* var, const fsm_params* p,
                                      int projection, int nthreads) {
  using namespace fsm;
  if (!path || !var || !p) {
    set_last_error("fsm_write_field: null argument");
    return FSM_ERR_INVALID_ARG;
  }
  const int NX = p->DIM_X, NY = p->DIM_Y, NE = p->DIM_ETA;
  if (NX < 1 || NY < 1 || NE < 1) {
    set_last_error("fsm_write_field: empty grid");
    return FSM_ERR_INVALID_ARG;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {  // the reference's ofstream fails silently; report it instead
    set_last_error(std::string("fsm_write_field: cannot open ") + path);
    return FSM_ERR_FILE;
  }
  // work unit: one x row (full grid) or one y row (projection)
  const int units = projection ? NY : NX;
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, units));
  std::vector<std::string> out(nt);
  auto work = [&](int t) {
    const int u0 = (int)((long long)units * t / nt), u1 = (int)((long long)units * (t + 1) / nt);
    std::string& s = out[t];
    if (projection) {
      const int ieta = (NE - 1) / 2;
      s.reserve((size_t)(u1 - u0) * NX * 12);
      for (int iy = u0; iy < u1; ++iy) {
        for (int ix = 0; ix < NX; ++ix) {
          const size_t is = (size_t)(NY * NE) * ix + (size_t)NE * iy + ieta;
          append_g(s, var[is]);
          s.push_back(' ');
        }
        s.push_back('\n');
      }
    } else {
      s.reserve((size_t)(u1 - u0) * NY * NE * 40);
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
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  bool ok = true;
  for (auto& s : out) ok = ok && (std::fwrite(s.data(), 1, s.size(), f) == s.size());
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    set_last_error(std::string("fsm_write_field: write failed for ") + path);
    return FSM_ERR_FILE;
  }
  return FSM_OK;
}
