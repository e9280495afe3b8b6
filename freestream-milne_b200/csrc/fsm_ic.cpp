// fsm_ic.cpp -- the reference's initial conditions on the host, producing
// profiles in fm^-4 as its run_freestream_milne uses them
// (src/FreestreamMilne.cpp:225-306, src/InitialConditions.cpp,
// src/FileIO.cpp:133-164): only IC_ENERGY = 5 (the caller's vector in
// GeV/fm^3) is converted by the compute entry points; every other initial
// condition is already in the internal units and goes to fsm_run_event_fm4.
//
// The float/double mixing of each reference expression is spelled out
// (compiled with FMA contraction off), so the profiles are bit-identical to
// the reference's; the Monte-Carlo ones draw from the C library's rand() in
// the reference's order (one draw per cell, cell order).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>

#include "../../include/fsm.h"
#include "fsm_plan.h"

namespace fsm {
namespace {

// Cell coordinate of InitialConditions.cpp: (float)i * d - ((float)(n-1)) / 2.0 * d
// (a float product minus a double product, rounded to float).
float ic_coord(int i, int n, float d) {
  return (float)((double)((float)i * d) - ((double)((float)(n - 1)) / 2.0) * (double)d);
}

struct Cell {
  float x, y, eta;
};
Cell ic_cell(const fsm_params& p, int is) {
  const int ix = is / (p.DIM_Y * p.DIM_ETA);
  const int iy = (is - (p.DIM_Y * p.DIM_ETA * ix)) / p.DIM_ETA;
  const int ieta = is - (p.DIM_Y * p.DIM_ETA * ix) - (p.DIM_ETA * iy);
  return Cell{ic_coord(ix, p.DIM_X, p.DX), ic_coord(iy, p.DIM_Y, p.DY), ic_coord(ieta, p.DIM_ETA, p.DETA)};
}

// e0 exp(-x^2/bx) exp(-y^2/by) exp(-eta^2/beta), e0 = 500 fm^-4
// (initializeEllipticalGauss, InitialConditions.cpp:46-71); with mc, times a
// rand() draw after e0 (initializeEllipticalMCGauss, :100-125).
void elliptical_gauss(const fsm_params& p, float bx, float by, float beta, bool mc, float* out) {
  const float e0 = 500.0;
  const int DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA;
  for (int is = 0; is < DIM; is++) {
    const Cell c = ic_cell(p, is);
    const double gx = std::exp(-(1.0 / bx) * (double)(c.x * c.x));
    const double gy = std::exp(-(1.0 / by) * (double)(c.y * c.y));
    const double ge = std::exp(-(1.0 / beta) * (double)(c.eta * c.eta));
    float a = e0;
    if (mc) a = e0 * ((float)std::rand() / RAND_MAX);
    out[is] = (float)((double)a * gx * gy * ge);
  }
}

// Two Gaussians at x = +-3 times a rand() draw per cell; the reference's
// norm is 0, so the profile is zero (initialize2Gaussians, :238-272); the
// draws are still taken, as the reference takes them.
void two_gaussians(const fsm_params& p, float* out) {
  const float e0 = 0.0;
  const float bx = 1.0f, by = 1.0f, beta = 1.0f;
  const int DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA;
  for (int is = 0; is < DIM; is++) {
    const Cell c = ic_cell(p, is);
    const float x1 = 3.0, y1 = 0.0, eta1 = 0.0, x2 = -3.0, y2 = 0.0, eta2 = 0.0;
    const double g1 = std::exp(-(1.0 / bx) * (double)((c.x - x1) * (c.x - x1))) *
                      std::exp(-(1.0 / by) * (double)((c.y - y1) * (c.y - y1))) *
                      std::exp(-(1.0 / beta) * (double)((c.eta - eta1) * (c.eta - eta1)));
    const double g2 = std::exp(-(1.0 / bx) * (double)((c.x - x2) * (c.x - x2))) *
                      std::exp(-(1.0 / by) * (double)((c.y - y2) * (c.y - y2))) *
                      std::exp(-(1.0 / beta) * (double)((c.eta - eta2) * (c.eta - eta2)));
    out[is] = (float)((double)e0 * (g1 + g2));
    out[is] *= ((float)std::rand() / RAND_MAX);
  }
}

// Longitudinal plateau of the block readers (:163-177): the transverse value
// times exp(-(|eta| - ETA_FLAT)^2 / (2 ETA_WIDTH^2)) beyond the plateau, plus
// 1e-3.
void eta_plateau(const fsm_params& p, float* out) {
  const float lower_tolerance = 1.0e-3;
  const int DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA;
  for (int is = 0; is < DIM; is++) {
    const int ix = is / (p.DIM_Y * p.DIM_ETA);
    const int iy = (is - (p.DIM_Y * p.DIM_ETA * ix)) / p.DIM_ETA;
    const int ieta = is - (p.DIM_Y * p.DIM_ETA * ix) - (p.DIM_ETA * iy);
    const float eta = ic_coord(ieta, p.DIM_ETA, p.DETA);
    const float d = std::fabs(eta) - p.ETA_FLAT;
    // (-1.0) * d * d / (2.0 * W * W) in double, left to right; exp of the
    // float argument in float
    float arg = (float)(((-1.0) * (double)d) * (double)d / ((2.0 * (double)p.ETA_WIDTH) * (double)p.ETA_WIDTH));
    arg = arg * (d < 0.0f ? 0.0f : 1.0f);
    out[is] = out[is] * std::exp(arg) + lower_tolerance;
  }
}

fsm_status missing(const std::string& path) {
  set_last_error("cannot open initial profile " + path);
  return FSM_ERR_FILE;
}

}  // namespace
}  // namespace fsm

extern "C" fsm_status fsm_read_profile(const char* path, const fsm_params* p, int format, float* out) {
  using namespace fsm;
  if (!path || !p || !out || p->DIM_X < 1 || p->DIM_Y < 1 || p->DIM_ETA < 1) return FSM_ERR_INVALID_ARG;
  const int NX = p->DIM_X, NY = p->DIM_Y, NE = p->DIM_ETA;
  std::ifstream in(path);
  if (!in) return missing(path);
  auto at = [&](int ix, int iy, int ie) -> float& {
    return out[(size_t)(NY * NE) * ix + (size_t)NE * iy + ie];
  };
  float v = 0.0f, dummy = 0.0f;
  switch (format) {
    case FSM_PROFILE_XYEV: {  // readDensityFile, FileIO.cpp:133-164
      const float xmin = (-1.0) * ((float)(NX - 1) / 2.0) * p->DX;
      const float ymin = (-1.0) * ((float)(NY - 1) / 2.0) * p->DY;
      const float etamin = (-1.0) * ((float)(NE - 1) / 2.0) * p->DETA;
      float x, y, eta;
      while (in >> x >> y >> eta >> v) {
        const int ix = (int)std::round((x - xmin) / p->DX);
        const int iy = (int)std::round((y - ymin) / p->DY);
        const int ie = (int)std::round((eta - etamin) / p->DETA);
        const long long is = (long long)(NY * NE) * ix + (long long)NE * iy + ie;
        if (is >= 0 && is < (long long)NX * NY * NE) out[is] = v;  // the reference writes unchecked
      }
      return FSM_OK;
    }
    case FSM_PROFILE_CPUVH:  // readEnergyDensityCPUVH, InitialConditions.cpp:316-355
      for (int ie = 0; ie < NE; ie++)
        for (int iy = 0; iy < NY; iy++)
          for (int ix = 0; ix < NX; ix++) {
            in >> dummy >> dummy >> dummy >> v;
            at(ix, iy, ie) = v * 1.0f + 1.0e-7f;
          }
      return FSM_OK;
    case FSM_PROFILE_SUPERMC_BLOCK:  // readEnergyDensitySuperMCBlock, :127-179
      for (int ix = 0; ix < NX; ix++)
        for (int iy = 0; iy < NY; iy++) {
          in >> v;
          for (int ie = 0; ie < NE; ie++) at(ix, iy, ie) = v;
        }
      eta_plateau(*p, out);
      return FSM_OK;
    case FSM_PROFILE_TRENTO_BLOCK: {  // readEnergyDensityTRENTOBlock, :181-236 (12 header lines)
      std::string line;
      for (int l = 0; l < 12; l++) std::getline(in, line);
      for (int iy = 0; iy < NY; iy++)
        for (int ix = 0; ix < NX; ix++) {
          in >> v;
          for (int ie = 0; ie < NE; ie++) at(ix, iy, ie) = v;
        }
      eta_plateau(*p, out);
      return FSM_OK;
    }
    case FSM_PROFILE_TRENTO3D_BLOCK:  // readEnergyDensityTRENTO3DBlock, :274-314
      for (int ix = 0; ix < NX; ix++)
        for (int iy = 0; iy < NY; iy++)
          for (int ie = 0; ie < NE; ie++) {
            in >> v;
            at(ix, iy, ie) = v + 1.0e-3f;
          }
      return FSM_OK;
    default:
      set_last_error("fsm_read_profile: unknown format");
      return FSM_ERR_INVALID_ARG;
  }
}

extern "C" fsm_status fsm_initial_energy(const fsm_params* p, const char* dir, float* e_fm4) {
  using namespace fsm;
  if (!p || !e_fm4) return FSM_ERR_INVALID_ARG;
  const std::string d = dir ? dir : "initial_profiles";
  switch (p->IC_ENERGY) {  // src/FreestreamMilne.cpp:231-281
    case 1:
      elliptical_gauss(*p, 15.0f, 15.0f, 15.0f, false, e_fm4);
      return FSM_OK;
    case 2:
      elliptical_gauss(*p, 15.0f, 15.0f, 15.0f, true, e_fm4);
      return FSM_OK;
    case 3:
      return fsm_read_profile((d + "/e.dat").c_str(), p, FSM_PROFILE_XYEV, e_fm4);
    case 4:
      return fsm_read_profile((d + "/e.dat").c_str(), p, FSM_PROFILE_CPUVH, e_fm4);
    case 6:
      two_gaussians(*p, e_fm4);
      return FSM_OK;
    default:  // 5: the caller's vector (GeV/fm^3, fsm_run_event); others: invalid
      set_last_error("fsm_initial_energy: IC_ENERGY " + std::to_string(p->IC_ENERGY) +
                     " is not an initial condition of the library (5: the caller's vector)");
      return FSM_ERR_INVALID_IC;
  }
}

extern "C" fsm_status fsm_initial_baryon(const fsm_params* p, const char* dir, float* nB) {
  using namespace fsm;
  if (!p || !nB) return FSM_ERR_INVALID_ARG;
  const std::string d = dir ? dir : "initial_profiles";
  switch (p->IC_BARYON) {  // src/FreestreamMilne.cpp:287-306
    case 1:
      elliptical_gauss(*p, 2.0f, 3.0f, 1.0f, false, nB);
      return FSM_OK;
    case 2:
      elliptical_gauss(*p, 2.0f, 3.0f, 1.0f, true, nB);
      return FSM_OK;
    case 3:
      return fsm_read_profile((d + "/nB.dat").c_str(), p, FSM_PROFILE_XYEV, nB);
    default:
      set_last_error("fsm_initial_baryon: IC_BARYON " + std::to_string(p->IC_BARYON) + " is not valid");
      return FSM_ERR_INVALID_IC;
  }
}
