// FreestreamMilne.cpp -- drop-in FREESTREAMMILNE class over libfsm.
//
// The same public interface as the reference's class (src/FreestreamMilne.cpp:
// 28-87), delivered the same way: one translation unit that callers include
// (src/RunWrapper.cpp:1).  run_freestream_milne() keeps the reference's
// behaviour around the compute -- freestream_input is read from the working
// directory with the same defaults and positional format, the initial profile
// comes from the vector (IC_ENERGY = 5) or from initial_profiles/*.dat
// (IC_ENERGY = 3, IC_BARYON = 3), the output/*.dat files and the final_*
// vectors are written in the reference's formats and units -- while the free
// streaming, moments and Landau matching run on the GPU through the C ABI of
// include/fsm.h.  Build: add this directory and include/ to the include path,
// link -lfsm -lcudart.
//
// Differences a caller sees: the initial-condition generators (IC_ENERGY 1, 2,
// 4, 6; IC_BARYON 1, 2) are not part of this build and are reported as an
// invalid initial condition (return 0, as the reference does for unknown
// values); a GPU-side failure prints the library's message and returns a
// non-zero status instead of aborting.
#ifndef FSM_COMPAT_FREESTREAMMILNE_
#define FSM_COMPAT_FREESTREAMMILNE_

#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "fsm.h"

class FREESTREAMMILNE {
 private:
  fsm_ctx* ctx_ = nullptr;

 public:
  FREESTREAMMILNE();
  ~FREESTREAMMILNE();

  int run_freestream_milne();

  int gridSize;  // the total number of grid points in x, y and eta

  // the free-streaming (Landau matching) time
  float tau_LandauMatch;

  // initial energy density in GeV / fm^3
  void initialize_from_vector(std::vector<float>);
  std::vector<float> init_energy_density;

  // final hydro variables (energy density and stresses in GeV / fm^3)
  void output_to_vectors(std::vector<double>&,   // e
                         std::vector<double>&,   // p
                         std::vector<double>&,   // ut
                         std::vector<double>&,   // ux
                         std::vector<double>&,   // uy
                         std::vector<double>&,   // un
                         std::vector<double>&,   // pitt
                         std::vector<double>&,   // pitx
                         std::vector<double>&,   // pity
                         std::vector<double>&,   // pitn
                         std::vector<double>&,   // pixx
                         std::vector<double>&,   // pixy
                         std::vector<double>&,   // pixn
                         std::vector<double>&,   // piyy
                         std::vector<double>&,   // piyn
                         std::vector<double>&,   // pinn
                         std::vector<double>&);  // Pi

  std::vector<double> final_energy_density;
  std::vector<double> final_pressure;
  std::vector<double> final_ut;
  std::vector<double> final_ux;
  std::vector<double> final_uy;
  std::vector<double> final_un;
  std::vector<double> final_pitt;
  std::vector<double> final_pitx;
  std::vector<double> final_pity;
  std::vector<double> final_pitn;
  std::vector<double> final_pixx;
  std::vector<double> final_pixy;
  std::vector<double> final_pixn;
  std::vector<double> final_piyy;
  std::vector<double> final_piyn;
  std::vector<double> final_pinn;
  std::vector<double> final_Pi;
};

inline FREESTREAMMILNE::FREESTREAMMILNE() : gridSize(0), tau_LandauMatch(0.0f) {}

inline FREESTREAMMILNE::~FREESTREAMMILNE() {
  if (ctx_) fsm_ctx_destroy(ctx_);
}

inline void FREESTREAMMILNE::initialize_from_vector(std::vector<float> energy_density_in) {
  init_energy_density = energy_density_in;
}

inline void FREESTREAMMILNE::output_to_vectors(
    std::vector<double>& e, std::vector<double>& p, std::vector<double>& ut, std::vector<double>& ux,
    std::vector<double>& uy, std::vector<double>& un, std::vector<double>& pitt,
    std::vector<double>& pitx, std::vector<double>& pity, std::vector<double>& pitn,
    std::vector<double>& pixx, std::vector<double>& pixy, std::vector<double>& pixn,
    std::vector<double>& piyy, std::vector<double>& piyn, std::vector<double>& pinn,
    std::vector<double>& Pi) {
  e = final_energy_density;
  p = final_pressure;
  ut = final_ut;
  ux = final_ux;
  uy = final_uy;
  un = final_un;
  pitt = final_pitt;
  pitx = final_pitx;
  pity = final_pity;
  pitn = final_pitn;
  pixx = final_pixx;
  pixy = final_pixy;
  pixn = final_pixn;
  piyy = final_piyy;
  piyn = final_piyn;
  pinn = final_pinn;
  Pi = final_Pi;
}

namespace fsm_compat {

inline void write_field(const std::vector<float>& v, size_t off, const char* name,
                        const fsm_params& p, bool projection) {
  const std::string path = std::string("output/") + name + ".dat";
  // the reference's ofstream fails silently when output/ is missing
  if (fsm_write_field(path.c_str(), v.data() + off, &p, projection ? 1 : 0, 0) != FSM_OK) return;
}

}  // namespace fsm_compat

inline int FREESTREAMMILNE::run_freestream_milne() {
  using namespace fsm_compat;
  const float hbarc = 0.197326938;

  fsm_params params;
  fsm_params_default(&params);  // src/FreestreamMilne.cpp:149-171
  if (fsm_params_read_file("freestream_input", &params) == FSM_ERR_FILE)
    printf("Couldn't open parameters.dat . Using default values!\n");
  fsm_params_derive(&params);
  const int DIM = params.DIM;
  gridSize = DIM;

  // initial energy density and baryon density (src/FreestreamMilne.cpp:225-306):
  // the caller's vector in GeV/fm^3 (IC_ENERGY 5, converted by fsm_run_event),
  // or one of the reference's initial conditions, already in fm^-4
  std::vector<float> e_in((size_t)DIM, 0.0f), nB;
  const bool from_vector = params.IC_ENERGY == 5;
  if (from_vector) {
    if ((size_t)params.DIM != init_energy_density.size()) {
      printf("Grid dimension of input vector does not match freestream_input file! \n");
      printf("Vector size : %d , DIM = %d \n", (int)init_energy_density.size(), params.DIM);
      exit(-1);
    }
    e_in = init_energy_density;
  } else {
    const fsm_status ic = fsm_initial_energy(&params, "initial_profiles", e_in.data());
    if (ic == FSM_ERR_INVALID_IC) {
      printf("Not a valid initial Condition... Goodbye\n");
      return 0;
    }
    if (ic == FSM_ERR_FILE && params.IC_ENERGY == 3) {  // src/FileIO.cpp:150-154
      printf("Couldn't open initial profile!\n");
      exit(1);
    }
    if (ic == FSM_ERR_FILE)  // IC 4: the reference prints and goes on with zeros
      printf("Could not find initial profile in initial_profiles!");
  }
  if (params.BARYON) {
    nB.assign((size_t)DIM, 0.0f);
    const fsm_status ic = fsm_initial_baryon(&params, "initial_profiles", nB.data());
    if (ic == FSM_ERR_INVALID_IC) {
      printf("Not a valid initial Condition... Goodbye\n");
      return 0;
    }
    if (ic == FSM_ERR_FILE) {
      printf("Couldn't open initial profile!\n");
      exit(1);
    }
  }

  // initial profiles in fm^-4 as the reference writes them
  // (src/FreestreamMilne.cpp:266-267, 310-313)
  {
    std::vector<float> e0(e_in);
    if (from_vector)
      for (int i = 0; i < DIM; ++i) e0[i] = e_in[i] * 1.0f / (float)hbarc + 1.0e-7f;
    write_field(e0, 0, "initial_e", params, false);
    if (params.BARYON) write_field(nB, 0, "initial_nB", params, false);
    write_field(e0, 0, "initial_e_projection", params, true);
    if (params.BARYON) write_field(nB, 0, "initial_nB_projection", params, true);
  }

  // total energy before streaming (src/FreestreamMilne.cpp:349-354): float
  // running sum of the profile in fm^-4, in cell order
  {
    float totalEnergy = 0.0;
    for (int is = 0; is < DIM; is++)
      totalEnergy += from_vector ? e_in[is] * 1.0f / (float)hbarc + 1.0e-7f : e_in[is];
    if (params.DIM_ETA > 1) totalEnergy *= (params.TAU0 * params.DX * params.DY * params.DETA);
    else totalEnergy *= (params.DX * params.DY);
    printf("Total energy on grid before streaming : %f \n", totalEnergy);
  }

  if (!ctx_ && fsm_ctx_create(&ctx_, nullptr) != FSM_OK) {
    printf("freestream-milne: %s\n", fsm_last_error());
    return 1;
  }
  const size_t n = (size_t)DIM;
  std::vector<float> T(10 * n), J, e(n), P(n), Pi(n), u(4 * n), pi(10 * n), nBo, V;
  if (params.BARYON) {
    J.resize(4 * n);
    nBo.resize(n);
    V.resize(4 * n);
  }
  fsm_outputs out = {T.data(), params.BARYON ? J.data() : nullptr, e.data(), P.data(), Pi.data(),
                     u.data(), pi.data(), params.BARYON ? nBo.data() : nullptr,
                     params.BARYON ? V.data() : nullptr};
  fsm_run_info info;
  const fsm_status st = from_vector
                            ? fsm_run_event(ctx_, &params, e_in.data(), params.BARYON ? nB.data() : nullptr,
                                            &out, &info)
                            : fsm_run_event_fm4(ctx_, &params, e_in.data(),
                                                params.BARYON ? nB.data() : nullptr, &out, &info);
  if (st != FSM_OK) {
    printf("freestream-milne: %s: %s\n", fsm_status_str(st), fsm_last_error());
    return 1;
  }
  tau_LandauMatch = info.tau;  // src/FreestreamMilne.cpp:326
  params.DTAU = info.dtau;
  params.TAU = info.tau;
  params.DIM_PHIP = info.dim_phip;

  // energy bookkeeping (src/FreestreamMilne.cpp:533-559)
  {
    float totalEnergyAfter = 0.0, inside = 0.0;
    for (int is = 0; is < DIM; is++) totalEnergyAfter += T[is];
    const float vol = (params.DIM_ETA > 1) ? params.TAU * params.DX * params.DY * params.DETA
                                           : params.TAU * params.DX * params.DY;
    totalEnergyAfter *= vol;
    printf("Total energy on grid after streaming : %f \n", totalEnergyAfter);
    for (int is = 0; is < DIM; is++)
      if ((e[is] * hbarc) > params.E_FREEZE) inside += T[is];
    inside *= vol;
    printf("Fraction of energy contained in Freezeout Hypersurface : %f \n", inside / totalEnergyAfter);
    std::ofstream f("output/energy_inside_switch_surf.dat");
    f << inside * hbarc << std::endl;
  }

  // hydro validity and thermal vorticity (src/FreestreamMilne.cpp:561-615),
  // computed on the GPU from the matched fields
  std::vector<float> dg(17 * n);
  fsm_diagnostics hdg = {dg.data(), dg.data() + n, dg.data() + 2 * n, dg.data() + 6 * n,
                         dg.data() + 7 * n, dg.data() + 11 * n};
  {
    fsm_outputs hin = {nullptr, nullptr, e.data(), P.data(), Pi.data(), u.data(), pi.data(),
                       nullptr, nullptr};
    if (fsm_diagnostics_host(ctx_, &params, &hin, &hdg) != FSM_OK) {
      printf("freestream-milne: %s\n", fsm_last_error());
      return 1;
    }
    const int ctr = (params.DIM_Y * params.DIM_ETA * ((params.DIM_X - 1) / 2)) +
                    (params.DIM_ETA * ((params.DIM_Y - 1) / 2)) + ((params.DIM_ETA - 1) / 2);
    printf("R_Pi_Inv at center : %f \n", dg[ctr]);
    printf("R_pimunu_Inv at center : %f \n", dg[n + ctr]);
  }

  // every output file of src/FreestreamMilne.cpp:561-673 in one call, the
  // files formatted concurrently (the reference's ofstream fails silently when
  // output/ is missing; so does this class)
  fsm_write_outputs("output", &params, &out, &hdg, 0);

  // vectors for the caller, GeV / fm^3 (src/FreestreamMilne.cpp:677-718)
  std::vector<double>* vs[17] = {&final_energy_density, &final_pressure, &final_ut, &final_ux,
                                 &final_uy, &final_un, &final_pitt, &final_pitx, &final_pity,
                                 &final_pitn, &final_pixx, &final_pixy, &final_pixn, &final_piyy,
                                 &final_piyn, &final_pinn, &final_Pi};
  for (auto* v : vs) v->resize(n);
  if ((params.OUTPUTFORMAT == 2) || (params.OUTPUTFORMAT == 3)) {
    for (size_t is = 0; is < n; is++) {
      final_energy_density[is] = (double)e[is] * hbarc;
      final_pressure[is] = (double)P[is] * hbarc;
      final_ut[is] = (double)u[is];
      final_ux[is] = (double)u[n + is];
      final_uy[is] = (double)u[2 * n + is];
      final_un[is] = (double)u[3 * n + is];
      for (int m = 0; m < 10; ++m) (*vs[6 + m])[is] = (double)pi[m * n + is] * hbarc;
      final_Pi[is] = (double)Pi[is] * hbarc;
    }
  }
  return 0;
}

#endif  // FSM_COMPAT_FREESTREAMMILNE_
