// ref_harness.cpp -- TEST INFRASTRUCTURE.  Compiles the freestream-milne
// reference's own, unmodified sources (the single translation unit rooted at
// src/FreestreamMilne.cpp) against the project's GSL-API stand-in
// (gslshim/gsl/*.h) and exposes its hot path to the tests through a C ABI.
//
// Built by oracle/Makefile into oracle/_ref/ only where the reference sources
// are present; never part of the product.  GSL itself is absent on this
// machine, so results are "the reference's loops with the project's spline and
// eigensolver", which pins everything except GSL's internals.
#include "FreestreamMilne.cpp"  // reference: src/FreestreamMilne.cpp (via -I <reference>/src)

#include <unistd.h>

#include <cstring>

#include "fsm_oracle.h"

static_assert(sizeof(oracle_params) == sizeof(parameters), "parameter layout must match");

// ref_run_fm4 passes a profile already in fm^-4 (used as is, as the
// reference uses its own initial conditions, src/FreestreamMilne.cpp:231-281).
static bool g_ref_raw_input = false;

// Runs the pipeline of src/FreestreamMilne.cpp:251-506 on the given inputs by
// calling the reference's own functions in the reference's order.
extern "C" int ref_run(const oracle_params* pin, const float* e_gev, const float* nB_in,
                       oracle_out* out) {
  parameters params;
  std::memcpy(&params, pin, sizeof(params));
  params.DIM = params.DIM_X * params.DIM_Y * params.DIM_ETA;
  params.TAU = params.TAU0 + params.DTAU;
  const int DIM = params.DIM;
  float hbarc = 0.197326938;
  float lower_tolerance = 1.0e-7;
  float rescale = 1.0;

  float* initialEnergyDensity = (float*)calloc(params.DIM, sizeof(float));
  for (int i = 0; i < DIM; i++)
    initialEnergyDensity[i] =
        g_ref_raw_input ? e_gev[i] : e_gev[i] * rescale / (float)hbarc + lower_tolerance;
  float* initialChargeDensity = NULL;
  if (params.BARYON) {
    initialChargeDensity = (float*)calloc(params.DIM, sizeof(float));
    for (int i = 0; i < DIM; i++) initialChargeDensity[i] = nB_in[i];
  }
  if (params.E_DEP_FS == 1) {
    float tau_fs = getEnergyDependentTau(initialEnergyDensity, params);
    params.DTAU = tau_fs;
    params.TAU = params.TAU0 + params.DTAU;
  }
  float min_dx_dy = min(params.DX, params.DY);
  int nphip = int(ceil((2.0 * M_PI * params.DTAU) / min_dx_dy));
  params.DIM_PHIP = max(params.DIM_PHIP, nphip);
  out->dim_phip = params.DIM_PHIP;
  out->dtau = params.DTAU;
  out->tau = params.TAU;

  float** density = NULL;
  density = calloc2dArrayf(density, params.DIM, params.DIM_RAP);
  float** chargeDensity = NULL;
  if (params.BARYON) chargeDensity = calloc2dArrayf(chargeDensity, params.DIM, params.DIM_RAP);
  convertInitialDensity(initialEnergyDensity, density, params);
  free(initialEnergyDensity);
  if (params.BARYON) convertInitialChargeDensity(initialChargeDensity, chargeDensity, params);
  if (params.BARYON) free(initialChargeDensity);

  float*** shiftedDensity = NULL;
  shiftedDensity = calloc3dArrayf(shiftedDensity, params.DIM, params.DIM_RAP, params.DIM_PHIP);
  float*** shiftedChargeDensity = NULL;
  if (params.BARYON)
    shiftedChargeDensity =
        calloc3dArrayf(shiftedChargeDensity, params.DIM, params.DIM_RAP, params.DIM_PHIP);
  freeStream(density, shiftedDensity, params);
  free2dArrayf(density, params.DIM);
  if (params.BARYON) freeStream(chargeDensity, shiftedChargeDensity, params);
  if (params.BARYON) free2dArrayf(chargeDensity, params.DIM);

  float** stressTensor = NULL;
  stressTensor = calloc2dArrayf(stressTensor, 10, params.DIM);
  float** baryonCurrent = NULL;
  if (params.BARYON) baryonCurrent = calloc2dArrayf(baryonCurrent, 4, params.DIM);
  float**** hypertrigTable = NULL;
  hypertrigTable =
      calloc4dArrayf(hypertrigTable, 10, params.DIM_RAP, params.DIM_PHIP, params.DIM_ETA);
  calculateHypertrigTable(hypertrigTable, params);
  calculateStressTensor(stressTensor, shiftedDensity, hypertrigTable, params);
  free3dArrayf(shiftedDensity, params.DIM, params.DIM_RAP);
  if (params.BARYON) {
    calculateBaryonCurrent(baryonCurrent, shiftedChargeDensity, hypertrigTable, params);
    free3dArrayf(shiftedChargeDensity, params.DIM, params.DIM_RAP);
  }
  free4dArrayf(hypertrigTable, 10, params.DIM_RAP, params.DIM_PHIP);

  float* energyDensity = (float*)calloc(params.DIM, sizeof(float));
  float* baryonDensity = NULL;
  if (params.BARYON) baryonDensity = (float*)calloc(params.DIM, sizeof(float));
  float** flowVelocity = NULL;
  flowVelocity = calloc2dArrayf(flowVelocity, 4, params.DIM);
  float* pressure = (float*)calloc(params.DIM, sizeof(float));
  float* bulkPressure = (float*)calloc(params.DIM, sizeof(float));
  float** shearTensor = NULL;
  shearTensor = calloc2dArrayf(shearTensor, 10, params.DIM);
  float** baryonDiffusion = NULL;
  if (params.BARYON) baryonDiffusion = calloc2dArrayf(baryonDiffusion, 4, params.DIM);

  solveEigenSystem(stressTensor, energyDensity, flowVelocity, params);
  if (params.BARYON) {
    calculateBaryonDensity(baryonDensity, baryonCurrent, flowVelocity, params);
    calculateBaryonDiffusion(baryonDiffusion, baryonCurrent, baryonDensity, flowVelocity, params);
  }
  calculatePressure(energyDensity, baryonDensity, pressure, params);
  if (params.VISCOUS_MATCHING) {
    calculateBulkPressure(stressTensor, energyDensity, pressure, bulkPressure, params);
    calculateShearViscTensor(stressTensor, energyDensity, flowVelocity, pressure, bulkPressure,
                             shearTensor, params);
  }

  int nfb = 0;
  for (int is = 0; is < DIM; ++is) {
    if (out->T)
      for (int v = 0; v < 10; ++v) out->T[(size_t)v * DIM + is] = stressTensor[v][is];
    if (out->J && params.BARYON)
      for (int v = 0; v < 4; ++v) out->J[(size_t)v * DIM + is] = baryonCurrent[v][is];
    if (out->e) out->e[is] = energyDensity[is];
    if (out->P) out->P[is] = pressure[is];
    if (out->Pi) out->Pi[is] = bulkPressure[is];
    if (out->u)
      for (int v = 0; v < 4; ++v) out->u[(size_t)v * DIM + is] = flowVelocity[v][is];
    if (out->pi)
      for (int v = 0; v < 10; ++v) out->pi[(size_t)v * DIM + is] = shearTensor[v][is];
    if (out->nB && params.BARYON) out->nB[is] = baryonDensity[is];
    if (out->V && params.BARYON)
      for (int v = 0; v < 4; ++v) out->V[(size_t)v * DIM + is] = baryonDiffusion[v][is];
    if (energyDensity[is] == 1.0e-3f && flowVelocity[0][is] == 1.0f && flowVelocity[1][is] == 0.0f &&
        flowVelocity[2][is] == 0.0f && flowVelocity[3][is] == 0.0f)
      ++nfb;
  }
  out->n_fallback = nfb;

  free2dArrayf(stressTensor, 10);
  free(energyDensity);
  free2dArrayf(flowVelocity, 4);
  free(pressure);
  free(bulkPressure);
  free2dArrayf(shearTensor, 10);
  if (params.BARYON) {
    free2dArrayf(baryonCurrent, 4);
    free(baryonDensity);
    free2dArrayf(baryonDiffusion, 4);
  }
  return 0;
}

// Runs the reference's public entry point end to end (FREESTREAMMILNE, i.e.
// src/FreestreamMilne.cpp:97-136,139-741) inside `workdir`, which must hold a
// `freestream_input` file and an `output/` directory.  out17 receives the 17
// output_to_vectors arrays (each n doubles) in the reference's argument order.
extern "C" int ref_run_full(const char* workdir, const float* e_gev, int n, double* out17) {
  char old[4096];
  if (!getcwd(old, sizeof(old))) return 1;
  if (chdir(workdir) != 0) return 2;
  FREESTREAMMILNE fs;
  std::vector<float> v(e_gev, e_gev + n);
  fs.initialize_from_vector(v);
  int rc = fs.run_freestream_milne();
  std::vector<double> o[17];
  fs.output_to_vectors(o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8], o[9], o[10], o[11],
                       o[12], o[13], o[14], o[15], o[16]);
  for (int k = 0; k < 17; ++k)
    for (int i = 0; i < n && i < (int)o[k].size(); ++i) out17[(size_t)k * n + i] = o[k][i];
  if (chdir(old) != 0) return 3;
  return rc;
}

extern "C" int ref_run_fm4(const oracle_params* pin, const float* e_fm4, const float* nB_in,
                           oracle_out* out) {
  g_ref_raw_input = true;
  const int rc = ref_run(pin, e_fm4, nB_in, out);
  g_ref_raw_input = false;
  return rc;
}

// The reference's own diagnostic functions (src/HydroValidity.cpp:8-101,
// src/LandauMatch.cpp:395-489) on given Landau-matched fields; out as
// oracle_diagnostics.
extern "C" void ref_diagnostics(const oracle_params* pin, float tau, const float* e, const float* P,
                                const float* Pi, const float* u, const float* pi, float* out) {
  parameters params;
  std::memcpy(&params, pin, sizeof(params));
  params.DIM = params.DIM_X * params.DIM_Y * params.DIM_ETA;
  params.TAU = tau;
  const int n = params.DIM;
  std::vector<float> ev(e, e + n), Pv(P, P + n), Piv(Pi, Pi + n);
  float** uu = calloc2dArrayf(nullptr, 4, n);
  float** sh = calloc2dArrayf(nullptr, 10, n);
  for (int m = 0; m < 4; ++m) std::memcpy(uu[m], u + (size_t)m * n, n * 4);
  for (int m = 0; m < 10; ++m) std::memcpy(sh[m], pi + (size_t)m * n, n * 4);
  float* o = out;
  std::fill(o, o + (size_t)17 * n, 0.0f);
  calculateBulkInvReynolds(Pv.data(), Piv.data(), o, params);
  calculateShearInvReynolds(ev.data(), Pv.data(), sh, o + n, params);
  calculate_pi_dot_u(uu, sh, o + 2 * n, o + 3 * n, o + 4 * n, o + 5 * n, params);
  calculate_pi_mu_mu(sh, o + 6 * n, params);
  float** beta = calloc2dArrayf(nullptr, 4, n);
  float** om = calloc2dArrayf(nullptr, 6, n);
  calculateThermalVorticityTensor(ev.data(), uu, beta, om, params);
  for (int m = 0; m < 4; ++m) std::memcpy(o + (size_t)(7 + m) * n, beta[m], n * 4);
  for (int m = 0; m < 6; ++m) std::memcpy(o + (size_t)(11 + m) * n, om[m], n * 4);
  free2dArrayf(uu, 4);
  free2dArrayf(sh, 10);
  free2dArrayf(beta, 4);
  free2dArrayf(om, 6);
}

// The reference's own writers (src/FileIO.cpp:11-131) called in the order of
// src/FreestreamMilne.cpp:561-673 on given host fields, inside `workdir`
// (which must hold an output/ directory).  diag17: R_Pi_Inv, R_pimunu_Inv,
// pi_dot_u (4), pi_mu_mu, beta (4), omega (6), each n floats.
extern "C" int ref_write_outputs(const char* workdir, const oracle_params* pin, const float* e,
                                 const float* P, const float* Pi, const float* u, const float* pi,
                                 const float* nB, const float* V, const float* diag17) {
  char old[4096];
  if (!getcwd(old, sizeof(old))) return 1;
  if (chdir(workdir) != 0) return 2;
  parameters params;
  std::memcpy(&params, pin, sizeof(params));
  params.DIM = params.DIM_X * params.DIM_Y * params.DIM_ETA;
  const int n = params.DIM;
  auto vec2d = [&](const float* src, int comps) {
    float** a = calloc2dArrayf(nullptr, comps, n);
    for (int m = 0; m < comps; ++m) std::memcpy(a[m], src + (size_t)m * n, (size_t)n * 4);
    return a;
  };
  std::vector<float> ev(e, e + n), Pv(P, P + n), Piv(Pi, Pi + n);
  float** flow = vec2d(u, 4);
  float** shear = vec2d(pi, 10);
  float** beta = vec2d(diag17 + (size_t)7 * n, 4);
  float** om = vec2d(diag17 + (size_t)11 * n, 6);
  std::vector<float> d0(diag17, diag17 + n), d1(diag17 + n, diag17 + 2 * (size_t)n);
  std::vector<float> pdu[4], pmm(diag17 + 6 * (size_t)n, diag17 + 7 * (size_t)n);
  for (int m = 0; m < 4; ++m) pdu[m].assign(diag17 + (2 + m) * (size_t)n, diag17 + (3 + m) * (size_t)n);
  writeScalarToFileProjection(d0.data(), (char*)"R_Pi_Inv_projection", params);
  writeScalarToFileProjection(d1.data(), (char*)"R_pimunu_Inv_projection", params);
  writeScalarToFileProjection(pdu[0].data(), (char*)"pi_dot_u_tau_projection", params);
  writeScalarToFileProjection(pdu[1].data(), (char*)"pi_dot_u_x_projection", params);
  writeScalarToFileProjection(pdu[2].data(), (char*)"pi_dot_u_y_projection", params);
  writeScalarToFileProjection(pdu[3].data(), (char*)"pi_dot_u_eta_projection", params);
  writeScalarToFileProjection(pmm.data(), (char*)"pi_mu_mu_projection", params);
  writeScalarToFile(ev.data(), (char*)"e", params);
  writeScalarToFile(Pv.data(), (char*)"p", params);
  writeScalarToFile(Piv.data(), (char*)"bulk_PI", params);
  writeScalarToFileProjection(ev.data(), (char*)"e_projection", params);
  writeScalarToFileProjection(Pv.data(), (char*)"p_projection", params);
  writeScalarToFileProjection(Piv.data(), (char*)"bulk_PI_projection", params);
  static const char* un[4] = {"ut", "ux", "uy", "un"};
  for (int m = 0; m < 4; ++m) writeVectorToFile(flow, (char*)un[m], m, params);
  for (int m = 0; m < 4; ++m)
    writeVectorToFileProjection(flow, (char*)(std::string(un[m]) + "_projection").c_str(), m, params);
  static const char* pn[10] = {"pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn", "pinn"};
  for (int m = 0; m < 10; ++m) writeVectorToFile(shear, (char*)pn[m], m, params);
  for (int m = 0; m < 10; ++m)
    writeVectorToFileProjection(shear, (char*)(std::string(pn[m]) + "_projection").c_str(), m, params);
  writeVectorToFileProjection(beta, (char*)"beta_x_projection", 1, params);
  writeVectorToFile(beta, (char*)"beta_x", 1, params);
  writeVectorToFileProjection(beta, (char*)"beta_y_projection", 2, params);
  writeVectorToFile(beta, (char*)"beta_y", 2, params);
  writeVectorToFileProjection(om, (char*)"w_xy_projection", 3, params);
  writeVectorToFile(om, (char*)"w_xy", 3, params);
  if (params.BARYON) {
    std::vector<float> nb(nB, nB + n);
    float** bd = vec2d(V, 4);
    writeScalarToFile(nb.data(), (char*)"nB", params);
    writeScalarToFileProjection(nb.data(), (char*)"nB_projection", params);
    writeVectorToFile(bd, (char*)"V_x", 1, params);
    writeVectorToFile(bd, (char*)"V_y", 2, params);
    writeVectorToFile(bd, (char*)"V_eta", 3, params);
    free2dArrayf(bd, 4);
  }
  free2dArrayf(flow, 4);
  free2dArrayf(shear, 10);
  free2dArrayf(beta, 4);
  free2dArrayf(om, 6);
  if (chdir(old) != 0) return 3;
  return 0;
}

// The reference's own initial conditions (src/InitialConditions.cpp,
// src/FileIO.cpp:133-164) inside `workdir` (whose initial_profiles/ holds the
// files the readers open).  which: 1 / 2 smooth / rand() elliptical Gaussian
// with the energy widths (15, 15, 15), 11 / 12 the same with the baryon
// widths (2, 3, 1), 3 readDensityFile of initial_profiles/e, 4 the CPU-VH
// reader, 6 the two-Gaussian profile, 21 / 22 / 23 the superMC, TRENTO and
// TRENTO 3D block readers.
extern "C" int ref_initial(const char* workdir, const oracle_params* pin, int which, float* out) {
  char old[4096];
  if (!getcwd(old, sizeof(old))) return 1;
  if (chdir(workdir) != 0) return 2;
  parameters params;
  std::memcpy(&params, pin, sizeof(params));
  params.DIM = params.DIM_X * params.DIM_Y * params.DIM_ETA;
  int rc = 0;
  switch (which) {
    case 1: initializeEllipticalGauss(out, 15.0, 15.0, 15.0, params); break;
    case 2: initializeEllipticalMCGauss(out, 15.0, 15.0, 15.0, params); break;
    case 11: initializeEllipticalGauss(out, 2.0, 3.0, 1.0, params); break;
    case 12: initializeEllipticalMCGauss(out, 2.0, 3.0, 1.0, params); break;
    case 3: readDensityFile(out, (char*)"initial_profiles/e", params); break;
    case 4: readEnergyDensityCPUVH(out, params); break;
    case 6: initialize2Gaussians(out, 1.0, 1.0, 1.0, params); break;
    case 21: readEnergyDensitySuperMCBlock(out, params); break;
    case 22: readEnergyDensityTRENTOBlock(out, params); break;
    case 23: readEnergyDensityTRENTO3DBlock(out, params); break;
    default: rc = 4;
  }
  if (chdir(old) != 0) return 3;
  return rc;
}
