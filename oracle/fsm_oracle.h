/* fsm_oracle.h -- TEST INFRASTRUCTURE: C interface of the CPU oracle.
 *
 * The oracle is a CPU restatement of the freestream-milne reference hot path
 * (src/FreestreamMilne.cpp:251-506) used only by tests, by the smoke check and
 * by the CPU-baseline leg of bench.py.  It is never part of the product.
 *
 * Two precisions:
 *   fp64 = 0  mirrors the reference's float/double mixing operation by
 *             operation (float arrays, float transcendentals where the
 *             reference calls them on floats, double GSL stand-ins);
 *   fp64 = 1  runs the same algorithm entirely in double;
 *   fp64 = 2  keeps the reference's float geometry (sample angles, shifted
 *             positions, index floors: the same set of in-grid samples) and
 *             computes every value in double -- the precision oracle.
 */
#ifndef FSM_ORACLE_H_
#define FSM_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order and meaning as `struct parameters` (src/Parameter.h:2-33). */
typedef struct oracle_params {
  int OUTPUTFORMAT;
  int BARYON;
  int IC_ENERGY;
  int IC_BARYON;
  float ETA_WIDTH;
  float ETA_FLAT;
  float SIGMA;
  float SIGMA_B;
  int DIM_X;
  int DIM_Y;
  int DIM_ETA;
  int DIM_RAP;
  int DIM_PHIP;
  float DX;
  float DY;
  float DETA;
  float DRAP;
  float DTAU;
  float TAU0;
  int EOS_TYPE;
  float E_FREEZE;
  int VISCOUS_MATCHING;
  int E_DEP_FS;
  float E_R;
  float TAU_R;
  float ALPHA;
  int DIM;
  float TAU;
} oracle_params;

/* Caller-owned output arrays, component-major ([comp][cell]) in the reference
 * cell order is = (DIM_Y*DIM_ETA)*ix + DIM_ETA*iy + ieta.  Any pointer may be
 * NULL to skip that output.  Units are the reference's internal ones (fm^-4,
 * fm^-3 for baryon quantities), i.e. before the hbar*c conversion of
 * src/FreestreamMilne.cpp:700-716. */
typedef struct oracle_out {
  double* T;   /* 10*DIM: tt tx ty tn xx xy xn yy yn nn (LandauMatch.cpp:46-55 order) */
  double* J;   /* 4*DIM, BARYON only */
  double* e;   /* DIM */
  double* P;   /* DIM */
  double* Pi;  /* DIM */
  double* u;   /* 4*DIM */
  double* pi;  /* 10*DIM */
  double* nB;  /* DIM, BARYON only */
  double* V;   /* 4*DIM, BARYON only */
  /* effective values after E_DEP_FS and the phi_p rule (FreestreamMilne.cpp:316-332) */
  int dim_phip;
  float dtau;
  float tau;
  int n_fallback; /* cells where no acceptable eigenvector was found */
} oracle_out;

/* e_gev: initial energy density in GeV/fm^3 (the initialize_from_vector input);
 * nB: initial baryon density exactly as the IC_BARYON=3 file reader stores it
 * (no unit conversion), may be NULL when BARYON == 0.
 * Returns 0 on success, nonzero on invalid parameters. */
int oracle_run(const oracle_params* p, int fp64, const float* e_gev, const float* nB,
               oracle_out* out, int nthreads);

/* Natural cubic spline node derivatives (unit tests against scipy). */
void oracle_spline_derivs(const double* x, const double* y, int n, double* d);

/* 2D bicubic spline evaluated at npts points; z[i + j*nx] = f(x[i], y[j]). */
void oracle_bicubic_eval(const double* x, const double* y, const double* z, int nx, int ny,
                         const double* px, const double* py, int npts, double* out);

/* General real eigen-decomposition (n <= 4), see fsm_numerics.h. */
int oracle_eig(int n, const double* A, double* wr, double* wi, double* vr);

/* Landau matching of one cell (LandauMatch.cpp:145-291) given its ten float
 * T^{mu nu} components; returns 1 if an eigenvector was accepted. */
int oracle_landau_cell(const float* T10, float tau, float* e, float* u4);

/* Hydro-validity and thermal-vorticity diagnostics of the Landau-matched
 * fields (src/HydroValidity.cpp:8-101, src/LandauMatch.cpp:395-489) at
 * proper time tau: out has 17 components of DIM floats: R_Pi_Inv,
 * R_pimunu_Inv, pi.u (4), pi^mu_mu, beta (4), omega (6). */
void oracle_diagnostics(const oracle_params* p, float tau, const float* e, const float* P,
                        const float* Pi, const float* u, const float* pi, float* out17);

#ifdef __cplusplus
}
#endif
#endif
