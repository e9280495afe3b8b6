// fsm_hosttest.cpp -- TEST-ONLY build of the Landau-matching algorithm of
// fsm_landau.cuh for the CPU, so unit tests can exercise the solver's logic
// against the oracle without a GPU.  Not part of libfsm.so; the product runs
// the same header only inside fsm_landau_kernel.
#include "fsm_landau.cuh"

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
