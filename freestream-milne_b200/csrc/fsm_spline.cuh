// fsm_spline.cuh -- windowed natural-spline slopes of the 2D prep kernels,
// __host__ __device__ so the CPU unit tests run the same code the kernels do.
#pragma once
#include "fsm_internal.h"

#ifndef FSM_HD
#if defined(__CUDACC__)
#define FSM_HD __host__ __device__ __forceinline__
#else
#define FSM_HD inline
#endif
#endif
#if defined(__CUDA_ARCH__)
#define FSM_LDG(p) __ldg(p)
#else
#define FSM_LDG(p) (*(p))
#endif

namespace fsm {

FSM_HD int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Natural cubic spline node slopes (src/FreeStream.cpp:121-154: the bicubic
// spline's x-, y- and mixed derivatives at the nodes), by windowed elimination
// so that every thread owns kSegP nodes of a line instead of a whole line:
// the forward sweep r'_k = rhs_k - f_k r'_{k-1} and the back substitution
// M_k = (r'_k - h_{k+1} M_{k+1}) / dg_k run over the segment plus kWinP nodes
// on each side, starting from zero, with the full line's factors; where the
// window reaches the end of the line the start is exact.  Both sweeps contract
// by about 2 - sqrt(3) per node, so the truncation error is below 1e-9 of the
// local data, far below the float rounding of the packed nodes.
//
// The axis table `ax` is indexed by the unknown/interval k and is zero outside
// the line (see AxisNode), which makes the sweeps branch-free: past the line
// ends the factors vanish, so r' never leaks in (f_0 = 0) and M is zero there.
// `y(i)` must return a finite value for every node i in
// [a - kPadLo, a + kSegP + kPadHi) (zero or any finite value outside the
// line).  On return s[t] is the slope dy/dx * D at node a + t (0 for a + t
// >= n).
constexpr int kSegNF = kSegP + kWinP + 2;  // forward values kept: unknowns a-2 .. a+kSegP-1+kWinP

template <class Tab, class Y>
FSM_HD void seg_slopes(Tab ax, int n, double D, int a, Y y, float (&s)[kSegP]) {
  const int kb = a - 2 - kWinP;  // first unknown of the window
  double rps[kSegNF];
  double rp = 0.0;
  double yb = y(kb + 1);
  double sla = ax(kb).g * (yb - y(kb));
#pragma unroll
  for (int t = 0; t < kSegP + 2 * kWinP + 2; ++t) {
    const int k = kb + t;
    const double yc = y(k + 2);
    const double slb = ax(k + 1).g * (yc - yb);
    rp = (slb - sla) - ax(k).f * rp;
    if (t >= kWinP) rps[t - kWinP] = rp;
    yb = yc;
    sla = slb;
  }
  // back substitution, descending; at node j = a - 1 + t the second
  // derivatives of j and j + 1 are at hand, which is what the slope at node j
  // (or at the last node j + 1 = n - 1) needs
  double Mn = 0.0;
#pragma unroll
  for (int t = kSegNF - 1; t >= 0; --t) {
    const int k = a - 2 + t;  // node j = k + 1
    const double Mj = (rps[t] - ax(k + 1).h * Mn) * ax(k).idg;
    if (t >= 1 && t <= kSegP) {
      const int i = a + t - 1;
      if (i <= n - 2)
        s[t - 1] = (float)(((y(i + 1) - y(i)) * ax(i).g - ax(i).h * (2.0 * Mj + Mn)) * (D / 6.0));
    }
    if (t <= kSegP - 1) {
      const int i = a + t;
      if (i == n - 1)
        s[t] = (float)(((y(i) - y(i - 1)) * ax(i - 1).g + ax(i - 1).h * (Mj + 2.0 * Mn)) * (D / 6.0));
      else if (i >= n)
        s[t] = 0.0f;
    }
    Mn = Mj;
  }
}

}  // namespace fsm
