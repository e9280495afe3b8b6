// fsm_kernels.cu -- sm_100a kernels of the free-streaming + Landau-matching path.
//
//   fsm_prep2d_lines_kernel   natural-spline x- and y-derivatives of F = e/(2 pi)
//   fsm_prep2d_pack_kernel    mixed derivative + float4 node packing
//   fsm_prep3d_kernel         GeV/fm^3 -> fm^-4 conversion of 3D profiles
//   fsm_stream2d_kernel       fused free streaming + moment quadrature, 2D
//   fsm_stream3d_kernel       fused free streaming + moment quadrature, 3D (+baryon)
//   fsm_landau_kernel         FP64 Landau matching + EoS + decomposition
//
// The stream kernels never store the momentum-resolved density F(x; phi_p, y):
// each thread evaluates the shifted profile for its cell and reduces it into
// moments on the fly (the reference stores DIM*DIM_RAP*DIM_PHIP floats,
// src/FreestreamMilne.cpp:364-365, and reads them back ten times,
// src/LandauMatch.cpp:76-107).
#include <cuda_runtime.h>
#include <stdint.h>

#include "fsm_internal.h"
#include "fsm_landau.cuh"

namespace fsm {

// e [GeV/fm^3] -> fm^-4 with the reference's float operations
// (src/FreestreamMilne.cpp:266-267: e * rescale / (float)hbarc + lower_tolerance).
__device__ __forceinline__ float to_fm4(float e_gev) {
  return __fadd_rn(__fdiv_rn(__fmul_rn(e_gev, 1.0f), 0.197326938f), 1.0e-7f);
}
// 2D initial density F = e/(2 pi), double division rounded to float
// (src/FreeStream.cpp:318).
__device__ __forceinline__ float F_of(float e_gev) {
  return (float)(__ddiv_rn((double)to_fm4(e_gev), 6.283185307179586));
}

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float x) {
  float y = __fsub_rn(x, comp);
  float t = __fadd_rn(sum, y);
  comp = __fsub_rn(__fsub_rn(t, sum), y);
  sum = t;
}

// ------------------------------------------------------------------ prep 2D
// One natural-spline line solve.  `val(i)` returns the data at node i,
// `scr(i)` is a double scratch slot per node; on return scr(i) holds the
// derivative dy/dx at node i.
template <class Val, class Scr>
__device__ __forceinline__ void spline_line(const SplineAxis& ax, Val val, Scr scr) {
  const int n = ax.n;
  const int m = n - 2;
  // forward elimination, r'_k stored at node k+1
  double y0 = val(0), y1 = val(1);
  double sl_prev = (y1 - y0) / ax.h[0];
  double rp = 0.0;
  for (int k = 0; k < m; ++k) {
    double y2 = val(k + 2);
    double sl = (y2 - y1) / ax.h[k + 1];
    double rhs = 6.0 * (sl - sl_prev);
    rp = (k == 0) ? rhs : rhs - ax.f[k] * rp;
    scr(k + 1) = rp;
    sl_prev = sl;
    y1 = y2;
  }
  // back substitution: second derivatives M[1..n-2]
  double Mnext = 0.0;  // M[n-1]
  for (int k = m - 1; k >= 0; --k) {
    double Mi = (scr(k + 1) - ((k == m - 1) ? 0.0 : ax.h[k + 1] * Mnext)) / ax.dg[k];
    scr(k + 1) = Mi;
    Mnext = Mi;
  }
  // derivatives at the nodes (M[0] = M[n-1] = 0)
  double Mi = 0.0, yi = val(0);
  for (int i = 0; i < n - 1; ++i) {
    double Mi1 = (i + 1 == n - 1) ? 0.0 : scr(i + 1);
    double yi1 = val(i + 1);
    double sl = (yi1 - yi) / ax.h[i];
    scr(i) = sl - ax.h[i] * (2.0 * Mi + Mi1) / 6.0;
    if (i == n - 2) scr(n - 1) = sl + ax.h[i] * (Mi + 2.0 * Mi1) / 6.0;
    Mi = Mi1;
    yi = yi1;
  }
}

// Lines [0, NY): x-direction spline at fixed iy -> zx.  Lines [NY, NY+NX):
// y-direction spline at fixed ix -> zy.
__global__ void __launch_bounds__(128) fsm_prep2d_lines_kernel(const Ev2D* __restrict__ evs,
                                                               const LineBlock* __restrict__ blocks) {
  const LineBlock b = blocks[blockIdx.x];
  const Ev2D& ev = evs[b.ev];
  const int line = b.begin + threadIdx.x;
  const int NX = ev.NX, NY = ev.NY;
  if (line >= NX + NY) return;
  const float* e = ev.e_gev;
  if (line < NY) {
    const int iy = line;
    double* zx = ev.zx;
    spline_line(ev.ax, [&](int i) { return (double)F_of(__ldg(e + (size_t)i * NY + iy)); },
                [&](int i) -> double& { return zx[(size_t)i * NY + iy]; });
  } else {
    const int ix = line - NY;
    double* zy = ev.zy + (size_t)ix * NY;
    const float* er = e + (size_t)ix * NY;
    spline_line(ev.ay, [&](int j) { return (double)F_of(__ldg(er + j)); },
                [&](int j) -> double& { return zy[j]; });
  }
}

// Mixed derivative zxy = d/dx of the zy field along x lines (fixed iy), then
// pack the node float4 (F, zx*DX, zy*DY, zxy*DX*DY).  zx is overwritten with
// the line scratch after it has been consumed.
__global__ void __launch_bounds__(128) fsm_prep2d_pack_kernel(const Ev2D* __restrict__ evs,
                                                              const LineBlock* __restrict__ blocks) {
  const LineBlock b = blocks[blockIdx.x];
  const Ev2D& ev = evs[b.ev];
  const int iy = b.begin + threadIdx.x;
  const int NX = ev.NX, NY = ev.NY;
  if (iy >= NY) return;
  const double DX = ev.DX, DY = ev.DY;
  const double* zy = ev.zy;
  double* zx = ev.zx;
  FSM_FLOAT4* nodes = ev.nodes;
  const float* e = ev.e_gev;
  // first consume zx into the nodes (x, y components), freeing zx as scratch
  for (int ix = 0; ix < NX; ++ix) {
    size_t k = (size_t)ix * NY + iy;
    float4 nd;
    nd.x = F_of(__ldg(e + k));
    nd.y = (float)(zx[k] * DX);
    nd.z = (float)(zy[k] * DY);
    nd.w = 0.0f;
    nodes[k] = nd;
  }
  spline_line(ev.ax, [&](int i) { return zy[(size_t)i * NY + iy]; },
              [&](int i) -> double& { return zx[(size_t)i * NY + iy]; });
  for (int ix = 0; ix < NX; ++ix) {
    size_t k = (size_t)ix * NY + iy;
    nodes[k].w = (float)(zx[k] * DX * DY);
  }
}

// ------------------------------------------------------------------ prep 3D
__global__ void __launch_bounds__(256) fsm_prep3d_kernel(const Ev3D* __restrict__ evs,
                                                         const CellBlock* __restrict__ blocks) {
  const CellBlock b = blocks[blockIdx.x];
  const Ev3D& ev = evs[b.ev];
  const int DIM = ev.NX * ev.NY * ev.NE;
  const int is = b.begin + threadIdx.x;
  if (is < DIM) ev.efield[is] = to_fm4(__ldg(ev.e_gev + is));
}

// ---------------------------------------------------------------- stream 2D
// Hermite basis on [0,1]: value weights H0,H1 and slope weights G0,G1.
__device__ __forceinline__ void hermite(float t, float& H0, float& H1, float& G0, float& G1) {
  const float t2 = t * t;
  H1 = t2 * (3.0f - 2.0f * t);
  H0 = 1.0f - H1;
  const float omt = 1.0f - t;
  G0 = t * omt * omt;
  G1 = t2 * (t - 1.0f);
}

template <bool kSmem>
__device__ __forceinline__ void stream2d_tile(const Ev2D& ev, int x0, int y0, float4* __restrict__ sn,
                                              const float2* __restrict__ scs, int* err) {
  const int NX = ev.NX, NY = ev.NY, NPHI = ev.NPHI;
  const int fx0 = max(0, x0 - ev.Rx), fx1 = min(NX - 1, x0 + kTileX + ev.Rx);
  const int fy0 = max(0, y0 - ev.Ry), fy1 = min(NY - 1, y0 + kTileY + ev.Ry);
  const int FW = fy1 - fy0 + 1, FH = fx1 - fx0 + 1;
  const float4* __restrict__ gnodes = reinterpret_cast<const float4*>(ev.nodes);
  if (kSmem) {
    for (int k = threadIdx.x; k < FW * FH; k += blockDim.x) {
      int r = k / FW, c = k - r * FW;
      sn[k] = __ldg(gnodes + (size_t)(fx0 + r) * NY + (fy0 + c));
    }
  }
  __syncthreads();

  const int lx = threadIdx.x / kTileY, ly = threadIdx.x - lx * kTileY;
  const int ix = x0 + lx, iy = y0 + ly;
  const bool active = (ix < NX) && (iy < NY);
  const float DX = ev.DX, DY = ev.DY, DTAU = ev.DTAU;
  const float xmin = ev.xmin, ymin = ev.ymin, inv_dx = ev.inv_dx, inv_dy = ev.inv_dy;
  const float xmax_i = ev.xmax_i, ymax_i = ev.ymax_i;
  const float NXm1 = (float)(NX - 1), NYm1 = (float)(NY - 1);
  // cell coordinates (src/FreeStream.cpp:163-164)
  const float x = __fadd_rn(__fmul_rn((float)ix, DX), xmin);
  const float y = __fadd_rn(__fmul_rn((float)iy, DY), ymin);

  float acc[6] = {0, 0, 0, 0, 0, 0}, tot[6] = {0, 0, 0, 0, 0, 0}, cmp[6] = {0, 0, 0, 0, 0, 0};
  int nerr = 0;
  for (int p = 0; p < NPHI; ++p) {
    const float2 cs = scs[p];
    // shifted position (src/FreeStream.cpp:187-199), same float rounding
    const float xn = __fsub_rn(x, __fmul_rn(cs.x, DTAU));
    const float yn = __fsub_rn(y, __fmul_rn(cs.y, DTAU));
    float qx = __fmul_rn(__fsub_rn(xn, xmin), inv_dx);
    float qy = __fmul_rn(__fsub_rn(yn, ymin), inv_dy);
    // Where the in-grid test (src/FreeStream.cpp:213) could flip, use the
    // reference's correctly rounded division.
    if (fabsf(qx - 1.0f) < 1.0e-3f || fabsf(qx - NXm1) < 1.0e-3f)
      qx = __fdiv_rn(__fsub_rn(xn, xmin), DX);
    if (fabsf(qy - 1.0f) < 1.0e-3f || fabsf(qy - NYm1) < 1.0e-3f)
      qy = __fdiv_rn(__fsub_rn(yn, ymin), DY);
    const float fxf = floorf(qx), fyf = floorf(qy);
    if (active && fxf >= 1.0f && fxf < NXm1 && fyf >= 1.0f && fyf < NYm1) {
      const int i = (int)fxf, j = (int)fyf;
      const float t = qx - fxf, u = qy - fyf;
      float4 n00, n10, n01, n11;
      if (kSmem) {
        const int si = i - fx0, sj = j - fy0;
        if ((unsigned)si > (unsigned)(FH - 2) || (unsigned)sj > (unsigned)(FW - 2)) {
          ++nerr;  // outside the staged footprint: cannot happen for a correct halo
          continue;
        }
        const int k = si * FW + sj;
        n00 = sn[k];
        n01 = sn[k + 1];
        n10 = sn[k + FW];
        n11 = sn[k + FW + 1];
      } else {
        const size_t k = (size_t)i * NY + j;
        n00 = __ldg(gnodes + k);
        n01 = __ldg(gnodes + k + 1);
        n10 = __ldg(gnodes + k + NY);
        n11 = __ldg(gnodes + k + NY + 1);
      }
      // bilinear (src/FreeStream.cpp:84-94)
      float v = ((1.0f - t) * (1.0f - u) * n00.x) + (t * (1.0f - u) * n10.x) +
                ((1.0f - t) * u * n01.x) + (t * u * n11.x);
      // bicubic spline inside its open domain, used when positive
      // (src/FreeStream.cpp:237-246)
      if ((xmin < xn) && (xn < xmax_i) && (ymin < yn) && (yn < ymax_i)) {
        float H0, H1, G0, G1, K0, K1, L0, L1;
        hermite(t, H0, H1, G0, G1);
        hermite(u, K0, K1, L0, L1);
        const float r0 = H0 * n00.x + H1 * n10.x + G0 * n00.y + G1 * n10.y;
        const float r1 = H0 * n01.x + H1 * n11.x + G0 * n01.y + G1 * n11.y;
        const float s0 = H0 * n00.z + H1 * n10.z + G0 * n00.w + G1 * n10.w;
        const float s1 = H0 * n01.z + H1 * n11.z + G0 * n01.w + G1 * n11.w;
        const float c = K0 * r0 + K1 * r1 + L0 * s0 + L1 * s1;
        if (c > 0.0f) v = c;
      }
      // moments with the 2D hypertrig rows 1, cos, sin, cos^2, cos sin, sin^2
      // (src/LandauMatch.cpp:46-55 at rap = eta = 0)
      acc[0] += v;
      acc[1] += v * cs.x;
      acc[2] += v * cs.y;
      acc[3] += v * (cs.x * cs.x);
      acc[4] += v * (cs.x * cs.y);
      acc[5] += v * (cs.y * cs.y);
    }
    if ((p & (kPhiChunk - 1)) == kPhiChunk - 1) {
#pragma unroll
      for (int m = 0; m < 6; ++m) {
        kahan_add(tot[m], cmp[m], acc[m]);
        acc[m] = 0.0f;
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 6; ++m) kahan_add(tot[m], cmp[m], acc[m]);
  if (nerr) atomicAdd(err, nerr);

  if (active) {
    // T = (sum over DIM_RAP identical rapidity copies) * d_phip / TAU
    // (src/LandauMatch.cpp:104)
    const float R = (float)ev.NR, dphi = ev.d_phip, TAU = ev.TAU;
    float Tv[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) Tv[m] = __fdiv_rn(__fmul_rn(__fmul_rn(tot[m], R), dphi), TAU);
    const size_t DIM = (size_t)NX * NY, is = (size_t)ix * NY + iy;
    float* T = ev.T;
    T[0 * DIM + is] = Tv[0];
    T[1 * DIM + is] = Tv[1];
    T[2 * DIM + is] = Tv[2];
    T[3 * DIM + is] = 0.0f;
    T[4 * DIM + is] = Tv[3];
    T[5 * DIM + is] = Tv[4];
    T[6 * DIM + is] = 0.0f;
    T[7 * DIM + is] = Tv[5];
    T[8 * DIM + is] = 0.0f;
    T[9 * DIM + is] = 0.0f;
  }
}

// Persistent kernel: each CTA takes output tiles from a global work list
// (largest first) until it is exhausted.  The work counter is a plain
// atomicAdd on a reset counter, so no CTA ever waits on another.
__global__ void __launch_bounds__(kThreads2D) fsm_stream2d_kernel(const Ev2D* __restrict__ evs,
                                                                  const Tile2D* __restrict__ tiles,
                                                                  int ntiles, int cs_cap,
                                                                  Counters* ctr, int* err) {
  extern __shared__ float4 smem4[];
  __shared__ int s_tile;
  float2* scs = reinterpret_cast<float2*>(smem4);
  float4* sn = smem4 + (cs_cap + 1) / 2;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctr->tile2d, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= ntiles) return;
    const Tile2D tl = tiles[t];
    const Ev2D& ev = evs[tl.ev];
    for (int k = threadIdx.x; k < ev.NPHI; k += blockDim.x) {
      const FSM_FLOAT2 c = ev.cs[k];
      scs[k] = make_float2(c.x, c.y);
    }
    if (ev.use_smem) stream2d_tile<true>(ev, tl.x0, tl.y0, sn, scs, err);
    else stream2d_tile<false>(ev, tl.x0, tl.y0, sn, scs, err);
    __syncthreads();
  }
}

// ---------------------------------------------------------------- stream 3D
// One thread per cell; cells of a CTA are consecutive in the reference order
// (eta fastest), so the trilinear corner loads of a warp are coalesced.
__global__ void __launch_bounds__(kThreads3D) fsm_stream3d_kernel(const Ev3D* __restrict__ evs,
                                                                  const CellBlock* __restrict__ blocks,
                                                                  int nblocks, int cs_cap,
                                                                  Counters* ctr) {
  extern __shared__ float4 smem4[];
  __shared__ int s_blk;
  float2* scs = reinterpret_cast<float2*>(smem4);
  for (;;) {
    if (threadIdx.x == 0) s_blk = atomicAdd(&ctr->block3d, 1);
    __syncthreads();
    const int bi = s_blk;
    if (bi >= nblocks) return;
    const CellBlock b = blocks[bi];
    const Ev3D& ev = evs[b.ev];
    const int NPHI = ev.NPHI;
    for (int k = threadIdx.x; k < NPHI; k += blockDim.x) {
      const FSM_FLOAT2 c = ev.cs[k];
      scs[k] = make_float2(c.x, c.y);
    }
    __syncthreads();
    const int NX = ev.NX, NY = ev.NY, NE = ev.NE, NR = ev.NR;
    const int DIM = NX * NY * NE;
    const int is = b.begin + threadIdx.x;
    if (is < DIM) {
      const int ix = is / (NY * NE);
      const int iy = (is - NY * NE * ix) / NE;
      const int ieta = is - NY * NE * ix - NE * iy;
      const float DX = ev.DX, DY = ev.DY, xmin = ev.xmin, ymin = ev.ymin;
      const float inv_dx = ev.inv_dx, inv_dy = ev.inv_dy;
      const float NXm1 = (float)(NX - 1), NYm1 = (float)(NY - 1);
      const float x = __fadd_rn(__fmul_rn((float)ix, DX), xmin);
      const float y = __fadd_rn(__fmul_rn((float)iy, DY), ymin);
      const float* __restrict__ ef = ev.efield;
      const float* __restrict__ nb = ev.nB;
      const bool baryon = ev.baryon != 0;
      const int sx = NY * NE;
      float Tt[10], Tc[10], Jt[4], Jc[4];
#pragma unroll
      for (int m = 0; m < 10; ++m) Tt[m] = Tc[m] = 0.0f;
#pragma unroll
      for (int m = 0; m < 4; ++m) Jt[m] = Jc[m] = 0.0f;
      for (int irap = ev.r_lo; irap < ev.r_hi; ++irap) {
        const RapEta re = ev.re[ieta * NR + irap];
        if (!(re.efl >= 1 && re.efl < NE - 1) || !isfinite(re.D)) continue;
        const float D = re.D, et = re.efrac;
        const float rf0 = __ldg(ev.rapf + re.efl * NR + irap), rf1 = __ldg(ev.rapf + (re.efl + 1) * NR + irap);
        float rb0 = 0.f, rb1 = 0.f;
        if (baryon) {
          rb0 = __ldg(ev.rapfB + re.efl * NR + irap);
          rb1 = __ldg(ev.rapfB + (re.efl + 1) * NR + irap);
        }
        float a[6] = {0, 0, 0, 0, 0, 0}, st[6] = {0, 0, 0, 0, 0, 0}, sc[6] = {0, 0, 0, 0, 0, 0};
        float ab[3] = {0, 0, 0}, sbt[3] = {0, 0, 0}, sbc[3] = {0, 0, 0};
        for (int p = 0; p < NPHI; ++p) {
          const float2 cs = scs[p];
          // (src/FreeStream.cpp:193-199)
          const float xn = __fsub_rn(x, __fmul_rn(cs.x, D));
          const float yn = __fsub_rn(y, __fmul_rn(cs.y, D));
          float qx = __fmul_rn(__fsub_rn(xn, xmin), inv_dx);
          float qy = __fmul_rn(__fsub_rn(yn, ymin), inv_dy);
          if (fabsf(qx - 1.0f) < 1.0e-3f || fabsf(qx - NXm1) < 1.0e-3f)
            qx = __fdiv_rn(__fsub_rn(xn, xmin), DX);
          if (fabsf(qy - 1.0f) < 1.0e-3f || fabsf(qy - NYm1) < 1.0e-3f)
            qy = __fdiv_rn(__fsub_rn(yn, ymin), DY);
          const float fxf = floorf(qx), fyf = floorf(qy);
          if (fxf >= 1.0f && fxf < NXm1 && fyf >= 1.0f && fyf < NYm1) {
            const int i = (int)fxf, j = (int)fyf;
            const float t = qx - fxf, u = qy - fyf;
            const int k = i * sx + j * NE + re.efl;
            const float w00 = (1.0f - t) * (1.0f - u), w10 = t * (1.0f - u), w01 = (1.0f - t) * u,
                        w11 = t * u;
            const float l0 = w00 * __ldg(ef + k) + w10 * __ldg(ef + k + sx) + w01 * __ldg(ef + k + NE) +
                             w11 * __ldg(ef + k + sx + NE);
            const float l1 = w00 * __ldg(ef + k + 1) + w10 * __ldg(ef + k + sx + 1) +
                             w01 * __ldg(ef + k + NE + 1) + w11 * __ldg(ef + k + sx + NE + 1);
            const float v = (1.0f - et) * (l0 * rf0) + et * (l1 * rf1);
            a[0] += v;
            a[1] += v * cs.x;
            a[2] += v * cs.y;
            a[3] += v * (cs.x * cs.x);
            a[4] += v * (cs.x * cs.y);
            a[5] += v * (cs.y * cs.y);
            if (baryon) {
              const float b0 = w00 * __ldg(nb + k) + w10 * __ldg(nb + k + sx) +
                               w01 * __ldg(nb + k + NE) + w11 * __ldg(nb + k + sx + NE);
              const float b1 = w00 * __ldg(nb + k + 1) + w10 * __ldg(nb + k + sx + 1) +
                               w01 * __ldg(nb + k + NE + 1) + w11 * __ldg(nb + k + sx + NE + 1);
              const float vb = (1.0f - et) * (b0 * rb0) + et * (b1 * rb1);
              ab[0] += vb;
              ab[1] += vb * cs.x;
              ab[2] += vb * cs.y;
            }
          }
          if ((p & (kPhiChunk - 1)) == kPhiChunk - 1) {
#pragma unroll
            for (int m = 0; m < 6; ++m) {
              kahan_add(st[m], sc[m], a[m]);
              a[m] = 0.0f;
            }
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              kahan_add(sbt[m], sbc[m], ab[m]);
              ab[m] = 0.0f;
            }
          }
        }
#pragma unroll
        for (int m = 0; m < 6; ++m) kahan_add(st[m], sc[m], a[m]);
#pragma unroll
        for (int m = 0; m < 3; ++m) kahan_add(sbt[m], sbc[m], ab[m]);
        // rows of the hypertrig table (src/LandauMatch.cpp:46-55) times the
        // rapidity Jacobian (src/LandauMatch.cpp:101) and the profile norm
        const float jw = ev.jac[irap] * ev.norm;
        const float S1 = st[0] * jw, Sc = st[1] * jw, Ss = st[2] * jw;
        kahan_add(Tt[0], Tc[0], S1);
        kahan_add(Tt[1], Tc[1], Sc * re.A);
        kahan_add(Tt[2], Tc[2], Ss * re.A);
        kahan_add(Tt[3], Tc[3], S1 * re.Dt);
        kahan_add(Tt[4], Tc[4], st[3] * jw * re.B);
        kahan_add(Tt[5], Tc[5], st[4] * jw * re.B);
        kahan_add(Tt[6], Tc[6], Sc * re.C);
        kahan_add(Tt[7], Tc[7], st[5] * jw * re.B);
        kahan_add(Tt[8], Tc[8], Ss * re.C);
        kahan_add(Tt[9], Tc[9], S1 * re.E);
        if (baryon) {
          const float B1 = sbt[0] * ev.normB, Bc = sbt[1] * ev.normB, Bs = sbt[2] * ev.normB;
          kahan_add(Jt[0], Jc[0], B1);
          kahan_add(Jt[1], Jc[1], Bc * re.A);
          kahan_add(Jt[2], Jc[2], Bs * re.A);
          kahan_add(Jt[3], Jc[3], B1 * re.Dt);
        }
      }
      const float dphi = ev.d_phip;
#pragma unroll
      for (int m = 0; m < 10; ++m) ev.T[(size_t)m * DIM + is] = Tt[m] * dphi;  // (LandauMatch.cpp:105)
      if (baryon) {
        const float jf = ev.DRAP * dphi;  // (LandauMatch.cpp:140)
#pragma unroll
        for (int m = 0; m < 4; ++m) ev.J[(size_t)m * DIM + is] = Jt[m] * jf;
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- Landau
__global__ void __launch_bounds__(kThreadsLandau) fsm_landau_kernel(const EvLandau* __restrict__ evs,
                                                                    const CellBlock* __restrict__ blocks,
                                                                    Counters* ctr) {
  const CellBlock b = blocks[blockIdx.x];
  const EvLandau& ev = evs[b.ev];
  const int DIM = ev.DIM;
  const int is = b.begin + threadIdx.x;
  int fb = 0;
  if (is < DIM) {
    float T[10], J[4] = {0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < 10; ++m) T[m] = __ldg(ev.T + (size_t)m * DIM + is);
    if (ev.baryon && ev.J) {
#pragma unroll
      for (int m = 0; m < 4; ++m) J[m] = __ldg(ev.J + (size_t)m * DIM + is);
    }
    CellOut o;
    landau_cell(T, J, ev.is3d, ev.baryon, ev.eos, ev.viscous, ev.TAU, &o);
    fb = o.fallback;
    if (ev.e) ev.e[is] = o.e;
    if (ev.P) ev.P[is] = o.P;
    if (ev.Pi) ev.Pi[is] = o.Pi;
    if (ev.u) {
#pragma unroll
      for (int m = 0; m < 4; ++m) ev.u[(size_t)m * DIM + is] = o.u[m];
    }
    if (ev.pi) {
#pragma unroll
      for (int m = 0; m < 10; ++m) ev.pi[(size_t)m * DIM + is] = o.pi[m];
    }
    if (ev.baryon) {
      if (ev.nB) ev.nB[is] = o.nB;
      if (ev.V) {
#pragma unroll
        for (int m = 0; m < 4; ++m) ev.V[(size_t)m * DIM + is] = o.V[m];
      }
    }
  }
  const unsigned mask = __ballot_sync(0xffffffffu, fb);
  if ((threadIdx.x & 31) == 0 && mask) atomicAdd(&ctr->fallback, __popc(mask));
}

}  // namespace fsm
