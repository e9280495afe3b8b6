// fsm_kernels.cu -- sm_100a kernels of the free-streaming + Landau-matching path.
//
//   fsm_prep2d_rows_kernel    F = e/(2 pi) and its natural-spline y-derivatives
//   fsm_prep2d_cols_kernel    x- and mixed derivatives + float4 node packing
//   fsm_prep2d_*_long_kernel  the same for grids whose lines exceed kMaxStrip
//   fsm_prep3d_kernel         GeV/fm^3 -> fm^-4 conversion into eta-pair node arrays (3D)
//   fsm_stream2d_kernel       fused free streaming + moment quadrature, 2D
//   fsm_stream3d_kernel       fused free streaming + moment quadrature, 3D
//   fsm_stream3d_baryon_kernel  the same with baryon charge
//   fsm_pack_kernel           gather of output fields for one-copy downloads
//   fsm_landau_kernel         FP64 Landau matching + EoS + decomposition, 2D
//   fsm_landau3d_kernel       the same for 3D events
//
// The stream kernels never store the momentum-resolved density F(x; phi_p, y):
// each thread evaluates the shifted profile for its cell and reduces it into
// moments on the fly (the reference stores DIM*DIM_RAP*DIM_PHIP floats,
// src/FreestreamMilne.cpp:364-365, and reads them back ten times,
// src/LandauMatch.cpp:76-107).
#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>
#include <cuda.h>

#include "fsm_internal.h"
#include "fsm_landau.cuh"
#include "fsm_spline.cuh"

namespace fsm {

// e [GeV/fm^3] -> fm^-4 with the reference's float operations
// (src/FreestreamMilne.cpp:266-267: e * rescale / (float)hbarc + lower_tolerance).
__device__ __forceinline__ float to_fm4(float e_gev) {
  return __fadd_rn(__fdiv_rn(__fmul_rn(e_gev, 1.0f), 0.197326938f), 1.0e-7f);
}
// 2D initial density F = e/(2 pi), double division rounded to float
// (src/FreeStream.cpp:318), from GeV/fm^3 or (raw) from fm^-4.
__device__ __forceinline__ float F_of(float e, int raw) {
  return (float)(__ddiv_rn((double)(raw ? e : to_fm4(e)), 6.283185307179586));
}


// ------------------------------------------------------------------ prep 2D
// Strip kernels: a block owns 32 lines of one event and stages them whole in
// shared memory (coalesced), zero-padded at both ends, together with the
// padded axis table; lane l takes line l and warp w the segments w, w + 8, ...
// of it, so the table reads are warp-uniform broadcasts and the line reads
// conflict-free.  Line lengths up to kMaxStrip.
__device__ __forceinline__ void stage_axis(AxisNode* dst, const AxisNode* __restrict__ src, int n) {
  const double* s = reinterpret_cast<const double*>(src - kPadLo);
  double* d = reinterpret_cast<double*>(dst);
  const int total = (n + kPadLo + kPadHi) * 4;
  constexpr int kB = 4;  // independent loads in flight per thread
  for (int i0 = threadIdx.x; i0 < total; i0 += blockDim.x * kB) {
    double v[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      v[u] = i < total ? __ldg(s + i) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < total) d[i] = v[u];
    }
  }
}

// y-lines (rows ix0 .. ix0+31, contiguous in memory): F = e/(2 pi) -> fa and
// its y-slopes -> sy.  Lines are staged with an odd stride.
__global__ void __launch_bounds__(kPrepThreads, 2) fsm_prep2d_rows_kernel(
    const Ev2D* __restrict__ evs, const LineBlock* __restrict__ blocks) {
  extern __shared__ __align__(16) unsigned char prep_smem[];
  const LineBlock b = blocks[blockIdx.x];
  const Ev2D& ev = evs[b.ev];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int NX = ev.NX, NY = ev.NY;
  const int ix0 = b.begin;
  const int nr = min(32, NX - ix0);
  const int ld = (NY + kPadLo + kPadHi) | 1;
  AxisNode* tab = reinterpret_cast<AxisNode*>(prep_smem);
  float* Fs = reinterpret_cast<float*>(tab + NY + kPadLo + kPadHi);
  float* Ss = Fs + 32 * ld;
  stage_axis(tab, ev.ay, NY);
  for (int r = warp; r < 32; r += kPrepThreads / 32) {
    float* fl = Fs + r * ld;
    for (int c = lane; c < ld; c += 32) fl[c] = 0.0f;  // padding (and rows past the grid)
  }
  __syncthreads();
  {
    // 8 independent loads in flight per thread before their stores (the
    // descriptor's pointers may alias as far as the compiler knows, so it
    // would not hoist a load above the preceding store by itself)
    const float* __restrict__ src = ev.e_gev;
    float* __restrict__ fa = ev.fa;
    constexpr int kB = 8;
    for (int r = warp; r < nr; r += kPrepThreads / 32) {
      const size_t row = (size_t)(ix0 + r) * NY;
      float* fl = Fs + r * ld + kPadLo;
      for (int c0 = lane; c0 < NY; c0 += 32 * kB) {
        float in[kB];
#pragma unroll
        for (int u = 0; u < kB; ++u) {
          const int c = c0 + 32 * u;
          in[u] = c < NY ? __ldg(src + row + c) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kB; ++u) {
          const int c = c0 + 32 * u;
          if (c < NY) {
            const float f = ev.charge ? __fmul_rn(in[u], ev.qnorm) : F_of(in[u], ev.raw);
            fl[c] = f;
            fa[row + c] = f;
          }
        }
      }
    }
  }
  __syncthreads();
  {
    const float* fl = Fs + lane * ld + kPadLo;
    float* sl = Ss + lane * ld;
    const AxisNode* A = tab + kPadLo;
    const int nseg = (NY + kSegP - 1) / kSegP;
    for (int sg = warp; sg < nseg; sg += kPrepThreads / 32) {
      float sv[kSegP];
      seg_slopes([&](int k) -> const AxisNode& { return A[k]; }, NY, (double)ev.DY, sg * kSegP,
                 [&](int j) { return (double)fl[j]; }, sv);
#pragma unroll
      for (int t = 0; t < kSegP; ++t)
        if (sg * kSegP + t < NY) sl[sg * kSegP + t] = sv[t];
    }
  }
  __syncthreads();
  for (int r = warp; r < nr; r += kPrepThreads / 32) {
    const size_t row = (size_t)(ix0 + r) * NY;
    for (int c = lane; c < NY; c += 32) ev.sy[row + c] = Ss[r * ld + c];
  }
}

// x-lines (columns iy0 .. iy0+31 at stride NY): x-slopes of F and of the
// y-slope field (the mixed derivative), packed with F and F_y into the nodes.
// A job is one field of one segment: (F, F_x) fills the first half of the
// node float4, (F_y, F_xy) the second.
__global__ void __launch_bounds__(kPrepThreads, 2) fsm_prep2d_cols_kernel(
    const Ev2D* __restrict__ evs, const LineBlock* __restrict__ blocks) {
  extern __shared__ __align__(16) unsigned char prep_smem[];
  const LineBlock b = blocks[blockIdx.x];
  const Ev2D& ev = evs[b.ev];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int NX = ev.NX, NY = ev.NY;
  const int iy0 = b.begin;
  const int nc = min(32, NY - iy0);
  const int np = NX + kPadLo + kPadHi;
  AxisNode* tab = reinterpret_cast<AxisNode*>(prep_smem);
  float* Fs = reinterpret_cast<float*>(tab + np);
  float* Ys = Fs + 32 * np;
  stage_axis(tab, ev.ax, NX);
  {
    constexpr int kB = 8;  // independent loads in flight per thread
    const float* __restrict__ fa = ev.fa;
    const float* __restrict__ sy = ev.sy;
    for (int i0 = warp; i0 < np; i0 += (kPrepThreads / 32) * kB) {
      float f[kB], yv[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int i = i0 + (kPrepThreads / 32) * u, ix = i - kPadLo;
        f[u] = yv[u] = 0.0f;
        if (i < np && ix >= 0 && ix < NX && lane < nc) {
          const size_t k = (size_t)ix * NY + iy0 + lane;
          f[u] = __ldg(fa + k);
          yv[u] = __ldg(sy + k);
        }
      }
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int i = i0 + (kPrepThreads / 32) * u;
        if (i < np) {
          Fs[i * 32 + lane] = f[u];
          Ys[i * 32 + lane] = yv[u];
        }
      }
    }
  }
  __syncthreads();
  if (lane >= nc) return;
  const float* fc = Fs + kPadLo * 32 + lane;
  const float* yc = Ys + kPadLo * 32 + lane;
  const AxisNode* A = tab + kPadLo;
  float2* nodes = reinterpret_cast<float2*>(reinterpret_cast<float4*>(ev.nodes) + iy0 + lane);
  const int nseg = (NX + kSegP - 1) / kSegP;
  for (int job = warp; job < 2 * nseg; job += kPrepThreads / 32) {
    const int a = (job >> 1) * kSegP, half = job & 1;
    const float* vc = half ? yc : fc;
    float sv[kSegP];
    seg_slopes([&](int k) -> const AxisNode& { return A[k]; }, NX, (double)ev.DX, a,
               [&](int i) { return (double)vc[i * 32]; }, sv);
#pragma unroll
    for (int t = 0; t < kSegP; ++t) {
      const int i = a + t;
      if (i < NX) nodes[(size_t)i * NY * 2 + half] = make_float2(vc[i * 32], sv[t]);
    }
  }
}

// Long lines.  y-lines: one warp per x row ix.  The row's F = e/(2 pi) is
// staged in shared memory (coalesced, zero-padded), lane l takes segments l,
// l+32, ..., and the slopes are stored back coalesced.
__global__ void __launch_bounds__(kPrepRows * 32) fsm_prep2d_rows_long_kernel(
    const Ev2D* __restrict__ evs, const LineBlock* __restrict__ blocks, int ny_cap) {
  extern __shared__ __align__(16) unsigned char prep_smem[];
  const LineBlock b = blocks[blockIdx.x];
  const Ev2D& ev = evs[b.ev];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int NX = ev.NX, NY = ev.NY;
  const int ix = b.begin + warp;
  if (ix >= NX) return;
  const int stride = ny_cap + kPadLo + kPadHi + 2;
  float* fr = reinterpret_cast<float*>(prep_smem) + (size_t)warp * 2 * stride;
  float* sr = fr + stride;
  const size_t row = (size_t)ix * NY;
  for (int c = lane; c < NY + kPadLo + kPadHi; c += 32) fr[c] = 0.0f;
  __syncwarp();
  {
    const float* __restrict__ src = ev.e_gev;
    float* __restrict__ fa = ev.fa;
    constexpr int kB = 8;  // independent loads in flight per thread
    for (int c0 = lane; c0 < NY; c0 += 32 * kB) {
      float in[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int c = c0 + 32 * u;
        in[u] = c < NY ? __ldg(src + row + c) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int c = c0 + 32 * u;
        if (c < NY) {
          const float f = ev.charge ? __fmul_rn(in[u], ev.qnorm) : F_of(in[u], ev.raw);
          fr[kPadLo + c] = f;
          fa[row + c] = f;
        }
      }
    }
  }
  __syncwarp();
  const float* fl = fr + kPadLo;
  const AxisNode* A = ev.ay;
  const int nseg = (NY + kSegP - 1) / kSegP;
  for (int sg = lane; sg < nseg; sg += 32) {
    float sv[kSegP];
    seg_slopes([&](int k) -> const AxisNode& { return A[k]; }, NY, (double)ev.DY, sg * kSegP,
               [&](int j) { return (double)fl[j]; }, sv);
#pragma unroll
    for (int t = 0; t < kSegP; ++t) {
      const int c = sg * kSegP + t;
      if (c < NY) sr[c] = sv[t];
    }
  }
  __syncwarp();
  for (int c = lane; c < NY; c += 32) ev.sy[row + c] = sr[c];
}

// Long x-lines and packing: thread (iy, segment) with consecutive iy in a warp,
// so every global access is coalesced.
__global__ void __launch_bounds__(128) fsm_prep2d_cols_long_kernel(
    const Ev2D* __restrict__ evs, const LineBlock* __restrict__ blocks) {
  const LineBlock b = blocks[blockIdx.x];
  const Ev2D& ev = evs[b.ev];
  const int NX = ev.NX, NY = ev.NY;
  const int iy = b.begin + (threadIdx.x & 31);
  const int a = (b.seg + (threadIdx.x >> 5)) * kSegP;
  if (iy >= NY || a >= NX) return;
  const float* fa = ev.fa + iy;
  const float* sy = ev.sy + iy;
  const AxisNode* A = ev.ax;
  auto at = [&](const float* p, int i) {
    return (i >= 0 && i < NX) ? (double)__ldg(p + (size_t)i * NY) : 0.0;
  };
  float sx[kSegP], sxy[kSegP];
  seg_slopes([&](int k) -> const AxisNode& { return A[k]; }, NX, (double)ev.DX, a,
             [&](int i) { return at(fa, i); }, sx);
  seg_slopes([&](int k) -> const AxisNode& { return A[k]; }, NX, (double)ev.DX, a,
             [&](int i) { return at(sy, i); }, sxy);
  float4* nodes = reinterpret_cast<float4*>(ev.nodes) + iy;
#pragma unroll
  for (int t = 0; t < kSegP; ++t) {
    const int i = a + t;
    if (i < NX) {
      const size_t k = (size_t)i * NY;
      nodes[k] = make_float4(__ldg(fa + k), sx[t], __ldg(sy + k), sxy[t]);
    }
  }
}

// --------------------------------------------------- energy-dependent DTAU
// The reference's sums for the energy-dependent free-streaming time: float
// running sums of eps^2 and eps over the converted profile, in cell order
// (src/FreeStream.cpp:404-409).  The rounding of a running float sum depends
// on its order, so one thread adds the cells of an event in that order (the
// DTAU that follows is then bit-identical to the reference's: a reordered sum
// of ~1e6 cells moves it by up to ~1e-4, beyond the tolerance of the moments).
// One block per event: while thread 0 adds a chunk from shared memory (two
// dependent float adds per cell, the sum's floor), the other threads load and
// convert the next chunk, so the one summing thread never waits on memory.
constexpr int kEdepChunk = 4096;
constexpr int kEdepThreads = 256;

__global__ void __launch_bounds__(kEdepThreads) fsm_edep_sums_kernel(const float* const* __restrict__ e_gev,
                                                                    const int* __restrict__ cells, int count,
                                                                    float* sums) {
  __shared__ __align__(16) float buf[2][kEdepChunk];
  const int ev = blockIdx.x;
  if (ev >= count) return;
  const float* __restrict__ e = e_gev[ev];
  const int n = cells[ev];
  const int nch = (n + kEdepChunk - 1) / kEdepChunk;
  const int tid = threadIdx.x;
  // chunk 0: every thread loads
  for (int i = tid; i < kEdepChunk && i < n; i += kEdepThreads) buf[0][i] = to_fm4(__ldg(e + i));
  __syncthreads();
  float num = 0.0f, den = 0.0f;
  for (int c = 0; c < nch; ++c) {
    const int base = c * kEdepChunk, len = min(kEdepChunk, n - base);
    if (tid == 0) {
      const float* __restrict__ b = buf[c & 1];
      int i = 0;
      for (; i + 4 <= len; i += 4) {
        const float4 v = *reinterpret_cast<const float4*>(b + i);
        num = __fadd_rn(num, __fmul_rn(v.x, v.x));
        den = __fadd_rn(den, v.x);
        num = __fadd_rn(num, __fmul_rn(v.y, v.y));
        den = __fadd_rn(den, v.y);
        num = __fadd_rn(num, __fmul_rn(v.z, v.z));
        den = __fadd_rn(den, v.z);
        num = __fadd_rn(num, __fmul_rn(v.w, v.w));
        den = __fadd_rn(den, v.w);
      }
      for (; i < len; ++i) {
        const float v = b[i];
        num = __fadd_rn(num, __fmul_rn(v, v));
        den = __fadd_rn(den, v);
      }
    } else if (c + 1 < nch) {
      const int nb = (c + 1) * kEdepChunk, nlen = min(kEdepChunk, n - nb);
      float* __restrict__ d = buf[(c + 1) & 1];
      for (int i = tid - 1; i < nlen; i += kEdepThreads - 1) d[i] = to_fm4(__ldg(e + nb + i));
    }
    __syncthreads();
  }
  if (tid == 0) {
    sums[2 * ev] = num;
    sums[2 * ev + 1] = den;
  }
}

// ------------------------------------------------------- energy bookkeeping
// The reference's convergence and freeze-out sums (src/FreestreamMilne.cpp:
// 349-354, 531-545): float running sums in cell order of the initial profile
// in fm^-4, of T^{tau tau}, and of T^{tau tau} where e hbar*c > E_FREEZE.  One
// thread adds them in that order, so the sums equal the reference's bit for
// bit; a block per event stages the next chunk of the three arrays into
// shared memory meanwhile (as the E_DEP_FS sums).  A cell outside E_FREEZE
// is staged as +0 and added: inside starts at +0 and x + 0 = x for every
// float the sum can reach, so the result is that of the reference's skip.
constexpr int kEnergyChunk = 1536;

__global__ void __launch_bounds__(kEdepThreads) fsm_energy_sums_kernel(const EvEnergy* __restrict__ evs,
                                                                      int count, float* sums) {
  __shared__ __align__(16) float sb[2][3][kEnergyChunk];
  const int ev = blockIdx.x;
  if (ev >= count) return;
  const EvEnergy E = evs[ev];
  const float hbarc = 0.197326938f;
  const int n = E.n;
  const int nch = (n + kEnergyChunk - 1) / kEnergyChunk;
  const int tid = threadIdx.x;
  auto stage = [&](int c, int t0, int step) {
    const int base = c * kEnergyChunk, len = min(kEnergyChunk, n - base);
    float(*d)[kEnergyChunk] = sb[c & 1];
    for (int i = t0; i < len; i += step) {
      const float a = __ldg(E.e_in + base + i);
      const float t = __ldg(E.T00 + base + i);
      d[0][i] = E.raw ? a : to_fm4(a);
      d[1][i] = t;
      d[2][i] = (__fmul_rn(__ldg(E.e + base + i), hbarc) > E.e_freeze) ? t : 0.0f;
    }
  };
  if (nch > 0) stage(0, tid, kEdepThreads);
  __syncthreads();
  float before = 0.0f, after = 0.0f, inside = 0.0f;
  for (int c = 0; c < nch; ++c) {
    const int len = min(kEnergyChunk, n - c * kEnergyChunk);
    if (tid == 0) {
      const float(*b)[kEnergyChunk] = sb[c & 1];
      for (int i = 0; i < len; ++i) {
        before = __fadd_rn(before, b[0][i]);
        after = __fadd_rn(after, b[1][i]);
        inside = __fadd_rn(inside, b[2][i]);
      }
    } else if (c + 1 < nch) {
      stage(c + 1, tid - 1, kEdepThreads - 1);
    }
    __syncthreads();
  }
  if (tid == 0) {
    sums[3 * ev] = before;
    sums[3 * ev + 1] = after;
    sums[3 * ev + 2] = inside;
  }
}

// ------------------------------------------------------------------ prep 3D
// Eta-pair node arrays of a 3D event: node (e, ix, iy) holds the converted
// energy density of slices e and e+1 at (ix, iy) (and the baryon density of
// both with BARYON), [NE-1][NX][NY], read by the rounding-sensitive exact
// samples of the stream kernel; and the combined planes of every sampled
// (slice, rapidity) pair that reads this eta pair (Ev3D::nodesc), in which the
// stream kernel's lanes (consecutive y) read consecutive nodes.  Thread per node.
__global__ void __launch_bounds__(256) fsm_prep3d_kernel(const Ev3D* __restrict__ evs,
                                                         const CellBlock* __restrict__ blocks) {
  const CellBlock b = blocks[blockIdx.x];
  const Ev3D& ev = evs[b.ev];
  const int NX = ev.NX, NY = ev.NY, NE = ev.NE;
  const int plane = NX * NY;
  const int q = b.begin + threadIdx.x;  // (e * NX + ix) * NY + iy
  if (q >= (NE - 1) * plane) return;
  const int e = q / plane, r = q - e * plane;
  const int ix = r / NY, iy = r - ix * NY;
  const size_t is = ((size_t)ix * NY + iy) * NE + e;  // the reference's cell order
  const float a0 = __ldg(ev.e_gev + is), a1 = __ldg(ev.e_gev + is + 1);
  const float E0 = ev.raw ? a0 : to_fm4(a0), E1 = ev.raw ? a1 : to_fm4(a1);
  // the combined planes that read this eta pair (weights uniform over the
  // block's threads of one pair: broadcast loads), written plane by plane
  const int c0 = __ldg(ev.cw_start + e), c1 = __ldg(ev.cw_start + e + 1);
  if (ev.baryon) {
    const float B0 = __ldg(ev.nB + is), B1 = __ldg(ev.nB + is + 1);
    reinterpret_cast<float4*>(ev.nodes3)[q] = make_float4(E0, E1, B0, B1);
    float2* C = reinterpret_cast<float2*>(ev.nodesc);
    for (int c = c0; c < c1; ++c) {
      const CombW w = ev.cw[c];
      C[(size_t)w.plane * plane + r] = make_float2(fmaf(w.w0, E0, w.w1 * E1), fmaf(w.b0, B0, w.b1 * B1));
    }
  } else {
    reinterpret_cast<float2*>(ev.nodes3)[q] = make_float2(E0, E1);
    float* C = reinterpret_cast<float*>(ev.nodesc);
    for (int c = c0; c < c1; ++c) {
      const CombW w = ev.cw[c];
      C[(size_t)w.plane * plane + r] = fmaf(w.w0, E0, w.w1 * E1);
    }
  }
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

__device__ __forceinline__ float4 node_at(const float4* __restrict__ sn, const float4* __restrict__ g,
                                          bool smem, int i, int j, int fx0, int fy0, int FW, int NY) {
  return smem ? sn[(i - fx0) * FW + (j - fy0)] : __ldg(g + (size_t)i * NY + j);
}

// One sample with the reference's own float arithmetic (src/FreeStream.cpp:
// 187-246): shifted point, correctly rounded index division, in-grid test,
// bilinear value and the bicubic patch inside the spline's open domain.  Used
// for the rare samples whose in-grid decision depends on the rounding.
__device__ __forceinline__ float exact_sample(const Ev2D& ev, const float4* __restrict__ sn, bool smem,
                                           int fx0, int fy0, int FW, int FH, float x, float y,
                                           float c, float s, int* err) {
  const int NX = ev.NX, NY = ev.NY;
  const float xn = __fsub_rn(x, __fmul_rn(c, ev.DTAU));
  const float yn = __fsub_rn(y, __fmul_rn(s, ev.DTAU));
  const float qx = __fdiv_rn(__fsub_rn(xn, ev.xmin), ev.DX);
  const float qy = __fdiv_rn(__fsub_rn(yn, ev.ymin), ev.DY);
  const float fxf = floorf(qx), fyf = floorf(qy);
  if (!(fxf >= 1.0f && fxf < (float)(NX - 1) && fyf >= 1.0f && fyf < (float)(NY - 1))) return 0.0f;
  const int i = (int)fxf, j = (int)fyf;
  (void)FH;
  const float4* g = reinterpret_cast<const float4*>(ev.nodes);
  const float4 n00 = node_at(sn, g, smem, i, j, fx0, fy0, FW, NY);
  const float4 n01 = node_at(sn, g, smem, i, j + 1, fx0, fy0, FW, NY);
  const float4 n10 = node_at(sn, g, smem, i + 1, j, fx0, fy0, FW, NY);
  const float4 n11 = node_at(sn, g, smem, i + 1, j + 1, fx0, fy0, FW, NY);
  const float t = qx - fxf, u = qy - fyf;
  float v = ((1.0f - t) * (1.0f - u) * n00.x) + (t * (1.0f - u) * n10.x) + ((1.0f - t) * u * n01.x) +
            (t * u * n11.x);
  if ((ev.xmin < xn) && (xn < ev.xmax_i) && (ev.ymin < yn) && (yn < ev.ymax_i)) {
    float H0, H1, G0, G1, K0, K1, L0, L1;
    hermite(t, H0, H1, G0, G1);
    hermite(u, K0, K1, L0, L1);
    const float r0 = H0 * n00.x + H1 * n10.x + G0 * n00.y + G1 * n10.y;
    const float r1 = H0 * n01.x + H1 * n11.x + G0 * n01.y + G1 * n11.y;
    const float s0 = H0 * n00.z + H1 * n10.z + G0 * n00.w + G1 * n10.w;
    const float s1 = H0 * n01.z + H1 * n11.z + G0 * n01.w + G1 * n11.w;
    const float cval = K0 * r0 + K1 * r1 + L0 * s0 + L1 * s1;
    if (cval > 0.0f) v = cval;
  }
  return v;
}

// ------------------------------------------------------- TMA / mbarrier helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on an mbarrier phase: returns false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Contiguous bulk copy global -> shared (16-byte multiple) completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Warp-cooperative staging of one source window (boxH rows x boxW nodes, node
// (0,0) = grid node (wx0, wy0)) with one bulk copy per in-grid row segment, all
// completing on `bar`; optionally also the phi_p table.  Window slots outside
// the grid are left unwritten: only samples that the in-grid test masks out
// read them.  Called by all 32 lanes of one warp.
__device__ __forceinline__ void stage_window(float4* buf, const float4* __restrict__ nodes, int NX,
                                             int NY, int wx0, int wy0, int boxW, int boxH,
                                             void* tab_dst, const void* tab_src, uint32_t tab_bytes,
                                             uint64_t* bar) {
  const int lane = threadIdx.x & 31;
  fence_proxy_async();  // the buffer was last read through the generic proxy
  const int c0 = max(0, wy0), c1 = min(NY - 1, wy0 + boxW - 1);
  const uint32_t rowbytes = (c1 >= c0) ? (uint32_t)(c1 - c0 + 1) * 16u : 0u;
  uint32_t bytes = 0;
  for (int r = lane; r < boxH; r += 32) {
    const int gr = wx0 + r;
    if (gr >= 0 && gr < NX) bytes += rowbytes;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
  if (lane == 0) {
    mbar_expect_tx(bar, bytes + tab_bytes);
    if (tab_bytes) bulk_load(tab_dst, tab_src, tab_bytes, bar);
  }
  __syncwarp();
  if (rowbytes) {
    for (int r = lane; r < boxH; r += 32) {
      const int gr = wx0 + r;
      if (gr >= 0 && gr < NX)
        bulk_load(buf + r * boxW + (c0 - wy0), nodes + (size_t)gr * NY + c0, rowbytes, bar);
    }
  }
}

// One phi_p run of one 32 x 32 output tile, on a staged window `win`
// (boxW columns per row) whose node (0, 0) is grid node (wx0, wy0).  Lane l of
// warp w owns the cells (x0 + 4w + k, y0 + l), k = 0..3.  For each phi_p every
// cell of the tile shifts by the same vector, so the per-phi_p table gives the
// source offset and the Hermite weights once for all cells; each cell applies a
// first-order correction for its own float-rounded coordinate (the reference
// positions samples relative to the float cell coordinate).  The y-direction
// Hermite pass of a node row -- the (value, x-slope) pair, one packed-FMA chain
// -- is shared by the two cells that use it, so a thread evaluates 5 node rows
// for its 4 samples.  Where the spline is not positive the reference falls back
// to bilinear interpolation (src/FreeStream.cpp:245-246); that is rare, so it
// is evaluated only in warps where some sample needs it.  Moments accumulate
// in FP32 chunks of ev.chunk (16 or 32, tuned) phi_p folded into FP32 totals
// (two-level summation).
//
// kInterior: every sample of the run provably lands inside the grid, so the
// in-grid test (src/FreeStream.cpp:213) is skipped.
//
// Consecutive phi_p often share the integer offset (the source point moves by
// at most about one cell per phi_p step): the thread keeps the 2 x (K + 1)
// nodes of the last offset in registers (nd0/nd1, node values of the grid,
// the same in every staged window) and reloads them only when the offset
// changes.  Out-of-grid window entries are never copied; samples that would
// read them are masked below, whatever the registers hold.
//
// `stab` holds the table entries of the run's phi_p p0 .. p1 - 1.
template <bool kInterior>
__device__ __forceinline__ void stream2d_run(const Ev2D& ev, const float4* __restrict__ win, int wx0,
                                             int wy0, int boxW, const float4* __restrict__ stab,
                                             int p0, int p1, int ixb, int iy, int wxa, int wxb,
                                             int wya, int wyb, int wxn, float ey,
                                             const float (&ex)[kCellsPerThread],
                                             float (&a0)[kCellsPerThread],
                                             float2 (&a12)[kCellsPerThread],
                                             float2 (&a34)[kCellsPerThread],
                                             float4 (&nd0)[kCellsPerThread + 1],
                                             float4 (&nd1)[kCellsPerThread + 1], int& pox,
                                             int& poy, float2* __restrict__ stot, int* err) {
  constexpr int K = kCellsPerThread;
  const int NX = ev.NX, NY = ev.NY;
  const float2 ey2 = make_float2(ey, ey);
  // phi_p in pieces that end at the fold points of the two-level sum, so the
  // inner loop carries no fold test
  for (int pc = p0; pc < p1;) {
    const int pe = min(p1, (pc | (ev.chunk - 1)) + 1);
    // Runs near the boundary: the warp's lanes test the piece's phi_p at once
    // (does any sample of this warp reach the grid; does every sample land two
    // or more nodes inside, so that no in-grid test is needed), and the warp
    // visits only the phi_p that reach it, in order.  A phi_p that reaches no
    // sample of the warp adds nothing to its sums.
    unsigned vis_mask = 0xffffffffu, in_mask = 0xffffffffu;
    if (!kInterior) {
      const int pl = pc + (threadIdx.x & 31);
      bool vis = false, ins = false;
      if (pl < pe) {
        const float4 tl4 = stab[kPhiTab2D * (pl - p0) + 5];
        const int lox = __float_as_int(tl4.z), loy = (int)(short)(__float_as_int(tl4.w) & 0xffff);
        // the warp's cells: x wxa .. wxb inside the grid (wxa .. wxa + wxn - 1
        // computed), y wya .. wyb inside the grid
        const int wa = wxa + lox, wb = wxb + lox;
        vis = (wb + 1 >= 1) && (wa - 1 <= NX - 2) && (wyb + loy + 1 >= 1) && (wya + loy - 1 <= NY - 2);
        ins = (wa >= 2) && (wa + wxn - 1 <= NX - 3) && (wya + loy >= 2) && (wyb + loy <= NY - 3);
      }
      vis_mask = __ballot_sync(0xffffffffu, vis);
      in_mask = __ballot_sync(0xffffffffu, ins);
    }
    unsigned m = kInterior ? 0u : vis_mask;
    for (int p = pc; kInterior ? (p < pe) : (m != 0u); ++p) {
      if (!kInterior) {
        p = pc + __ffs(m) - 1;
        m &= m - 1u;
      }
      const float4* e = stab + kPhiTab2D * (p - p0);
      const float4 wx = e[0], dwx = e[1], wy = e[2], dwy = e[3], tu = e[5];
      const int ox = __float_as_int(tu.z), oyn = __float_as_int(tu.w);
      const int oy = (int)(short)(oyn & 0xffff);
      const int j = iy + oy, i0 = ixb + ox;
      // y weights of this lane, first-order corrected for its own coordinate
      const float2 Kp = __ffma2_rn(ey2, make_float2(dwy.x, dwy.y), make_float2(wy.x, wy.y));
      const float2 Lp = __ffma2_rn(ey2, make_float2(dwy.z, dwy.w), make_float2(wy.z, wy.w));
      const float4* rowp = win + (i0 - wx0) * boxW + (j - wy0);
      if (ox != pox || oy != poy) {  // uniform over the block: the offset is per phi_p
#pragma unroll
        for (int r = 0; r <= K; ++r) {
          nd0[r] = rowp[r * boxW];
          nd1[r] = rowp[r * boxW + 1];
        }
        pox = ox;
        poy = oy;
      }
      float cv[K];
      float2 VDp = make_float2(0.f, 0.f);
#pragma unroll
      for (int r = 0; r <= K; ++r) {
        const float4 n0 = nd0[r], n1 = nd1[r];
        // y pass of the node row: (value, x-slope) interpolated to the sample's y
        float2 VD = __fmul2_rn(make_float2(Kp.x, Kp.x), make_float2(n0.x, n0.y));
        VD = __ffma2_rn(make_float2(Kp.y, Kp.y), make_float2(n1.x, n1.y), VD);
        VD = __ffma2_rn(make_float2(Lp.x, Lp.x), make_float2(n0.z, n0.w), VD);
        VD = __ffma2_rn(make_float2(Lp.y, Lp.y), make_float2(n1.z, n1.w), VD);
        if (r > 0) {
          const int k = r - 1;
          const float2 ex2 = make_float2(ex[k], ex[k]);
          const float2 HG0 = __ffma2_rn(ex2, make_float2(dwx.x, dwx.y), make_float2(wx.x, wx.y));
          const float2 HG1 = __ffma2_rn(ex2, make_float2(dwx.z, dwx.w), make_float2(wx.z, wx.w));
          const float2 cc = __ffma2_rn(HG1, VD, __fmul2_rn(HG0, VDp));
          cv[k] = cc.x + cc.y;  // bicubic
        }
        VDp = VD;
      }
      // bilinear where the bicubic value is not positive (or not a number)
      bool pos = true;
#pragma unroll
      for (int k = 0; k < K; ++k) pos = pos && (cv[k] > 0.0f);
      if (__any_sync(0xffffffffu, !pos)) {
        const float uu = tu.y + ey;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!(cv[k] > 0.0f)) {
            const float4 a00 = nd0[k], a01 = nd1[k];
            const float4 a10 = nd0[k + 1], a11 = nd1[k + 1];
            const float B0 = fmaf(uu, a01.x - a00.x, a00.x);
            const float B1 = fmaf(uu, a11.x - a10.x, a10.x);
            cv[k] = fmaf(tu.x + ex[k], B1 - B0, B0) * ev.fb_scale;
          }
        }
      }
      const float4 mw = e[4];
      if (!kInterior && !((in_mask >> (p - pc)) & 1u)) {
        const bool nearx = (oyn >> 16) & 1, neary = (oyn >> 17) & 1;
        const bool in_y = (unsigned)(j - 1) <= (unsigned)(NY - 3);
        if (!(nearx || neary)) {
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const bool in = in_y && ((unsigned)(i0 + k - 1) <= (unsigned)(NX - 3));
            cv[k] = in ? cv[k] : 0.0f;
          }
        } else {
          // the fraction lies within 1e-3 of an integer: a sample next to the
          // grid boundary may fall in or out with the rounding of its float
          // position, so those samples are decided and evaluated with the
          // reference arithmetic
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const int ik = i0 + k;
            const bool cx = (ik >= 1) && (ik <= NX - 2);
            const bool ux = nearx && (ik == 0 || ik == 1 || ik == NX - 2 || ik == NX - 1);
            const bool uy = neary && (j == 0 || j == 1 || j == NY - 2 || j == NY - 1);
            if (ixb + k < NX && iy < NY && (ux || uy) && (ux || cx) && (uy || in_y)) {
              const float x = __fadd_rn(__fmul_rn((float)(ixb + k), ev.DX), ev.xmin);
              const float y = __fadd_rn(__fmul_rn((float)iy, ev.DY), ev.ymin);
              cv[k] = exact_sample(ev, win, true, wx0, wy0, boxW, 0, x, y, mw.x, mw.y, err);
            } else {
              cv[k] = (cx && in_y && !ux && !uy) ? cv[k] : 0.0f;
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const float2 v2 = make_float2(cv[k], cv[k]);
        a0[k] += cv[k];
        a12[k] = __ffma2_rn(v2, make_float2(mw.x, mw.y), a12[k]);
        a34[k] = __ffma2_rn(v2, make_float2(mw.z, mw.w), a34[k]);
      }
    }
    if ((pe & (ev.chunk - 1)) == 0) {
      // second level of the two-level sum, thread-private slots in shared memory
      // packed slots: a0 of cells (0, 1) and (2, 3), then a12[k], a34[k]
#pragma unroll
      for (int k = 0; k < K; k += 2)
        stot[(k >> 1) * kThreads2D] = __fadd2_rn(stot[(k >> 1) * kThreads2D], make_float2(a0[k], a0[k + 1]));
#pragma unroll
      for (int k = 0; k < K; ++k) {
        stot[(2 + k) * kThreads2D] = __fadd2_rn(stot[(2 + k) * kThreads2D], a12[k]);
        stot[(6 + k) * kThreads2D] = __fadd2_rn(stot[(6 + k) * kThreads2D], a34[k]);
        a0[k] = 0.0f;
        a12[k] = a34[k] = make_float2(0.f, 0.f);
      }
    }
    pc = pe;
  }
}

// Persistent kernel over 32 x 32 output tiles taken from a global work list
// (largest events first).  Per tile, the event's phi_p table and the source
// window of each phi_p run are staged into shared memory by bulk copies
// (cp.async.bulk, one per in-grid window row) completing on mbarriers,
// double-buffered so the next run's window loads while the current one is
// computed.  Every mbarrier wait gives up after wait_polls polls; on time-out
// the CTA records an error, waits (bounded) until every copy it issued has
// landed, and leaves.
__global__ void __launch_bounds__(kThreads2D, 2) fsm_stream2d_kernel(const Ev2D* __restrict__ evs,
                                                                     const Tile2D* __restrict__ tiles,
                                                                     int ntiles, int box_cap,
                                                                     Counters* ctr, int* err,
                                                                     int wait_polls) {
  extern __shared__ __align__(128) float4 smem4[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int s_tile;
  constexpr int kTabF4 = kMaxRunPhi2D * kPhiTab2D;  // one run table (a 128-byte multiple)
  static_assert(kTabF4 % 8 == 0, "run tables keep the windows 128-byte aligned");
  float4* const tab0 = smem4;
  float4* const tab1 = smem4 + kTabF4;
  float4* const buf0 = smem4 + 2 * kTabF4;
  float4* const buf1 = buf0 + box_cap;
  // per-thread moment totals, packed pairs: [a0 of cells 0,1], [a0 of 2,3],
  // a12[0..3], a34[0..3]
  static_assert(kCellsPerThread == 4 && kTotSlots2D == 20, "packed moment totals of 4 cells");
  float2* const stot = reinterpret_cast<float2*>(buf1 + box_cap) + threadIdx.x;
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase0 = 0u, phase1 = 0u;
  constexpr int K = kCellsPerThread;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctr->tile2d, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= ntiles) return;
    const Tile2D tl = tiles[t];
    const Ev2D& ev = evs[tl.ev];
    const int sh = tl.shape;
    const int nch = ev.nch[sh];
    const Chunk2D* __restrict__ chunks = ev.chunks + ev.choff[sh];
    const float4* __restrict__ gnodes = reinterpret_cast<const float4*>(ev.nodes);
    if (warp == 0) {
      const Chunk2D c0 = chunks[0];
      stage_window(buf0, gnodes, ev.NX, ev.NY, tl.x0 + c0.ox0 - 1, tl.y0 + c0.oy0 - 1, win_w(c0, sh),
                   win_h(c0, sh), tab0, ev.tab + c0.p0,
                   (uint32_t)(c0.p1 - c0.p0) * (uint32_t)sizeof(PhiEntry2D), &bars[0]);
    }
    // the tile's shape: lanes run along y in groups of ly cells (32 / ly
    // groups of K x cells side by side), wy warps stacked along y
    const int lyl = shape_ly_log(sh), wyl = shape_wy_log(sh);
    const int ly = 32 >> lyl, gx = 1 << lyl, wxcount = kWarps2D >> wyl;
    const int wxi = warp & (wxcount - 1), wyi = warp >> (3 - wyl);
    const int TX = K * gx * wxcount, TY = ly << wyl;
    // per-thread cell constants
    const int iy = tl.y0 + wyi * ly + (lane & (ly - 1));
    const int ixb = tl.x0 + K * (wxi * gx + (lane >> (5 - lyl)));
    // the last cell the tile stores (x1, y1 <= the grid's size)
    const int x_hi = min(tl.x0 + TX, tl.x1) - 1, y_hi = min(tl.y0 + TY, tl.y1) - 1;
    // this warp's cells
    const int wxa = tl.x0 + K * wxi * gx, wxn = K * gx;
    const int wxb = min(wxa + wxn - 1, x_hi);
    const int wya = tl.y0 + wyi * ly, wyb = min(wya + ly - 1, y_hi);
    const float DX = ev.DX, DY = ev.DY, xmin = ev.xmin, ymin = ev.ymin;
    const float y = __fadd_rn(__fmul_rn((float)iy, DY), ymin);  // src/FreeStream.cpp:164
    // the cells' rounding offsets in cells (a first-order correction, so one
    // reciprocal per tile instead of a division per cell)
    const double rdx = 1.0 / (double)DX, rdy = 1.0 / (double)DY;
    const float ey = (float)(((double)y - ((double)ymin + (double)iy * (double)DY)) * rdy);
    float ex[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int ix = ixb + k;
      const float x = __fadd_rn(__fmul_rn((float)ix, DX), xmin);
      ex[k] = (float)(((double)x - ((double)xmin + (double)ix * (double)DX)) * rdx);
    }
    float a0[K];
    float2 a12[K], a34[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      a0[k] = 0.0f;
      a12[k] = a34[k] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int m = 0; m < kTotSlots2D / 2; ++m) stot[m * kThreads2D] = make_float2(0.f, 0.f);
    float4 nd0[K + 1], nd1[K + 1];
    int pox = INT_MIN, poy = INT_MIN;  // no nodes held yet
    // warps whose cells all lie past the grid's edge skip the runs
    const bool live = wxa <= x_hi && wya <= y_hi;

    for (int c = 0; c < nch; ++c) {
      const int b = c & 1;
      if (warp == 0 && c + 1 < nch) {
        const Chunk2D cn = chunks[c + 1];
        stage_window(b ? buf0 : buf1, gnodes, ev.NX, ev.NY, tl.x0 + cn.ox0 - 1, tl.y0 + cn.oy0 - 1,
                     win_w(cn, sh), win_h(cn, sh), b ? tab0 : tab1, ev.tab + cn.p0,
                     (uint32_t)(cn.p1 - cn.p0) * (uint32_t)sizeof(PhiEntry2D), &bars[b ^ 1]);
      }
      const uint32_t ph = b ? phase1 : phase0;
      const bool ok = mbar_wait(&bars[b], ph, wait_polls);
      if (b) phase1 ^= 1u;
      else phase0 ^= 1u;
      if (__syncthreads_or(!ok)) {
        // a staged copy did not complete in time: record it; before leaving,
        // let both copies this CTA may have in flight land (run c's, and run
        // c + 1's when it was issued) so that none writes into shared memory
        // after the CTA has exited
        if (threadIdx.x == 0) {
          atomicAdd(err + 1, 1);
          mbar_wait(&bars[b], ph, kWaitPolls);
          if (c + 1 < nch) mbar_wait(&bars[b ^ 1], b ? phase0 : phase1, kWaitPolls);
        }
        return;
      }
      const Chunk2D ch = chunks[c];
      const int wx0 = tl.x0 + ch.ox0 - 1, wy0 = tl.y0 + ch.oy0 - 1, boxW = win_w(ch, sh);
      const float4* win = b ? buf1 : buf0;
      const float4* stab = b ? tab1 : tab0;
      // every sample of this run lands at least one node inside the grid
      // boundary (cells past the grid edge are computed but never stored)
      const bool interior = (tl.x0 + ch.ox0 >= 2) && (x_hi + ch.ox1 <= ev.NX - 3) &&
                            (tl.y0 + ch.oy0 >= 2) && (y_hi + ch.oy1 <= ev.NY - 3);
      if (!live) {
      } else if (interior) {
        stream2d_run<true>(ev, win, wx0, wy0, boxW, stab, ch.p0, ch.p1, ixb, iy, wxa, wxb, wya, wyb, wxn,
                           ey, ex, a0, a12, a34, nd0, nd1, pox, poy, stot, err);
      } else {
        stream2d_run<false>(ev, win, wx0, wy0, boxW, stab, ch.p0, ch.p1, ixb, iy, wxa, wxb, wya, wyb, wxn,
                            ey, ex, a0, a12, a34, nd0, nd1, pox, poy, stot, err);
      }
      __syncthreads();  // buffer b is free for the load of run c + 2
    }
    // T = (sum over DIM_RAP identical rapidity copies) * d_phip / TAU
    // (src/LandauMatch.cpp:104), one scale per tile; T^yy = sum v sin^2 =
    // S1 - S_cc.
    const float R = (float)ev.NR, dphi = ev.d_phip, TAU = ev.TAU;
    const float tscale = __fdiv_rn(__fmul_rn(R, dphi), TAU);
    const size_t DIM = (size_t)ev.NX * ev.NY;
    float* T = ev.T;
    if (ev.charge) {
      // J = (rapidity sum) * DRAP * d_phip (src/LandauMatch.cpp:137-140);
      // in 2D the hypertrig rows are (1, cos, sin, 0)
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (ixb + k > x_hi || iy > y_hi) continue;
        const size_t is = (size_t)(ixb + k) * ev.NY + iy;
        const float2 p0 = stot[(k >> 1) * kThreads2D], p12 = stot[(2 + k) * kThreads2D];
        const float s0 = ((k & 1) ? p0.y : p0.x) + a0[k];
        const float s1 = p12.x + a12[k].x;
        const float s2 = p12.y + a12[k].y;
        ev.J[0 * DIM + is] = __fmul_rn(__fmul_rn(__fmul_rn(s0, ev.jscale), ev.DRAP), dphi);
        ev.J[1 * DIM + is] = __fmul_rn(__fmul_rn(__fmul_rn(s1, ev.jscale), ev.DRAP), dphi);
        ev.J[2 * DIM + is] = __fmul_rn(__fmul_rn(__fmul_rn(s2, ev.jscale), ev.DRAP), dphi);
        ev.J[3 * DIM + is] = 0.0f;
      }
      continue;
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (ixb + k > x_hi || iy > y_hi) continue;
      const float2 p0 = stot[(k >> 1) * kThreads2D], p12 = stot[(2 + k) * kThreads2D],
                   p34 = stot[(6 + k) * kThreads2D];
      const float tot[5] = {((k & 1) ? p0.y : p0.x) + a0[k], p12.x + a12[k].x, p12.y + a12[k].y,
                            p34.x + a34[k].x, p34.y + a34[k].y};
      float S[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) S[m] = __fmul_rn(tot[m], tscale);
      const size_t is = (size_t)(ixb + k) * ev.NY + iy;
      T[0 * DIM + is] = S[0];
      T[1 * DIM + is] = S[1];
      T[2 * DIM + is] = S[2];
      T[3 * DIM + is] = 0.0f;
      T[4 * DIM + is] = S[3];
      T[5 * DIM + is] = S[4];
      T[6 * DIM + is] = 0.0f;
      T[7 * DIM + is] = S[0] - S[3];
      T[8 * DIM + is] = 0.0f;
      T[9 * DIM + is] = 0.0f;
    }
  }
}

// ---------------------------------------------------------------- stream 3D
// Node of the eta-pair arrays: (E[e], E[e+1], B[e], B[e+1]) with baryons,
// (E[e], E[e+1]) without.
template <bool kB> struct Node3D;
template <> struct Node3D<true> { using T = float4; };
template <> struct Node3D<false> { using T = float2; };
__device__ __forceinline__ float node_b0(const float4& n) { return n.z; }
__device__ __forceinline__ float node_b1(const float4& n) { return n.w; }
__device__ __forceinline__ float node_b0(const float2&) { return 0.0f; }
__device__ __forceinline__ float node_b1(const float2&) { return 0.0f; }
// Linear interpolation a + w (b - a) of both components, with b - a rounded
// once (b + (-1) a is exact before the rounding) as the scalar fmaf(w, b - a, a).
__device__ __forceinline__ float2 lerp2(float2 w, float2 a, float2 b) {
  return __ffma2_rn(w, __ffma2_rn(a, make_float2(-1.0f, -1.0f), b), a);
}

// One sample with the reference's own float arithmetic (src/FreeStream.cpp:
// 193-276): shifted point, correctly rounded index division, in-grid test and
// trilinear interpolation (the eta fraction and slice from the host table).
// Used for the rare samples whose in-grid decision depends on the rounding.
// N points at the eta pair of the sample's slice.  Returns false for a sample
// outside the grid.
template <bool kB>
__device__ __forceinline__ bool exact_sample3d(const Ev3D& ev, const typename Node3D<kB>::T* __restrict__ N,
                                               float x, float y, float c, float s, float D, float et,
                                               float rf0, float rf1, float rb0, float rb1, float& v,
                                               float& vb) {
  const int NX = ev.NX, NY = ev.NY;
  const float xn = __fsub_rn(x, __fmul_rn(c, D));
  const float yn = __fsub_rn(y, __fmul_rn(s, D));
  const float qx = __fdiv_rn(__fsub_rn(xn, ev.xmin), ev.DX);
  const float qy = __fdiv_rn(__fsub_rn(yn, ev.ymin), ev.DY);
  const float fx = floorf(qx), fy = floorf(qy);
  if (!(fx >= 1.0f && fx < (float)(NX - 1) && fy >= 1.0f && fy < (float)(NY - 1))) return false;
  const int i = (int)fx, j = (int)fy;
  const float t = qx - fx, u = qy - fy;
  const size_t k = (size_t)i * NY + j;
  const auto n00 = __ldg(N + k), n10 = __ldg(N + k + NY), n01 = __ldg(N + k + 1),
             n11 = __ldg(N + k + NY + 1);
  auto lin = [&](float a00, float a10, float a01, float a11) {
    return (1.0f - t) * (1.0f - u) * a00 + t * (1.0f - u) * a10 + (1.0f - t) * u * a01 + t * u * a11;
  };
  v = (1.0f - et) * (lin(n00.x, n10.x, n01.x, n11.x) * rf0) +
      et * (lin(n00.y, n10.y, n01.y, n11.y) * rf1);
  if (kB)
    vb = (1.0f - et) * (lin(node_b0(n00), node_b0(n10), node_b0(n01), node_b0(n11)) * rb0) +
         et * (lin(node_b1(n00), node_b1(n10), node_b1(n01), node_b1(n11)) * rb1);
  return true;
}

// exact_sample3d for (eta slice, rapidity) pair rp / irap: its eta pair, eta
// fraction and rapidity weights are read here, on the rare exact path, rather
// than held in registers through the phi_p loop.
template <bool kB>
__device__ __forceinline__ bool exact_sample3d_pair(const Ev3D& ev, const RapEta* __restrict__ rp, int irap,
                                                    float x, float y, float c, float s, float& v, float& vb) {
  const RapEta r = *rp;
  const int NR = ev.NR;
  const float rf0 = __ldg(ev.rapf + r.efl * NR + irap), rf1 = __ldg(ev.rapf + (r.efl + 1) * NR + irap);
  float rb0 = 0.0f, rb1 = 0.0f;
  if (kB) {
    rb0 = __ldg(ev.rapfB + r.efl * NR + irap);
    rb1 = __ldg(ev.rapfB + (r.efl + 1) * NR + irap);
  }
  const auto* N = reinterpret_cast<const typename Node3D<kB>::T*>(ev.nodes3) + (size_t)r.efl * ev.NX * ev.NY;
  return exact_sample3d<kB>(ev, N, x, y, c, s, r.D, r.efrac, rf0, rf1, rb0, rb1, v, vb);
}

// Persistent kernel over 32 x 32 output tiles of one eta slice (largest
// rapidity count first).  For a fixed slice and rapidity node the shift length
// D is the same for every cell, so for each phi_p the whole tile shifts by one
// vector: the host table gives the integer offset and the fractions once, each
// cell corrects the fraction for its own float-rounded coordinate, and the
// lanes (consecutive y) read consecutive nodes of the (slice, rapidity) pair's
// combined plane, in which the prep kernel has already interpolated the two
// source eta slices with their rapidity weights: one load per node for both
// fields, a bilinear interpolation per sample.  Lane l of warp
// w owns the cells (x0 + 4w + k, y0 + l); a thread interpolates 5 x rows for
// its 4 samples and keeps those 2 x 5 nodes in registers
// while consecutive phi_p share the offset.  phi_p whose whole tile lands outside the grid are
// skipped; runs inside it skip the in-grid test.  Moments: FP32 partial sums
// over 16 phi_p folded, with the rapidity factors (src/LandauMatch.cpp:76-143),
// straight into T^{mu nu} / J^mu in thread-private shared-memory slots (per
// cell T 0..9, J 10..13): no per-rapidity slots, so that the shared memory
// of two CTAs leaves L1 room for the tiles' node footprints.
// Combined-plane nodes (Ev3D::nodesc): (E, B) with baryon charge, E without.
template <bool kB> struct NodeC;
template <> struct NodeC<true> { using T = float2; };
template <> struct NodeC<false> { using T = float; };
__device__ __forceinline__ float2 lerpc(float w, float2 a, float2 b) { return lerp2(make_float2(w, w), a, b); }
__device__ __forceinline__ float lerpc(float w, float a, float b) { return fmaf(w, fmaf(a, -1.0f, b), a); }
__device__ __forceinline__ float comb_e(float2 n) { return n.x; }
__device__ __forceinline__ float comb_e(float n) { return n; }
__device__ __forceinline__ float comb_b(float2 n) { return n.y; }
__device__ __forceinline__ float comb_b(float) { return 0.0f; }

template <bool kB>
constexpr int slots3d() {
  return kB ? kSlots3DBaryon : kSlots3D;
}

// The phi_p loop of one rapidity node for one tile (nodes of eta pair efl).
template <bool kB>
__device__ __forceinline__ void stream3d_rap(const Ev3D& ev, int ixb, int iy, int wxa, int wxb,
                                             int wxn, int wya, int wyb, int wyn, float y, float ey,
                                             const float (&ex)[kCellsPerThread],
                                             const bool (&act)[kCellsPerThread],
                                             const typename NodeC<kB>::T* __restrict__ Nc,
                                             const PhiEntry3D* __restrict__ tab, int irap,
                                             const RapEta* __restrict__ rp, float jw,
                                             float2* __restrict__ sl) {
  using NodeT = typename NodeC<kB>::T;
  constexpr int K = kCellsPerThread;
  constexpr int kS = slots3d<kB>();
  const int NX = ev.NX, NY = ev.NY, NP = ev.NPHI;
  // moment partial sums: (energy, baryon) pairs of the weights 1, cos, sin
  // and the energy-only cos^2, cos sin, sin^2
  float2 a01[K], a1c[K], a1s[K];
  float2 a34[K];  // (cos^2, cos sin) moments of the energy
  float a5[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    a01[k] = a1c[k] = a1s[k] = make_float2(0.f, 0.f);
    a34[k] = make_float2(0.f, 0.f);
    a5[k] = 0.0f;
  }
  // the nodes of the pair's combined plane (eta interpolation and rapidity
  // weights applied once per node by the prep kernel): (E, B) float2 with
  // baryons, E float without; those of the last offset stay in registers
  constexpr bool kCache = true;
  NodeT n0[K + 1], n1[K + 1];
  int pox = INT_MIN, poy = INT_MIN;  // no nodes held yet
  // phi_p in blocks of 32: the warp's lanes test the 32 phi_p at once (does
  // any sample of this warp reach the grid; does every sample land two or
  // more nodes inside) and the warp then visits only the phi_p that reach it,
  // in order, folding the partial sums at the same points (every kPhiChunk
  // phi_p) as a visit of every phi_p would
  static_assert(32 % kPhiChunk == 0, "fold points inside a 32-phi_p block");
  const int lane = threadIdx.x & 31;
  for (int pb = 0; pb < NP; pb += 32) {
    unsigned vis_mask, in_mask;
    {
      const int p = pb + lane;
      bool vis = false, ins = false;
      if (p < NP && wxa <= wxb && wya <= wyb) {
        const PhiEntry3D e = tab[p];
        const int ox = e.ox;
        const int oy = (int)(short)(e.oy_near & 0xffff);
        // sample floor indices of this warp's stored cells, rows wxa .. wxb
        // and columns wya .. wyb, shifted (one more either side when the
        // fraction is near an integer)
        const int ya = wya + oy, yb = wyb + oy;
        const int wa = wxa + ox, wb = wxb + ox;
        vis = !((yb + 1 < 1) || (ya - 1 > NY - 2) || (wb + 1 < 1) || (wa - 1 > NX - 2));
        // every sample of this warp lands two or more nodes inside the grid:
        // all its lanes' rows wxa .. wxa + wxn - 1 and columns wya .. wya +
        // wyn - 1 (cells past the grid edge included, so that their loads
        // stay inside the arrays)
        ins = (wa >= 2) && (wxa + wxn - 1 + ox <= NX - 3) && (ya >= 2) && (wya + wyn - 1 + oy <= NY - 3);
      }
      vis_mask = __ballot_sync(0xffffffffu, vis);
      in_mask = __ballot_sync(0xffffffffu, ins);
    }
    for (int pc = pb; pc < min(NP, pb + 32); pc += kPhiChunk) {
      const unsigned cm = (vis_mask >> (pc - pb)) & ((1u << kPhiChunk) - 1u);
      unsigned m = cm;
      while (m) {
        const int bit = __ffs(m) - 1;
        m &= m - 1u;
        const int p = pc + bit;
        const PhiEntry3D e = tab[p];
        const int ox = e.ox;
        const int oy = (int)(short)(e.oy_near & 0xffff);
        {
          const int i0 = ixb + ox, j = iy + oy;
          const bool inside = (in_mask >> (p - pb)) & 1u;
          if (!kCache || ox != pox || oy != poy) {  // uniform over the block: the offset is per phi_p
            if (inside) {
              // one base index, rows NY apart
              const int q0 = i0 * NY + j;
#pragma unroll
              for (int r = 0; r <= K; ++r) {
                n0[r] = __ldg(Nc + (q0 + r * NY));
                n1[r] = __ldg(Nc + (q0 + r * NY + 1));
              }
            } else {
              // clamped indices keep the loads of edge lanes inside the arrays
              // (their samples are masked below); inside the grid they are exact
              const int jj = min(max(j, 0), NY - 2);
#pragma unroll
              for (int r = 0; r <= K; ++r) {
                const int i = min(max(i0 + r, 0), NX - 1);
                const NodeT* q = Nc + (size_t)i * NY + jj;
                n0[r] = __ldg(q);
                n1[r] = __ldg(q + 1);
              }
            }
            pox = ox;
            poy = oy;
          }
          const float uc = e.u + ey;
          float v[K], vb[K];
          NodeT Bp = NodeT();
#pragma unroll
          for (int r = 0; r <= K; ++r) {
            // y interpolation of the row (energy and charge as one packed pair)
            const NodeT B = lerpc(uc, n0[r], n1[r]);
            if (r > 0) {
              const int q = r - 1;
              // x interpolation
              const NodeT L = lerpc(e.t + ex[q], Bp, B);
              v[q] = comb_e(L);
              vb[q] = comb_b(L);
            }
            Bp = B;
          }
          const FSM_FLOAT2 cs = ev.cs[p];
          if (!inside) {
            const bool nearx = (e.oy_near >> 16) & 1, neary = (e.oy_near >> 17) & 1;
            const bool in_y = (unsigned)(j - 1) <= (unsigned)(NY - 3);
            if (!(nearx || neary)) {  // uniform: no decision depends on the rounding
#pragma unroll
              for (int k = 0; k < K; ++k) {
                const bool in = in_y && ((unsigned)(i0 + k - 1) <= (unsigned)(NX - 3));
                v[k] = in ? v[k] : 0.0f;
                vb[k] = in ? vb[k] : 0.0f;
              }
            } else {
#pragma unroll
              for (int k = 0; k < K; ++k) {
                const int ik = i0 + k;
                const bool ux = nearx && (ik == 0 || ik == 1 || ik == NX - 2 || ik == NX - 1);
                const bool uy = neary && (j == 0 || j == 1 || j == NY - 2 || j == NY - 1);
                bool in = in_y && ((unsigned)(ik - 1) <= (unsigned)(NX - 3));
                if (act[k] && (ux || uy)) {
                  // the in-grid decision depends on the rounding: reference arithmetic
                  const float x = __fadd_rn(__fmul_rn((float)(ixb + k), ev.DX), ev.xmin);
                  in = exact_sample3d_pair<kB>(ev, rp, irap, x, y, cs.x, cs.y, v[k], vb[k]);
                }
                if (!in) {
                  v[k] = 0.0f;
                  vb[k] = 0.0f;
                }
              }
            }
          }
          const float csn = cs.x * cs.y, ss = cs.y * cs.y;
          const float2 ccs = make_float2(cs.x * cs.x, csn);
          const float2 c2 = make_float2(cs.x, cs.x), s2 = make_float2(cs.y, cs.y);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const float2 w = make_float2(v[k], vb[k]);
            a01[k] = __fadd2_rn(a01[k], w);
            a1c[k] = __ffma2_rn(w, c2, a1c[k]);
            a1s[k] = __ffma2_rn(w, s2, a1s[k]);
            a34[k] = __ffma2_rn(make_float2(v[k], v[k]), ccs, a34[k]);
            a5[k] = fmaf(v[k], ss, a5[k]);
          }
        }
      }
      {
        // second level of the two-level sum: the partial sums times the rows
        // of the hypertrig table (src/LandauMatch.cpp:46-55), the rapidity
        // Jacobian and the profile norm (:101), into T^{mu nu} (and J^mu with
        // the charge norm, :120-139)
        // (a chunk none of whose phi_p reached this warp left its partial
        // sums at zero: nothing to fold)
        if (!cm) continue;
        const RapEta r = *rp;
        const float cA = jw * r.A, cB = jw * r.B, cC = jw * r.C, cD = jw * r.Dt, cE = jw * r.E;
        // packed slot pairs: (T0, T3), (T1, T2), (T4, T5), (T6, T8), (T7, T9)
        // [, (J0, J3), (J1, J2)], each component a fused multiply-add
#pragma unroll
        for (int k = 0; k < K; ++k) {
          float2* q = sl + k * (kS / 2) * kThreads3D;
          auto acc = [&](int j, float2 a, float2 c) { q[j * kThreads3D] = __ffma2_rn(a, c, q[j * kThreads3D]); };
          acc(0, make_float2(a01[k].x, a01[k].x), make_float2(jw, cD));
          acc(1, make_float2(a1c[k].x, a1s[k].x), make_float2(cA, cA));
          acc(2, a34[k], make_float2(cB, cB));
          acc(3, make_float2(a1c[k].x, a1s[k].x), make_float2(cC, cC));
          acc(4, make_float2(a5[k], a01[k].x), make_float2(cB, cE));
          if (kB) {
            const float nb = ev.normB, bA = nb * r.A, bD = nb * r.Dt;
            acc(5, make_float2(a01[k].y, a01[k].y), make_float2(nb, bD));
            acc(6, make_float2(a1c[k].y, a1s[k].y), make_float2(bA, bA));
          }
          a01[k] = a1c[k] = a1s[k] = make_float2(0.f, 0.f);
          a34[k] = make_float2(0.f, 0.f);
          a5[k] = 0.0f;
        }
      }
    }
  }
}

// The tile loop of the 3D kernels; kB: the tiles' events carry baryon charge
// (one kind per launch, so that each kernel is register-allocated for its own
// path: compiled together, the two paths spilled).
template <bool kB>
__device__ __forceinline__ void stream3d_tiles(const Ev3D* __restrict__ evs,
                                               const Tile3D* __restrict__ tiles, int ntiles,
                                               int* counter) {
  extern __shared__ float slots3[];  // thread-private slots, [slot][thread]
  __shared__ int s_tile;
  constexpr int K = kCellsPerThread;
  constexpr int kS = slots3d<kB>();
  static_assert(kThreads3D * kParts3D == kWarps2D * 32 && kWarps2D == 8, "the tile shapes are laid out for 8 warps");
  const int lane = threadIdx.x & 31;
  static_assert(kSlots3D % 2 == 0 && kSlots3DBaryon % 2 == 0, "slots in pairs");
  float2* const sl = reinterpret_cast<float2*>(slots3) + threadIdx.x;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1);
    __syncthreads();
    const int unit = s_tile;  // part unit % kParts3D of tile unit / kParts3D
    if (unit >= ntiles * kParts3D) return;
    const Tile3D tl = tiles[unit / kParts3D];
    // this warp's place in the 8-warp layout of the tile
    const int warp = (unit % kParts3D) * (kThreads3D / 32) + (threadIdx.x >> 5);
    const Ev3D& ev = evs[tl.ev];
    const int NX = ev.NX, NY = ev.NY, NE = ev.NE, NR = ev.NR, NP = ev.NPHI;
    const int ieta = tl.ieta;
    constexpr bool baryon = kB;
    // the tile's shape (as in 2D): lanes along y in groups of ly cells, wy
    // warps stacked along y
    const int sh = tl.shape;
    const int lyl = shape_ly_log(sh), wyl = shape_wy_log(sh);
    const int ly = 32 >> lyl, gx = 1 << lyl, wxcount = kWarps2D >> wyl;
    const int wxi = warp & (wxcount - 1), wyi = warp >> (3 - wyl);
    const int iy = tl.y0 + wyi * ly + (lane & (ly - 1));
    const int ixb = tl.x0 + K * (wxi * gx + (lane >> (5 - lyl)));
    // the last cell the tile stores (x1, y1 <= the grid's size)
    const int x_hi = min(tl.x0 + K * gx * wxcount, tl.x1) - 1, y_hi = min(tl.y0 + (ly << wyl), tl.y1) - 1;
    // this warp's cells: all of them, and those the tile stores
    const int wxa = tl.x0 + K * wxi * gx, wxn = K * gx, wxb = min(wxa + wxn - 1, x_hi);
    const int wya = tl.y0 + wyi * ly, wyb = min(wya + ly - 1, y_hi);
    const float DX = ev.DX, DY = ev.DY, xmin = ev.xmin, ymin = ev.ymin;
    const float y = __fadd_rn(__fmul_rn((float)iy, DY), ymin);  // src/FreeStream.cpp:164
    // the cells' rounding offsets in cells (a first-order correction, so one
    // reciprocal per tile instead of a division per cell)
    const double rdx = 1.0 / (double)DX, rdy = 1.0 / (double)DY;
    const float ey = (float)(((double)y - ((double)ymin + (double)iy * (double)DY)) * rdy);
    float ex[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int ix = ixb + k;
      const float x = __fadd_rn(__fmul_rn((float)ix, DX), xmin);
      ex[k] = (float)(((double)x - ((double)xmin + (double)ix * (double)DX)) * rdx);
      act[k] = (ix <= x_hi) && (iy <= y_hi);
    }
#pragma unroll
    for (int m = 0; m < K * kS / 2; ++m) sl[m * kThreads3D] = make_float2(0.f, 0.f);
    const size_t plane = (size_t)NX * NY;
    for (int irap = ev.r_lo; irap < ev.r_hi; ++irap) {
      const RapEta re = ev.re[ieta * NR + irap];
      // a pair without a combined plane has no sample inside the grid
      const int pl = __ldg(ev.plane_of + ieta * NR + irap);
      if (!(re.efl >= 1 && re.efl < NE - 1) || !isfinite(re.D) || pl < 0) continue;
      const PhiEntry3D* tab = ev.tab3 + ((size_t)ieta * NR + irap) * NP;
      // rapidity Jacobian (src/LandauMatch.cpp:101) times the profile norm
      const float jw = ev.jac[irap] * ev.norm;
      const RapEta* rp = ev.re + ieta * NR + irap;
      if constexpr (kB) {
        const float2* Nc = reinterpret_cast<const float2*>(ev.nodesc) + (size_t)pl * plane;
        stream3d_rap<true>(ev, ixb, iy, wxa, wxb, wxn, wya, wyb, ly, y, ey, ex, act, Nc, tab, irap, rp, jw, sl);
      } else {
        const float* Nc = reinterpret_cast<const float*>(ev.nodesc) + (size_t)pl * plane;
        stream3d_rap<false>(ev, ixb, iy, wxa, wxb, wxn, wya, wyb, ly, y, ey, ex, act, Nc, tab, irap, rp, jw, sl);
      }
    }
    const float dphi = ev.d_phip;
    const size_t DIM = (size_t)NX * NY * NE;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!act[k]) continue;
      const size_t is = ((size_t)(ixb + k) * NY + iy) * NE + ieta;
      const float2* q = sl + k * (kS / 2) * kThreads3D;
      auto P = [&](int j) { return q[j * kThreads3D]; };
      const float2 p0 = P(0), p1 = P(1), p2 = P(2), p3 = P(3), p4 = P(4);
      const float t[10] = {p0.x, p1.x, p1.y, p0.y, p2.x, p2.y, p3.x, p4.x, p3.y, p4.y};
      for (int m = 0; m < 10; ++m) ev.T[(size_t)m * DIM + is] = t[m] * dphi;  // (LandauMatch.cpp:105)
      if (baryon) {
        const float jf = ev.DRAP * dphi;  // (LandauMatch.cpp:140)
        const float2 p5 = P(5), p6 = P(6);
        const float jv[4] = {p5.x, p6.x, p6.y, p5.y};
        for (int m = 0; m < 4; ++m) ev.J[(size_t)m * DIM + is] = jv[m] * jf;
      }
    }
    __syncthreads();
  }
}

// 3D events without baryon charge (float2 eta-pair nodes).
__global__ void __launch_bounds__(kThreads3D, 2 * kParts3D) fsm_stream3d_kernel(const Ev3D* __restrict__ evs,
                                                                     const Tile3D* __restrict__ tiles,
                                                                     int ntiles, Counters* ctr) {
  stream3d_tiles<false>(evs, tiles, ntiles, &ctr->block3d);
}

// 3D events with baryon charge (float4 eta-pair nodes of energy and charge).
__global__ void __launch_bounds__(kThreads3D, 2 * kParts3D) fsm_stream3d_baryon_kernel(
    const Ev3D* __restrict__ evs, const Tile3D* __restrict__ tiles, int ntiles, Counters* ctr) {
  stream3d_tiles<true>(evs, tiles, ntiles, &ctr->block3d_b);
}

// ------------------------------------------------------------- packing
// Gathers the output-slab segments a packed download asks for into one
// contiguous device buffer (block per segment, coalesced).
__global__ void __launch_bounds__(256) fsm_pack_kernel(const float* __restrict__ slab,
                                                       float* __restrict__ out,
                                                       const CopySeg* __restrict__ segs) {
  const CopySeg sg = segs[blockIdx.x];
  const float* a = slab + sg.src;
  float* d = out + sg.dst;
  for (int i = threadIdx.x; i < sg.len; i += blockDim.x) d[i] = __ldg(a + i);
}

// ----------------------------------------------------------------- Landau
// Eight 128-thread blocks per SM (64 registers, some spilled to L1): the
// solver is latency-bound, and the extra warps gain more than the spills cost
// (measured against 4 to 7 blocks, and 64- and 256-thread blocks).
// Boost-invariant and 3D events run in separate instantiations (the union of
// the 3x3 and 4x4 eigenproblems spilled 492 bytes per thread, the 3x3 path
// alone 156).
template <bool k3D>
__device__ __forceinline__ void landau_block(const EvLandau* __restrict__ evs,
                                             const CellBlock* __restrict__ blocks, Counters* ctr) {
  const CellBlock b = blocks[blockIdx.x];
  const EvLandau& ev = evs[b.ev];
  const int DIM = ev.DIM;
  const int is = b.begin + threadIdx.x;
  int fb = 0;
  if (is < DIM) {
    float T[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, J[4] = {0, 0, 0, 0};
    if constexpr (k3D) {
#pragma unroll
      for (int m = 0; m < 10; ++m) T[m] = __ldg(ev.T + (size_t)m * DIM + is);
    } else {  // boost-invariant: the stream kernel wrote T^{tau eta} = T^{x eta} = T^{y eta} = T^{eta eta} = 0
      constexpr int nz[6] = {0, 1, 2, 4, 5, 7};
#pragma unroll
      for (int m = 0; m < 6; ++m) T[nz[m]] = __ldg(ev.T + (size_t)nz[m] * DIM + is);
    }
    if (ev.baryon && ev.J) {
#pragma unroll
      for (int m = 0; m < 4; ++m) J[m] = __ldg(ev.J + (size_t)m * DIM + is);
    }
    CellOut o;
    landau_cell_t<k3D>(T, J, ev.baryon, ev.eos, ev.viscous, ev.TAU, &o);
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

// Boost-invariant events (3x3 eigenproblem).
__global__ void __launch_bounds__(kThreadsLandau, 8) fsm_landau_kernel(const EvLandau* __restrict__ evs,
                                                                    const CellBlock* __restrict__ blocks,
                                                                    Counters* ctr) {
  landau_block<false>(evs, blocks, ctr);
}

// 3D events (4x4 eigenproblem).
__global__ void __launch_bounds__(kThreadsLandau, 8) fsm_landau3d_kernel(const EvLandau* __restrict__ evs,
                                                                      const CellBlock* __restrict__ blocks,
                                                                      Counters* ctr) {
  landau_block<true>(evs, blocks, ctr);
}

// ------------------------------------------------------------- diagnostics
// Hydro-validity and thermal-vorticity fields of the Landau-matched outputs
// (src/HydroValidity.cpp:8-101, src/LandauMatch.cpp:395-489), thread per
// cell, with the reference's float/double mixing spelled out (no
// contraction).  beta and omega follow the reference's own indexing: the
// interior (ix, iy) pairs at index DIM_Y * ix + iy.
__global__ void __launch_bounds__(256) fsm_diag_kernel(int NX, int NY, int NE, float DX, float DY,
                                                       float tau, const float* __restrict__ e,
                                                       const float* __restrict__ P,
                                                       const float* __restrict__ Pi,
                                                       const float* __restrict__ u,
                                                       const float* __restrict__ pi, float* rpi,
                                                       float* rsh, float* pdu, float* pmm,
                                                       float* beta, float* om) {
  const size_t n = (size_t)NX * NY * NE;
  const size_t is = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (is >= n) return;
  auto S = [&](int m) { return __ldg(pi + m * n + is); };
  const float tau2 = __fmul_rn(tau, tau);
  {
    const float p = __ldg(P + is);
    const float pp = ((double)p < 1.0e-5) ? (float)1.0e-5 : p;
    if (rpi) rpi[is] = __fdiv_rn(__ldg(Pi + is), pp);
  }
  if (rsh) {
    const float s0 = S(0), s1 = S(1), s2 = S(2), s3 = S(3), s4 = S(4), s5 = S(5), s6 = S(6),
                s7 = S(7), s8 = S(8), s9 = S(9);
    const float b = __fadd_rn(__fadd_rn(__fmul_rn(s1, s1), __fmul_rn(s2, s2)),
                              __fmul_rn(__fmul_rn(tau2, s3), s3));
    const float c = __fadd_rn(__fadd_rn(__fmul_rn(s4, s4), __fmul_rn(s7, s7)),
                              __fmul_rn(__fmul_rn(__fmul_rn(tau2, tau2), s9), s9));
    const float d = __fadd_rn(__fadd_rn(__fmul_rn(s5, s5), __fmul_rn(__fmul_rn(tau2, s6), s6)),
                              __fmul_rn(__fmul_rn(tau2, s8), s8));
    double acc = __dsub_rn((double)__fmul_rn(s0, s0), __dmul_rn(2.0, (double)b));
    acc = __dadd_rn(acc, (double)c);
    acc = __dadd_rn(acc, __dmul_rn(2.0, (double)d));
    const float num = (float)acc;
    const float ev = __ldg(e + is), pv = __ldg(P + is);
    float den;
    if ((double)ev < 1.0e-5) den = (float)1.0e-5;
    else den = (float)__dadd_rn((double)__fmul_rn(ev, ev), __dmul_rn(__dmul_rn(3.0, (double)pv), (double)pv));
    rsh[is] = __fdiv_rn(__fsqrt_rn(fabsf(num)), __fsqrt_rn(fabsf(den)));
  }
  if (pdu || pmm) {
    const float ut = __ldg(u + is), ux = -__ldg(u + n + is), uy = -__ldg(u + 2 * n + is);
    const float un = __fmul_rn(__fmul_rn(-tau, tau), __ldg(u + 3 * n + is));
    auto dot = [&](float a, float b2, float c2, float d2) {
      return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a, ut), __fmul_rn(b2, ux)), __fmul_rn(c2, uy)),
                       __fmul_rn(d2, un));
    };
    if (pdu) {
      pdu[is] = dot(S(0), S(1), S(2), S(3));
      pdu[n + is] = dot(S(1), S(4), S(5), S(6));
      pdu[2 * n + is] = dot(S(2), S(5), S(7), S(8));
      pdu[3 * n + is] = dot(S(3), S(6), S(8), S(9));
    }
    if (pmm) {
      const float pxx = -S(4), pyy = -S(7), pnn = __fmul_rn(__fmul_rn(-tau, tau), S(9));
      pmm[is] = __fadd_rn(__fadd_rn(__fadd_rn(S(0), pxx), pyy), pnn);
    }
  }
  if (beta || om) {
    float b[4] = {0.f, 0.f, 0.f, 0.f}, w_xy = 0.f;
    if (is < (size_t)NX * NY) {
      const int ix = (int)(is / NY), iy = (int)(is % NY);
      if (ix >= 1 && ix < NX - 1 && iy >= 1 && iy < NY - 1) {
        auto T = [&](size_t k) { return powf(__fdiv_rn(__ldg(e + k), 13.8997f), 0.25f); };
        const size_t px = (size_t)NY * (ix + 1) + iy, mx = (size_t)NY * (ix - 1) + iy,
                     py = (size_t)NY * ix + (iy + 1), my = (size_t)NY * ix + (iy - 1);
        const float Tc = T(is);
        b[0] = __fdiv_rn(__ldg(u + is), Tc);
        b[1] = __fdiv_rn(-__ldg(u + n + is), Tc);
        b[2] = __fdiv_rn(-__ldg(u + 2 * n + is), Tc);
        b[3] = __fdiv_rn(0.0f, Tc);
        const float bx_py = __fdiv_rn(-__ldg(u + n + py), T(py));
        const float bx_my = __fdiv_rn(-__ldg(u + n + my), T(my));
        const float by_px = __fdiv_rn(-__ldg(u + 2 * n + px), T(px));
        const float by_mx = __fdiv_rn(-__ldg(u + 2 * n + mx), T(mx));
        const double gy = __ddiv_rn(__ddiv_rn((double)__fsub_rn(bx_py, bx_my), 2.0), (double)DY);
        const double gx = __ddiv_rn(__ddiv_rn((double)__fsub_rn(by_px, by_mx), 2.0), (double)DX);
        w_xy = (float)__dmul_rn(0.5, __dsub_rn(gy, gx));
      }
    }
    if (beta)
      for (int m = 0; m < 4; ++m) beta[m * n + is] = b[m];
    if (om)
      for (int m = 0; m < 6; ++m) om[m * n + is] = (m == 3) ? w_xy : 0.0f;
  }
}

}  // namespace fsm
