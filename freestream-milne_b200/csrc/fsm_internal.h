// fsm_internal.h -- descriptors shared by the host planner and the sm_100a kernels.
//
// Layout in HBM (per event; fields in the reference cell order
// is = (DIM_Y*DIM_ETA)*ix + DIM_ETA*iy + ieta):
//   2D: nodes[is]  float4 (F, F_x*DX, F_y*DY, F_xy*DX*DY): the bicubic node data
//       of F = e/(2 pi), 16 B/cell, read by the stream kernel through staged
//       shared-memory windows of each output tile.
//   3D: nodes3[e][ix][iy] eta-pair nodes (e in fm^-4 of slices e and e+1, and
//       n_B of both with BARYON), float2 / float4, read by the exact boundary
//       samples; nodesc[plane][ix][iy] combined planes (one per sampled eta
//       slice x rapidity pair: both source slices eta-interpolated with the
//       pair's rapidity weights), float / float2 (e, n_B), read through L1.
//   T[10][DIM], J[4][DIM]: moments written by the stream kernels, read by the
//   Landau kernel.  Outputs e,P,Pi,u[4],pi[10],nB,V[4] are [comp][DIM] floats.
#pragma once
#include <stdint.h>
#include <stddef.h>

#ifndef __CUDACC__
struct float2_h { float x, y; };
struct float4_h { float x, y, z, w; };
#define FSM_FLOAT2 float2_h
#define FSM_FLOAT4 float4_h
#else
#define FSM_FLOAT2 float2
#define FSM_FLOAT4 float4
#endif

namespace fsm {

constexpr int kCellsPerThread = 4;  // 2D: consecutive x cells owned by one thread
constexpr int kTileY = 32;           // 2D output tile: y extent (fast index) = warp lanes
constexpr int kWarps2D = 8;
constexpr int kTileX = kWarps2D * kCellsPerThread;  // 2D output tile: x extent (slow index)
constexpr int kThreads2D = kWarps2D * 32;
constexpr int kPhiTab2D = 6;         // float4 per phi_p entry of the 2D table
constexpr int kMaxRunPhi2D = 64;     // phi_p per staged run (the run's table slice is staged with it)
// 3D stream CTAs of 4 warps, each taking one part (warps 0-3 or 4-7 of the
// 8-warp tile layout) of an output tile: the CTA's end-of-tile barrier then
// waits for 4 warps of unequal work instead of 8
constexpr int kThreads3D = 128;
constexpr int kParts3D = kWarps2D * 32 / kThreads3D;  // work units per 3D tile
constexpr int kThreadsLandau = 128;
// Polls of one bounded mbarrier wait of a staged copy (a context may lower it
// to exercise the time-out path; the drain after a time-out always uses this).
constexpr int kWaitPolls = 1 << 20;
constexpr int kPhiChunk = 16;  // FP32 partial sums over 16 phi_p are added into FP32 totals (two-level sum)

// Natural-spline axis data for the 2D prep kernels (host computed, double),
// one entry per interval / unknown k of an axis with n nodes, on the float grid
// coordinates x_i: h = x[k+1] - x[k] and g = 6/h (k <= n-2); the elimination
// factor f and the inverse modified diagonal 1/dg of the tridiagonal system for
// the second derivative at node k+1 (k <= n-3).  Tables are stored with
// kPadLo zero entries before k = 0 and kPadHi after the line, and all fields
// outside the ranges above are 0.
struct AxisNode {
  double g, f, h, idg;
};

// Windowed natural-spline elimination of the prep kernels: a thread produces
// the slopes of kSegP consecutive nodes from a forward/backward sweep over the
// segment plus kWinP nodes on each side, started from zero.  The sweeps'
// factors are the exact full-line ones and the influence of the truncated
// start decays like (2 - sqrt 3)^kWinP < 1e-9.
constexpr int kSegP = 8;
constexpr int kWinP = 16;
constexpr int kPadLo = kWinP + 4;           // table/line padding before node 0
constexpr int kPadHi = kWinP + kSegP + 4;   // and after node n-1
constexpr int kPrepRows = 4;  // y-lines (rows) per block of the long-row kernel, one warp each
constexpr int kMaxNY2D = 5120;  // longest 2D row the long-row kernel stages in shared memory
constexpr int kMaxStrip = 720;  // longest line of the 32-line strip kernels
constexpr int kPrepThreads = 256;  // strip kernels

// Dynamic shared memory of the strip kernels for lines of up to n nodes: the
// padded axis table and two padded fields of 32 lines (odd line stride).
inline int strip_ld(int n) { return (n + kPadLo + kPadHi) | 1; }
inline size_t prep_strip_smem(int n) {
  return (size_t)(n + kPadLo + kPadHi) * sizeof(AxisNode) + (size_t)2 * 32 * strip_ld(n) * 4;
}

// Dynamic shared memory of the long-row kernel: two padded rows of up to
// ny_cap floats per warp.
inline size_t prep_rows_smem(int ny_cap) {
  return (size_t)kPrepRows * 2 * (size_t)(ny_cap + kPadLo + kPadHi + 2) * 4;
}

// Per-phi_p entry of the 2D stream table (6 float4, host computed).  With the
// reference's float shift s = fl(cos(phi_p) * DTAU), the source point of cell ix
// is ix + sx, sx = -s/DX, split into the integer offset ox = floor(sx) and the
// fraction t = sx - ox (likewise y).  Stored, laid out for packed-pair FMAs: the
// cubic Hermite weights of t and u and their derivatives (for the first-order
// correction of each cell's own float-rounded coordinate), the moment weights,
// the offsets and a flag telling whether t or u lies within 1e-3 of an integer
// (then a sample on the grid boundary is re-evaluated with the reference's
// exact float arithmetic).
struct PhiEntry2D {
  float H0, G0, H1, G1;      // Hermite weights of t (value/slope pairs of nodes 0 and 1)
  float dH0, dG0, dH1, dG1;  // their derivatives in t
  float K0, K1, L0, L1;      // Hermite weights of u
  float dK0, dK1, dL0, dL1;
  float c, s, cc, cs;        // cos, sin (reference floats), cos^2, cos sin
  float t, u;
  int ox;
  int oy_near;               // low 16 bits: oy (signed); bit 16: near in x; bit 17: near in y;
                             // bit 18: (ox, oy) differs from the previous phi_p's (or phi_p 0)
};
constexpr int kReloadBit2D = 1 << 18;

// A run of consecutive phi_p nodes whose source offsets fit one staged window:
// for a tile at (x0, y0) the window starts at row x0 + ox0 - 1, column
// y0 + oy0 - 1 (a one-node margin on each side for samples decided with the
// reference arithmetic).  [ox0, ox1] x [oy0, oy1] is the run's offset range;
// its window is win_h(c) rows of win_w(c) nodes.
struct Chunk2D {
  int p0, p1, ox0, oy0, ox1, oy1;
};
#if defined(__CUDACC__)
#define FSM_HDI __host__ __device__ inline
#else
#define FSM_HDI inline
#endif
// 2D output tile shapes.  A warp's lanes run along y in groups of Ly
// consecutive cells (32 / Ly groups of 4 x cells side by side), and Wy warps
// are stacked along y: TX = 4 * (32 / Ly) * (8 / Wy) x cells by TY = Ly * Wy
// y cells, always 256 threads and 1024 cells.  Shape 0 (32 x 32) tiles an
// event; the narrow shapes cover its partial last strips, so that fewer lanes
// and warps run past the grid edge: 1 (64 x 16), 2 (128 x 8) and 6 (256 x 4)
// for a last y strip of at most 16 / 8 / 4 cells, 3 (16 x 64), 4 (8 x 128)
// and 5 (4 x 256) for a last x strip of at most 16 / 8 / 4 cells.
constexpr int kShapes2D = 7;
// log2(32 / Ly) and log2(Wy) of shapes 0..6, 3 bits per shape
constexpr int kShapeLyLog = (1 << 3) | (2 << 6) | (3 << 18);
constexpr int kShapeWyLog = (1 << 9) | (2 << 12) | (3 << 15);
FSM_HDI int shape_ly_log(int s) { return (kShapeLyLog >> (3 * s)) & 7; }
FSM_HDI int shape_wy_log(int s) { return (kShapeWyLog >> (3 * s)) & 7; }
FSM_HDI int shape_ly(int s) { return 32 >> shape_ly_log(s); }
FSM_HDI int shape_wy(int s) { return 1 << shape_wy_log(s); }
FSM_HDI int shape_tx(int s) { return kCellsPerThread * (32 / shape_ly(s)) * (kWarps2D / shape_wy(s)); }
FSM_HDI int shape_ty(int s) { return shape_ly(s) * shape_wy(s); }
// Staged window of a run for a tile of shape s: rows (x) and row length (y).
FSM_HDI int win_h(const Chunk2D& c, int s) { return shape_tx(s) + (c.ox1 - c.ox0) + 3; }
FSM_HDI int win_w(const Chunk2D& c, int s) { return shape_ty(s) + (c.oy1 - c.oy0) + 3; }
constexpr int kMaxChunks2D = 64;
constexpr int kWindowBudget2D = 32 * 1024;  // bytes of one staged window (default)
constexpr int kMaxWindow2D = 64 * 1024;     // largest staged window the planner raises to
constexpr int kTotSlots2D = 5 * 4;          // per-thread moment totals kept in shared memory
// Dynamic shared memory of the 2D stream kernel with staged windows of up to
// box_cap nodes: two run tables, two windows, the moment totals.
inline size_t stream2d_smem(int box_cap) {
  return ((size_t)2 * kMaxRunPhi2D * kPhiTab2D + 2 * (size_t)box_cap) * 16 +
         (size_t)kTotSlots2D * kThreads2D * 4;
}

struct Ev2D {
  int NX, NY, NPHI, NR;
  float DX, DY, DTAU, TAU;
  float xmin, ymin, xmax_i, ymax_i;  // grid origin and spline domain (src/FreeStream.cpp:113,142-146)
  float d_phip;
  const PhiEntry2D* tab; // [NPHI]
  const Chunk2D* chunks; // the runs of every tile shape the event uses
  int choff[kShapes2D];  // first run of shape s in chunks
  int nch[kShapes2D];    // runs of shape s (0: shape unused)
  int chunk;             // phi_p per FP32 partial sum of the two-level moment sum (16 or 32)
  int raw;               // e_gev already holds fm^-4 (no GeV/fm^3 conversion)
  // prep
  const float* e_gev;    // input
  const AxisNode* ax;   // [NX] x-axis spline data
  const AxisNode* ay;   // [NY] y-axis spline data
  float* fa;             // scratch [DIM]: F = e/(2 pi)
  float* sy;             // scratch [DIM]: y-slopes dF/dy * DY
  FSM_FLOAT4* nodes;     // [DIM]
  // outputs of the stream kernel
  float* T;              // [10][DIM]
  // charge pass of a boost-invariant event with BARYON = 1: the field is
  // B = n_B * qnorm, the bilinear fallback is scaled by fb_scale, and the
  // moments go to J = (S, S cos, S sin, 0) * jscale * DRAP * d_phip
  int charge;
  float qnorm, fb_scale, jscale, DRAP;
  float* J;              // [4][DIM]
};

// Per-(ieta, irap) quantities of the 3D path, computed on the host with the
// reference's float arithmetic (src/FreeStream.cpp:174-201, LandauMatch.cpp:36-55).
// Thread-private shared-memory slots per cell of the 3D stream kernels:
// T^{mu nu} (10), with baryon charge also J^mu (4).
constexpr int kSlots3D = 10;
constexpr int kSlots3DBaryon = 14;

struct RapEta {
  float D;      // TAU*cosh(rap-eta_new) - TAU0*cosh(rap-eta): transverse shift length
  float efrac;  // fractional part of the shifted eta index
  int efl;      // floor of the shifted eta index (sample valid iff 1 <= efl < NE-1)
  float A;      // 1/cosh(d),  d = rap - eta                (rows 1,2)
  float B;      // 1/cosh(d)^2                             (rows 4,5,7)
  float C;      // tanh(d)/(TAU cosh d)                     (rows 6,8)
  float Dt;     // tanh(d)/TAU                              (row 3)
  float E;      // tanh(d)^2/TAU^2                          (row 9)
};

// Per-(ieta, irap, phi_p) entry of the 3D stream table (host computed): with
// the reference's float shift s = fl(cos(phi_p) * D), the source point of cell
// ix is ix + sx, sx = -s/DX, split into the integer offset ox = floor(sx) and
// the fraction t (likewise y), and flags telling whether t or u lies within
// 1e-3 of an integer.
struct PhiEntry3D {
  float t, u;
  int ox;
  int oy_near;  // low 16 bits: oy (signed); bit 16: near in x; bit 17: near in y
};

// Weights of one combined node plane of a 3D event: the plane of pair (ieta,
// irap) holds, per transverse node, the eta interpolation of the pair's two
// source slices efl, efl+1 with the rapidity weights of that pair,
// w0 E[efl] + w1 E[efl+1] (and b0 B[efl] + b1 B[efl+1]), w0 = (1 - efrac)
// rf(efl), w1 = efrac rf(efl+1) (src/FreeStream.cpp:264-266 with the
// rapidity factors of :345, 381-382).  Grouped by efl, so that the prep
// kernel's thread of source node (efl, ix, iy) writes every plane that reads it.
struct CombW {
  int plane;
  float w0, w1, b0, b1;
};

// A 3D output tile: 32 x 32 cells of one eta slice of one event.
// A 3D output tile of eta slice ieta: shape `shape` (as the 2D shapes) from
// (x0, y0), storing the cells below (x1, y1).
struct Tile3D {
  int ev, x0, y0, ieta, shape, x1, y1;
};

struct Ev3D {
  int NX, NY, NE, NR, NPHI;
  int r_lo, r_hi;  // live rapidity nodes [r_lo, r_hi)
  int baryon;
  int raw;         // e_gev already holds fm^-4 (no GeV/fm^3 conversion)
  float DX, DY;
  float xmin, ymin;
  float norm, normB, d_phip, DRAP;
  const FSM_FLOAT2* cs;   // [NPHI]
  const RapEta* re;       // [NE*NR]
  const float* rapf;      // [NE*NR] energy rapidity weight  cosh^2 d exp(-d^2/2 sigma^2)
  const float* rapfB;     // [NE*NR] baryon weight on the uniform rapidity grid
  const float* jac;       // [NR] tan-map Jacobian (src/LandauMatch.cpp:92-93)
  const PhiEntry3D* tab3; // [NE*NR*NPHI]
  const float* e_gev;     // input
  const float* nB;        // input baryon density
  // eta-pair nodes [NE-1][NX][NY]: (E[e], E[e+1], B[e], B[e+1]) float4 with
  // BARYON, (E[e], E[e+1]) float2 without; E in fm^-4
  void* nodes3;
  // combined node planes [nplanes][NX][NY]: (E, B) float2 with BARYON, E
  // float without; plane_of[ieta * NR + irap] is the pair's plane (-1: the
  // pair is never sampled); cw[cw_start[e] .. cw_start[e+1]) the planes that
  // read source eta pair e
  void* nodesc;
  const int* plane_of;    // [NE*NR]
  const int* cw_start;    // [NE]
  const CombW* cw;        // [nplanes]
  float* T;               // [10][DIM]
  float* J;               // [4][DIM]
  long long cell_begin;   // first global cell index of this event in the 3D work list
};

struct EvLandau {
  int DIM;
  int is3d;
  int baryon;
  int eos;
  int viscous;
  float TAU;
  const float* T;
  const float* J;
  float *e, *P, *Pi, *u, *pi, *nB, *V;
  long long cell_begin;   // first global cell index of this event in the Landau work list
};

// Work-list entries: a block of spline lines / cells of one event.  For the
// row kernel `begin` is the first x row; for the column kernel `begin` is the
// first y column and `seg` the first x segment (kSegP nodes) of the block.
struct LineBlock {
  int ev, begin, seg;
};
struct CellBlock {
  int ev, begin;
};
// One contiguous run of a packed download: len floats from src (output-slab
// element offset) to dst (packed element offset).
struct CopySeg {
  long long src, dst;
  int len, pad;
};
constexpr int kMaxCopySeg = 1 << 16;  // floats per segment (one block each)

// One 2D output tile of one event; interior = 1 when every sample of every
// cell of the tile provably lands inside the grid (no bounds logic needed).
// A 2D output tile: shape `shape` from (x0, y0), storing the cells below
// (x1, y1) (the grid, or the end of the strip the tile belongs to).
struct Tile2D {
  int ev, x0, y0, shape, x1, y1;
};

// Inputs of the energy bookkeeping of one event (fsm_batch_energy).
struct EvEnergy {
  const float* e_in;  // input profile (GeV/fm^3, or fm^-4 with raw)
  const float* T00;   // T^{tau tau} after streaming
  const float* e;     // Landau-matched energy density (fm^-4)
  int n, raw;
  float e_freeze;     // GeV/fm^3
};

// Counters reset before each launch sequence.
struct Counters {
  int tile2d;
  int block3d;    // 3D tiles without baryon charge
  int fallback;
  int block3d_b;  // 3D tiles with baryon charge
};

}  // namespace fsm
