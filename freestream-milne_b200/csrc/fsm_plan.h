// fsm_plan.h -- host-side event planning: effective parameters and the small
// per-event tables the kernels read.  Implemented in fsm_plan.cpp, which is
// compiled by the host compiler with FMA contraction disabled so that every
// table entry is rounded exactly as the reference computes it.
#pragma once
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fsm.h"
#include "fsm_internal.h"

namespace fsm {

// Host threads for planning and staging copies (at most 16).
int host_threads();
// Nesting depth of parallel_for on this thread (loops run serially above 0).
int& parallel_depth();
// Runs f(i) for i in [0, n) on up to `threads` threads of a process-wide
// worker pool (the caller's thread included).  Serial for threads <= 1,
// inside another parallel_for (nested loops never multiply the thread count)
// and while another host thread has the pool.
void run_parallel(int n, int threads, const std::function<void(int)>& f);
template <class F>
void parallel_for(int n, int threads, F f) {
  run_parallel(n, threads, std::function<void(int)>(f));
}
// memcpy in 1 MiB pieces on several threads when it is large.
void parallel_copy(void* dst, const void* src, size_t bytes);

struct EventPlan {
  fsm_params p;  // effective parameters (E_DEP_FS and phi_p rule applied, DIM/TAU set)
  bool is3d = false;
  bool baryon = false;
  int DIM = 0;
  float xmin = 0, ymin = 0, etamin = 0, xmax_i = 0, ymax_i = 0, d_phip = 0;
  std::vector<FSM_FLOAT2> cs;  // (cos, sin) of phi_p
  std::vector<PhiEntry2D> tab2;  // 2D stream table
  std::vector<Chunk2D> chunks2;  // phi_p runs staged as one window each, shape by shape
  int choff[kShapes2D] = {}, nch[kShapes2D] = {};  // runs of tile shape s: chunks2[choff[s]..]
  int y_shape = -1, x_shape = -1;  // narrow tile shapes of the last y / x strip (-1: 32 x 32)
  int box_elems = 0;             // largest staged window (nodes) of one run
  int ox_min = 0, ox_max = 0, oy_min = 0, oy_max = 0;  // offset range over all phi_p
  // 2D spline axes
  std::vector<AxisNode> axx, axy;
  // 3D tables
  std::vector<RapEta> re;
  // [NE*NR*NPHI]; shared, so that copies of a cached plan do not copy it
  std::shared_ptr<std::vector<PhiEntry3D>> tab3;
  std::vector<int> live_eta;     // live rapidity nodes per eta slice
  std::vector<float> rapf, rapfB, jac;
  // combined node planes (Ev3D::nodesc): plane per sampled (ieta, irap) pair,
  // weights grouped by source eta pair
  std::vector<int> plane_of;     // [NE*NR], -1: never sampled
  std::vector<int> cw_start;     // [NE]
  std::vector<CombW> cw;         // [nplanes]
  int r_lo = 0, r_hi = 0;
  float norm = 0, normB = 0;
  // 2D with BARYON: fallback and output scales of the charge pass (Ev2D)
  float fb_scale2 = 1.0f, jscale2 = 0.0f;
  int phi_chunk = kPhiChunk;  // 2D: phi_p per FP32 partial sum (tuning; 16 or 32)
  bool input_fm4 = false;     // the profile is already in fm^-4 (no conversion)
  double samples = 0;  // cell x momentum samples the stream kernel evaluates
  double ref_samples = 0;  // DIM * DIM_RAP * DIM_PHIP, the reference's count
};

// Validates `in`, applies the energy-dependent free-streaming time (needs the
// host profile; pass NULL to reject E_DEP_FS=1) and the phi_p arc-length rule,
// and fills the tables; 2D phi_p runs are cut so that each run's staged window
// stays within window_budget bytes.  Returns FSM_OK or an error with a message
// in *why.
fsm_status plan_event(const fsm_params& in, const float* host_e_gev, EventPlan* out,
                      std::string* why, int window_budget = kWindowBudget2D, bool input_fm4 = false,
                      bool tail_tiles = true);

// Narrow tile shape for the last, partial strip of a 2D grid along y (x):
// 6, 2, 1 (5, 4, 3) when at most 4, 8, 16 cells are left over, else -1
// (32 x 32 tiles).
int y_tail_shape(int NY);
int x_tail_shape(int NX);
// The output tiles of 2D event `ev` (of plan P): 32 x 32 tiles over the grid
// minus its narrow last strips, tiles of the planned narrow shapes over those
// strips (the x strip's including the corner).  Every cell is stored by one
// tile.
// square: 32 x 32 tiles only (for launches too small to fill the GPU, where
// the narrow tiles' longer staging would lengthen the slowest tile).
void tiles_2d(const EventPlan& P, int ev, std::vector<Tile2D>& out, bool square = false);
// The same tiling of an NX x NY grid with narrow shapes ys / xs (-1: none),
// as (x0, y0, shape, x1, y1) entries; the 3D tiles of each eta slice use it.
struct TileXY {
  int x0, y0, shape, x1, y1;
};
void grid_tiles(int NX, int NY, int ys, int xs, std::vector<TileXY>& out);

// Energy-dependent free-streaming time tau_R (e_T / e_R)^alpha from the
// reference's float sums of eps^2 and eps over the converted profile
// (src/FreeStream.cpp:389-417).
float edep_dtau(const fsm_params& p, float numerator, float denominator);

// Natural-spline axis table of n float grid coordinates i*d + lo, with
// kPadLo + kPadHi zero padding entries (entry k of the line at kPadLo + k).
void build_axis(int n, float d, float lo, std::vector<AxisNode>& ax);

// Output components of one event in the slab order used by batches:
// T(10) e P Pi u(4) pi(10) [J(4) nB V(4)].
int output_components(bool baryon);

void set_last_error(const std::string& msg);

}  // namespace fsm
