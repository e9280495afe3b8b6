// fsm_runtime.cu -- contexts, batches, launches and the C ABI of libfsm.so.
//
// A batch is the unit of execution: n events (2D and/or 3D, any sizes) planned
// on the host, laid out in one device allocation (tables, scratch, descriptor
// arrays, work lists and optionally input/output slabs), and run as a fixed
// sequence of six launches on one stream:
//   memset(counters) -> prep2d_rows -> prep2d_cols -> prep3d -> stream2d
//   -> stream3d -> landau
// The sequence is captured into a CUDA graph on the first fsm_batch_launch and
// replayed afterwards.  The single-event entry points run a cached one-event
// batch, so a repeated call with the same shape allocates nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fsm.h"
#include "fsm_internal.h"
#include "fsm_plan.h"
#include "fsm_runtime.h"

namespace fsm {
__global__ void fsm_prep2d_rows_kernel(const Ev2D*, const LineBlock*);
__global__ void fsm_prep2d_cols_kernel(const Ev2D*, const LineBlock*);
__global__ void fsm_prep2d_rows_long_kernel(const Ev2D*, const LineBlock*, int);
__global__ void fsm_prep2d_cols_long_kernel(const Ev2D*, const LineBlock*);
__global__ void fsm_prep3d_kernel(const Ev3D*, const CellBlock*);
__global__ void fsm_stream2d_kernel(const Ev2D*, const Tile2D*, int, int, Counters*, int*, int);
__global__ void fsm_stream3d_kernel(const Ev3D*, const Tile3D*, int, Counters*);
__global__ void fsm_stream3d_baryon_kernel(const Ev3D*, const Tile3D*, int, Counters*);
__global__ void fsm_landau_kernel(const EvLandau*, const CellBlock*, Counters*);
__global__ void fsm_landau3d_kernel(const EvLandau*, const CellBlock*, Counters*);
__global__ void fsm_pack_kernel(const float*, float*, const CopySeg*);
__global__ void fsm_edep_sums_kernel(const float* const*, const int*, int, float*);
__global__ void fsm_energy_sums_kernel(const EvEnergy*, int, float*);
__global__ void fsm_diag_kernel(int, int, int, float, float, float, const float*, const float*,
                                const float*, const float*, const float*, float*, float*, float*,
                                float*, float*, float*);
}  // namespace fsm

using namespace fsm;

using namespace fsm::rt;

namespace fsm {
namespace rt {

struct Layout {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes);
    return o;
  }
};

bool has_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n > 0;
}

void batch_free(fsm_batch* b) {
  if (!b) return;
  batch_free(b->inner);
  if (b->d_edep) cudaFree(b->d_edep);
  if (b->h_sums) cudaFreeHost(b->h_sums);
  if (b->d_energy) cudaFree(b->d_energy);
  if (b->h_energy) cudaFreeHost(b->h_energy);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->d_segs) cudaFree(b->d_segs);
  if (b->d_pack) cudaFree(b->d_pack);
  if (!b->ext_mem && (b->d_mem || b->h_stage)) {
    // the context keeps the larger allocations for its next batch; the work
    // still using them ends first (as it would before a cudaFree)
    fsm_ctx* c = b->ctx;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    char* free_dev = b->d_mem;
    char* free_host = b->h_stage;
    {
      std::lock_guard<std::mutex> g(c->spare_mu);
      if (b->d_mem && b->dev_cap > c->spare_dev_cap) {
        free_dev = c->spare_dev;
        c->spare_dev = b->d_mem;
        c->spare_dev_cap = b->dev_cap;
      }
      if (b->h_stage && b->host_cap > c->spare_host_cap) {
        free_host = c->spare_host;
        c->spare_host = b->h_stage;
        c->spare_host_cap = b->host_cap;
      }
    }
    if (free_dev) cudaFree(free_dev);
    if (free_host) cudaFreeHost(free_host);
  }
  delete b;
}

// The dynamic shared-memory limit of a kernel is a process-wide attribute, so
// it only ever grows: a batch built later with a smaller footprint must not
// shrink the limit under a batch (or captured graph) built earlier.
fsm_status ensure_dyn_smem(const void* fn, int device, size_t bytes, int* slot) {
  static std::mutex mu;
  std::lock_guard<std::mutex> g(mu);
  (void)device;
  if ((int)bytes > *slot) {
    FSM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    *slot = (int)bytes;
  }
  return FSM_OK;
}
int g_smem2[64] = {0}, g_smem3[64] = {0}, g_smem3b[64] = {0}, g_smem_rows[64] = {0},
    g_smem_srows[64] = {0}, g_smem_scols[64] = {0};

int tuning_bucket(const fsm_params& p) {
  const int side = std::max(p.DIM_X, p.DIM_Y);
  const int sc = side < 128 ? 0 : side < 192 ? 1 : side < 256 ? 2 : 3;
  const float cells = p.DTAU / std::max(1e-30f, std::min(p.DX, p.DY));
  const int hc = cells < 8.0f ? 0 : cells < 16.0f ? 1 : cells < 24.0f ? 2 : 3;
  return sc * 4 + hc;
}

void event_tuning(const fsm_ctx* ctx, const fsm_params& p, int* window, int* chunk, bool* tail) {
  *window = ctx->window_budget;
  *chunk = kPhiChunk;
  *tail = true;
  if (p.DIM_ETA > 1) return;  // 3D events: the 3D kernel has no staged windows; chunk 16
  const fsm_tuning_bucket& t = ctx->buckets[tuning_bucket(p)];
  if (t.window_bytes > 0) *window = t.window_bytes;
  if (t.phi_chunk == 16 || t.phi_chunk == 32) *chunk = t.phi_chunk;
  if (t.tile_shapes == FSM_TILES_SQUARE) *tail = false;
}

// Builds descriptors and uploads everything.  ext_in / ext_out (one event)
// select external device buffers instead of owned slabs.
fsm_status batch_build(fsm_ctx* ctx, int n, const fsm_params* params, const float* const* host_e,
                       const float* const* ext_in_e, const float* const* ext_in_nB,
                       const fsm_outputs* ext_out, fsm_batch** out, const BatchMem* mem) {
  if (n <= 0 || !params) return FSM_ERR_INVALID_ARG;
  std::unique_ptr<fsm_batch, void (*)(fsm_batch*)> b(new fsm_batch(), batch_free);
  b->ctx = ctx;
  b->wait_polls = ctx->wait_polls;
  b->own_io = (ext_in_e == nullptr);
  b->plans.resize(n);
  {
    // events are planned independently: several host threads when the tables
    // are large (3D events: one entry per eta slice x rapidity x phi_p)
    double work = 0;
    for (int i = 0; i < n; ++i)
      work += (double)std::max(1, params[i].DIM_ETA) * std::max(1, params[i].DIM_RAP) *
              std::max(1, params[i].DIM_PHIP);
    std::vector<fsm_status> st(n, FSM_OK);
    std::vector<std::string> why(n);
    // (many small events also pay: ~35 us of host planning each)
    const bool fm4 = mem && mem->input_fm4;
    parallel_for(n, (work > 2.0e5 || n >= 16) ? host_threads() : 1, [&](int i) {
      int window = 0, chunk = 0;
      bool tail = true;
      event_tuning(ctx, params[i], &window, &chunk, &tail);
      // a 3D plan depends on nothing but the parameters and the tuning
      // (E_DEP_FS: also on the profile, so never cached)
      const bool cacheable = params[i].DIM_ETA > 1 && params[i].E_DEP_FS != 1;
      std::string key;
      if (cacheable) {
        const int extra[4] = {window, chunk, tail ? 1 : 0, fm4 ? 1 : 0};
        key.assign(reinterpret_cast<const char*>(&params[i]), sizeof(fsm_params));
        key.append(reinterpret_cast<const char*>(extra), sizeof(extra));
        std::lock_guard<std::mutex> g(ctx->plan_mu);
        auto it = ctx->plan_cache.find(key);
        if (it != ctx->plan_cache.end()) {
          b->plans[i] = *it->second;
          return;
        }
      }
      st[i] = plan_event(params[i], host_e ? host_e[i] : nullptr, &b->plans[i], &why[i], window, fm4,
                         tail);
      b->plans[i].phi_chunk = chunk;
      const size_t tab_bytes = b->plans[i].tab3 ? b->plans[i].tab3->size() * sizeof(PhiEntry3D) : 0;
      if (cacheable && st[i] == FSM_OK && tab_bytes <= kPlanCacheMaxPlan) {
        auto cached = std::make_shared<const EventPlan>(b->plans[i]);
        std::lock_guard<std::mutex> g(ctx->plan_mu);
        if (ctx->plan_cache.emplace(key, std::move(cached)).second) {
          ctx->plan_order.push_back(key);
          ctx->plan_bytes += tab_bytes;
          while (ctx->plan_order.size() > kPlanCacheEntries || ctx->plan_bytes > kPlanCacheBytes) {
            auto old = ctx->plan_cache.find(ctx->plan_order.front());
            const auto& t = old->second->tab3;
            ctx->plan_bytes -= t ? t->size() * sizeof(PhiEntry3D) : 0;
            ctx->plan_cache.erase(old);
            ctx->plan_order.erase(ctx->plan_order.begin());
          }
        }
      }
    });
    for (int i = 0; i < n; ++i)
      if (st[i] != FSM_OK) {  // the first failing event, as a serial loop would report
        set_last_error("event " + std::to_string(i) + ": " + why[i]);
        return st[i];
      }
  }
  // ---- layout
  Layout L;
  struct EvOffs {
    size_t cs, tab2, chunks, axx, axy, re, rapf, rapfB, jac, tab3, plane_of, cw_start, cw;
    size_t fa, sy, nodes, nodes3, nodesc, T, J, in_e, in_nB, out;
    size_t qfa, qsy, qnodes;  // charge pass scratch (2D with BARYON)
  };
  std::vector<EvOffs> eo(n);
  int n2 = 0, n3 = 0;
  b->ev2_of.assign(n, -1);
  b->ev3_of.assign(n, -1);
  b->evq_of.assign(n, -1);
  b->in_off.assign(n, 0);
  b->out_off.assign(n, 0);
  size_t in_elems = 0, out_elems = 0;
  for (int i = 0; i < n; ++i) {
    const EventPlan& P = b->plans[i];
    b->in_off[i] = in_elems;
    in_elems += (size_t)P.DIM * (P.baryon ? 2 : 1);
    b->out_off[i] = out_elems;
    out_elems += (size_t)P.DIM * output_components(P.baryon);
    if (P.is3d) {
      b->ev3_of[i] = n3++;
    } else {
      b->ev2_of[i] = n2++;
      if (P.baryon) b->evq_of[i] = n2++;
    }
  }
  // tables
  for (int i = 0; i < n; ++i) {
    const EventPlan& P = b->plans[i];
    EvOffs& o = eo[i];
    o.cs = L.take(P.cs.size() * sizeof(FSM_FLOAT2));
    if (!P.is3d) {
      o.tab2 = L.take(P.tab2.size() * sizeof(PhiEntry2D));
      o.chunks = L.take(P.chunks2.size() * sizeof(Chunk2D));
      o.axx = L.take(P.axx.size() * sizeof(AxisNode));
      o.axy = L.take(P.axy.size() * sizeof(AxisNode));
    } else {
      o.re = L.take(P.re.size() * sizeof(RapEta));
      o.rapf = L.take(P.rapf.size() * 4);
      o.rapfB = L.take(P.rapfB.size() * 4);
      o.jac = L.take(P.jac.size() * 4);
      o.tab3 = L.take(P.tab3->size() * sizeof(PhiEntry3D));
      o.plane_of = L.take(P.plane_of.size() * 4);
      o.cw_start = L.take(P.cw_start.size() * 4);
      o.cw = L.take(std::max<size_t>(P.cw.size(), 1) * sizeof(CombW));
    }
  }
  // work lists (host side first, to know their sizes)
  std::vector<Tile2D> tiles;
  std::vector<LineBlock> rows, cols, rows_l, cols_l;
  std::vector<CellBlock> prep3, bl;
  std::vector<Tile3D> tiles3;
  {
    std::vector<int> order2;
    for (int i = 0; i < n; ++i)
      if (!b->plans[i].is3d) order2.push_back(i);
    std::stable_sort(order2.begin(), order2.end(), [&](int a, int c) {
      return b->plans[a].p.DIM_PHIP > b->plans[c].p.DIM_PHIP;
    });
    // narrow tiles on the partial last strips pay where the launch has work
    // for every SM; a launch with fewer 32 x 32 tiles than two per SM (one
    // small event) is bound by its slowest tile, which narrow tiles (taller
    // staged windows, more runs) would lengthen
    long long sq = 0;
    for (int i : order2) {
      const EventPlan& P = b->plans[i];
      sq += (long long)((P.p.DIM_X + kTileX - 1) / kTileX) * ((P.p.DIM_Y + kTileY - 1) / kTileY) *
            (b->evq_of[i] >= 0 ? 2 : 1);
    }
    const bool square = sq < 2LL * ctx->num_sms;
    std::vector<Tile2D> tt;
    for (int i : order2) {
      tt.clear();
      tiles_2d(b->plans[i], b->ev2_of[i], tt, square);
      for (const Tile2D& t : tt) {
        tiles.push_back(t);
        // the charge pass of a 2D baryon event: the same tiles
        if (b->evq_of[i] >= 0) tiles.push_back(Tile2D{b->evq_of[i], t.x0, t.y0, t.shape, t.x1, t.y1});
      }
    }
    for (int i = 0; i < n; ++i) {
      const EventPlan& P = b->plans[i];
      if (P.is3d) continue;
      const int NX = P.p.DIM_X, NY = P.p.DIM_Y;
      for (int e2 : {b->ev2_of[i], b->evq_of[i]}) {
        if (e2 < 0) continue;
        if (NX <= kMaxStrip && NY <= kMaxStrip) {
          for (int x = 0; x < NX; x += 32) rows.push_back(LineBlock{e2, x, 0});
          for (int y = 0; y < NY; y += 32) cols.push_back(LineBlock{e2, y, 0});
          b->strip_cap2 = std::max(b->strip_cap2, std::max(NX, NY));
        } else {
          for (int x = 0; x < NX; x += kPrepRows) rows_l.push_back(LineBlock{e2, x, 0});
          const int nseg = (NX + kSegP - 1) / kSegP;
          for (int y = 0; y < NY; y += 32)
            for (int g = 0; g < nseg; g += 4) cols_l.push_back(LineBlock{e2, y, g});
          b->ny_cap2 = std::max(b->ny_cap2, NY);
        }
      }
    }
    std::vector<int> order3;
    for (int i = 0; i < n; ++i)
      if (b->plans[i].is3d) order3.push_back(i);
    std::stable_sort(order3.begin(), order3.end(), [&](int a, int c) {
      const EventPlan &A = b->plans[a], &C = b->plans[c];
      return A.samples / std::max(1, A.DIM) > C.samples / std::max(1, C.DIM);
    });
    // 3D tiles: 32 x 32 cells of one eta slice; the tiles of events with
    // baryon charge first (their own kernel), then the others, each group
    // with the slices of most live rapidity nodes first
    struct T3 {
      int work;
      bool baryon;
      Tile3D t;
    };
    std::vector<T3> t3;
    std::vector<TileXY> txy;
    for (int i : order3) {
      const EventPlan& P = b->plans[i];
      const int NX = P.p.DIM_X, NY = P.p.DIM_Y, NE = P.p.DIM_ETA;
      // the 2D tiling of a slice, narrow tiles on partial last strips (a 3D
      // event has tiles for every SM)
      txy.clear();
      grid_tiles(NX, NY, y_tail_shape(NY), x_tail_shape(NX), txy);
      for (int ie = 0; ie < NE; ++ie) {
        // slices without a live rapidity node still get tiles: they write zeros
        for (const TileXY& q : txy)
          t3.push_back({P.live_eta[ie] * P.p.DIM_PHIP, P.p.BARYON != 0,
                        Tile3D{b->ev3_of[i], q.x0, q.y0, ie, q.shape, q.x1, q.y1}});
      }
    }
    std::stable_sort(t3.begin(), t3.end(), [](const T3& a, const T3& c) {
      return a.baryon != c.baryon ? a.baryon : a.work > c.work;
    });
    for (auto& t : t3) {
      tiles3.push_back(t.t);
      b->ntiles3b += t.baryon ? 1 : 0;
    }
    for (int i = 0; i < n; ++i) {
      const EventPlan& P = b->plans[i];
      if (P.is3d)
        for (int s = 0; s < (P.p.DIM_ETA - 1) * P.p.DIM_X * P.p.DIM_Y; s += 256)
          prep3.push_back(CellBlock{b->ev3_of[i], s});
    }
    // Landau blocks: the boost-invariant events' first (their kernel), then
    // the 3D events'
    for (int pass = 0; pass < 2; ++pass)
      for (int i = 0; i < n; ++i) {
        const EventPlan& P = b->plans[i];
        if ((int)P.is3d != pass) continue;
        for (int s = 0; s < P.DIM; s += kThreadsLandau) bl.push_back(CellBlock{i, s});
        if (!P.is3d) b->nbl2 = (int)bl.size();
      }
  }
  // descriptors + work lists
  size_t o_ev2 = L.take(std::max(n2, 1) * sizeof(Ev2D));
  size_t o_ev3 = L.take(std::max(n3, 1) * sizeof(Ev3D));
  size_t o_evl = L.take(n * sizeof(EvLandau));
  size_t o_tiles = L.take(std::max<size_t>(tiles.size(), 1) * sizeof(Tile2D));
  size_t o_rows = L.take(std::max<size_t>(rows.size(), 1) * sizeof(LineBlock));
  size_t o_cols = L.take(std::max<size_t>(cols.size(), 1) * sizeof(LineBlock));
  size_t o_rows_l = L.take(std::max<size_t>(rows_l.size(), 1) * sizeof(LineBlock));
  size_t o_cols_l = L.take(std::max<size_t>(cols_l.size(), 1) * sizeof(LineBlock));
  size_t o_prep3 = L.take(std::max<size_t>(prep3.size(), 1) * sizeof(CellBlock));
  size_t o_tiles3 = L.take(std::max<size_t>(tiles3.size(), 1) * sizeof(Tile3D));
  size_t o_bl = L.take(bl.size() * sizeof(CellBlock));
  size_t o_ctr = L.take(sizeof(Counters));
  size_t o_err = L.take(sizeof(int) * 4);
  const size_t upload_bytes = L.off;  // everything above comes from the host
  // scratch and moments (none for a batch that only holds slabs)
  const bool io_only = mem && mem->io_only;
  for (int i = 0; i < n && !io_only; ++i) {
    const EventPlan& P = b->plans[i];
    EvOffs& o = eo[i];
    if (!P.is3d) {
      o.fa = L.take((size_t)P.DIM * 4);
      o.sy = L.take((size_t)P.DIM * 4);
      if (P.baryon) {
        o.qfa = L.take((size_t)P.DIM * 4);
        o.qsy = L.take((size_t)P.DIM * 4);
        o.qnodes = L.take((size_t)P.DIM * 16);
      }
      o.nodes = L.take((size_t)P.DIM * 16);
    } else {
      o.nodes3 = L.take((size_t)(P.p.DIM_ETA - 1) * P.p.DIM_X * P.p.DIM_Y * (P.baryon ? 16 : 8));
      o.nodesc = L.take(std::max<size_t>(P.cw.size(), 1) * P.p.DIM_X * P.p.DIM_Y * (P.baryon ? 8 : 4));
    }
    if (!b->own_io) {
      o.T = L.take((size_t)P.DIM * 10 * 4);
      o.J = P.baryon ? L.take((size_t)P.DIM * 4 * 4) : 0;
    }
  }
  if (b->own_io) {
    b->in_slab_off = L.take(in_elems * 4);
    b->in_slab_bytes = in_elems * 4;
    b->out_slab_off = L.take(out_elems * 4);
    b->out_slab_bytes = out_elems * 4;
  }
  b->bytes = L.off;
  b->stage_bytes = upload_bytes;
  if (mem && mem->dev) {
    b->ext_mem = true;
    b->d_mem = mem->dev(mem->user, b->bytes);
    b->h_stage = b->d_mem ? mem->host(mem->user, b->stage_bytes) : nullptr;
    if (!b->d_mem || !b->h_stage) {
      set_last_error("batch memory pool exhausted");
      return FSM_ERR_OUT_OF_MEMORY;
    }
  } else {
    {  // the allocations of a destroyed batch, when they are large enough
      std::lock_guard<std::mutex> g(ctx->spare_mu);
      if (ctx->spare_dev && ctx->spare_dev_cap >= b->bytes) {
        b->d_mem = ctx->spare_dev;
        b->dev_cap = ctx->spare_dev_cap;
        ctx->spare_dev = nullptr;
        ctx->spare_dev_cap = 0;
      }
      if (ctx->spare_host && ctx->spare_host_cap >= b->stage_bytes) {
        b->h_stage = ctx->spare_host;
        b->host_cap = ctx->spare_host_cap;
        ctx->spare_host = nullptr;
        ctx->spare_host_cap = 0;
      }
    }
    // allocations with 1/8 of headroom, rounded up on a coarse grid (at most
    // another 1/8), so that a later batch of similar size -- a new event set
    // of the same mix -- fits the one this batch leaves
    auto rounded = [](size_t need) {
      need += need / 8;
      size_t step = 1;
      while (step * 8 < need) step <<= 1;
      return (need + step - 1) / step * step;
    };
    if (!b->d_mem) {
      const size_t cap = rounded(b->bytes);
      cudaError_t ce = cudaMalloc(&b->d_mem, cap);
      if (ce != cudaSuccess) {
        cudaGetLastError();
        b->d_mem = nullptr;
        set_last_error(std::string("cudaMalloc of ") + std::to_string(cap) + " bytes: " +
                       cudaGetErrorString(ce));
        return FSM_ERR_OUT_OF_MEMORY;
      }
      b->dev_cap = cap;
    }
    if (!b->h_stage) {
      const size_t cap = rounded(b->stage_bytes);
      FSM_CUDA_TRY(cudaMallocHost(&b->h_stage, cap));
      b->host_cap = cap;
    }
  }
  char* D = b->d_mem;
  char* H = b->h_stage;
  std::memset(H, 0, upload_bytes);
  b->desc_off = o_ev2;
  b->desc_bytes = o_tiles - o_ev2;
  // ---- fill tables (per event; several threads for large tables)
  parallel_for(n, upload_bytes > ((size_t)8 << 20) ? host_threads() : 1, [&](int i) {
    const EventPlan& P = b->plans[i];
    const EvOffs& o = eo[i];
    std::memcpy(H + o.cs, P.cs.data(), P.cs.size() * sizeof(FSM_FLOAT2));
    if (!P.is3d) {
      std::memcpy(H + o.tab2, P.tab2.data(), P.tab2.size() * sizeof(PhiEntry2D));
      std::memcpy(H + o.chunks, P.chunks2.data(), P.chunks2.size() * sizeof(Chunk2D));
      std::memcpy(H + o.axx, P.axx.data(), P.axx.size() * sizeof(AxisNode));
      std::memcpy(H + o.axy, P.axy.data(), P.axy.size() * sizeof(AxisNode));
    } else {
      std::memcpy(H + o.re, P.re.data(), P.re.size() * sizeof(RapEta));
      std::memcpy(H + o.rapf, P.rapf.data(), P.rapf.size() * 4);
      std::memcpy(H + o.rapfB, P.rapfB.data(), P.rapfB.size() * 4);
      std::memcpy(H + o.jac, P.jac.data(), P.jac.size() * 4);
      parallel_copy(H + o.tab3, P.tab3->data(), P.tab3->size() * sizeof(PhiEntry3D));
      std::memcpy(H + o.plane_of, P.plane_of.data(), P.plane_of.size() * 4);
      std::memcpy(H + o.cw_start, P.cw_start.data(), P.cw_start.size() * 4);
      std::memcpy(H + o.cw, P.cw.data(), P.cw.size() * sizeof(CombW));
    }
  });
  // ---- output slab layout: per event (default) or group by group
  b->grouped_out = mem && mem->grouped_out;
  b->out_goff.assign(n, {});
  {
    size_t off = 0;
    for (int g = 0; g < kOutGroups; ++g) {
      b->group_off[g] = off;
      size_t ge = 0;
      for (int i = 0; i < n; ++i) {
        const EventPlan& P = b->plans[i];
        if (g >= 6 && !P.baryon) continue;
        ge += (size_t)kOutGroupComps[g] * P.DIM;
      }
      b->group_elems[g] = ge;
      off += ge;
    }
    size_t gcur[kOutGroups];
    for (int g = 0; g < kOutGroups; ++g) gcur[g] = b->group_off[g];
    for (int i = 0; i < n; ++i) {
      const EventPlan& P = b->plans[i];
      size_t within = 0;
      for (int g = 0; g < kOutGroups; ++g) {
        if (g >= 6 && !P.baryon) {
          b->out_goff[i][g] = 0;
          continue;
        }
        const size_t sz = (size_t)kOutGroupComps[g] * P.DIM;
        if (b->grouped_out) {
          b->out_goff[i][g] = gcur[g];
          gcur[g] += sz;
        } else {
          b->out_goff[i][g] = b->out_off[i] + within;
        }
        within += sz;
      }
    }
  }
  // ---- per-event io views
  b->d_in_e.assign(n, nullptr);
  b->d_in_nB.assign(n, nullptr);
  b->d_out.assign(n, fsm_outputs{});
  b->d_T.assign(n, nullptr);
  b->d_J.assign(n, nullptr);
  for (int i = 0; i < n; ++i) {
    const EventPlan& P = b->plans[i];
    const size_t DIM = P.DIM;
    if (b->own_io) {
      float* in = reinterpret_cast<float*>(D + b->in_slab_off) + b->in_off[i];
      b->d_in_e[i] = in;
      b->d_in_nB[i] = P.baryon ? in + DIM : nullptr;
      float* o = reinterpret_cast<float*>(D + b->out_slab_off);
      const auto& go = b->out_goff[i];
      fsm_outputs v{};
      v.T = o + go[0];
      v.e = o + go[1];
      v.P = o + go[2];
      v.Pi = o + go[3];
      v.u = o + go[4];
      v.pi = o + go[5];
      if (P.baryon) {
        v.J = o + go[6];
        v.nB = o + go[7];
        v.V = o + go[8];
      }
      b->d_out[i] = v;
      b->d_T[i] = v.T;
      b->d_J[i] = v.J;
    } else {
      b->d_in_e[i] = const_cast<float*>(ext_in_e[i]);
      b->d_in_nB[i] = ext_in_nB ? const_cast<float*>(ext_in_nB[i]) : nullptr;
      b->d_out[i] = ext_out[i];
      b->d_T[i] = ext_out[i].T ? ext_out[i].T : reinterpret_cast<float*>(D + eo[i].T);
      b->d_J[i] = P.baryon ? (ext_out[i].J ? ext_out[i].J : reinterpret_cast<float*>(D + eo[i].J))
                           : nullptr;
    }
  }
  // ---- descriptors
  b->ev2.assign(n2, Ev2D{});
  b->ev3.assign(n3, Ev3D{});
  b->evl.assign(n, EvLandau{});
  int max_np2 = 0, max_np3 = 0;
  for (int i = 0; i < n; ++i) {
    const EventPlan& P = b->plans[i];
    const EvOffs& o = eo[i];
    const fsm_params& p = P.p;
    if (!P.is3d) {
      Ev2D& e = b->ev2[b->ev2_of[i]];
      e.NX = p.DIM_X;
      e.NY = p.DIM_Y;
      e.NPHI = p.DIM_PHIP;
      e.NR = p.DIM_RAP;
      e.DX = p.DX;
      e.DY = p.DY;
      e.DTAU = p.DTAU;
      e.TAU = p.TAU;
      e.xmin = P.xmin;
      e.ymin = P.ymin;
      e.xmax_i = P.xmax_i;
      e.ymax_i = P.ymax_i;
      e.d_phip = P.d_phip;
      e.tab = reinterpret_cast<const PhiEntry2D*>(D + o.tab2);
      e.chunks = reinterpret_cast<const Chunk2D*>(D + o.chunks);
      for (int sh = 0; sh < kShapes2D; ++sh) {
        e.choff[sh] = P.choff[sh];
        e.nch[sh] = P.nch[sh];
      }
      b->box_cap2 = std::max(b->box_cap2, P.box_elems);
      e.e_gev = b->d_in_e[i];
      e.ax = reinterpret_cast<const AxisNode*>(D + o.axx) + kPadLo;
      e.ay = reinterpret_cast<const AxisNode*>(D + o.axy) + kPadLo;
      e.fa = reinterpret_cast<float*>(D + o.fa);
      e.sy = reinterpret_cast<float*>(D + o.sy);
      e.nodes = reinterpret_cast<FSM_FLOAT4*>(D + o.nodes);
      e.T = b->d_T[i];
      e.charge = 0;
      e.fb_scale = 1.0f;
      e.chunk = P.phi_chunk;
      e.raw = P.input_fm4 ? 1 : 0;
      if (P.baryon) {  // charge pass: same geometry and tables, its own field and scratch
        Ev2D& q = b->ev2[b->evq_of[i]];
        q = e;
        q.charge = 1;
        q.qnorm = P.normB;
        q.fb_scale = P.fb_scale2;
        q.jscale = P.jscale2;
        q.DRAP = p.DRAP;
        q.e_gev = b->d_in_nB[i];
        q.fa = reinterpret_cast<float*>(D + o.qfa);
        q.sy = reinterpret_cast<float*>(D + o.qsy);
        q.nodes = reinterpret_cast<FSM_FLOAT4*>(D + o.qnodes);
        q.T = nullptr;
        q.J = b->d_J[i];
      }
      max_np2 = std::max(max_np2, p.DIM_PHIP);
    } else {
      Ev3D& e = b->ev3[b->ev3_of[i]];
      e.NX = p.DIM_X;
      e.NY = p.DIM_Y;
      e.NE = p.DIM_ETA;
      e.NR = p.DIM_RAP;
      e.NPHI = p.DIM_PHIP;
      e.r_lo = P.r_lo;
      e.r_hi = P.r_hi;
      e.baryon = P.baryon ? 1 : 0;
      e.raw = P.input_fm4 ? 1 : 0;
      e.DX = p.DX;
      e.DY = p.DY;
      e.xmin = P.xmin;
      e.ymin = P.ymin;
      e.norm = P.norm;
      e.normB = P.normB;
      e.d_phip = P.d_phip;
      e.DRAP = p.DRAP;
      e.cs = reinterpret_cast<const FSM_FLOAT2*>(D + o.cs);
      e.re = reinterpret_cast<const RapEta*>(D + o.re);
      e.rapf = reinterpret_cast<const float*>(D + o.rapf);
      e.rapfB = reinterpret_cast<const float*>(D + o.rapfB);
      e.jac = reinterpret_cast<const float*>(D + o.jac);
      e.e_gev = b->d_in_e[i];
      e.nodes3 = D + o.nodes3;
      e.nodesc = D + o.nodesc;
      e.plane_of = reinterpret_cast<const int*>(D + o.plane_of);
      e.cw_start = reinterpret_cast<const int*>(D + o.cw_start);
      e.cw = reinterpret_cast<const CombW*>(D + o.cw);
      e.tab3 = reinterpret_cast<const PhiEntry3D*>(D + o.tab3);
      e.nB = b->d_in_nB[i];
      e.T = b->d_T[i];
      e.J = b->d_J[i];
      max_np3 = std::max(max_np3, p.DIM_PHIP);
    }
    EvLandau& l = b->evl[i];
    l.DIM = P.DIM;
    l.is3d = P.is3d ? 1 : 0;
    l.baryon = P.baryon ? 1 : 0;
    l.eos = p.EOS_TYPE;
    l.viscous = p.VISCOUS_MATCHING;
    l.TAU = p.TAU;
    l.T = b->d_T[i];
    l.J = b->d_J[i];
    const fsm_outputs& v = b->d_out[i];
    l.e = v.e;
    l.P = v.P;
    l.Pi = v.Pi;
    l.u = v.u;
    l.pi = v.pi;
    l.nB = v.nB;
    l.V = v.V;
    b->samples += P.samples;
  }
  b->cs_cap2 = max_np2;
  b->cs_cap3 = (max_np3 + 1) & ~1;
  b->box_cap2 = (b->box_cap2 + 7) & ~7;  // float4 units, 128-byte multiple
  b->smem2 = stream2d_smem(b->box_cap2);
  // thread-private moment slots of the two 3D kernels
  b->smem3 = (size_t)kThreads3D * kCellsPerThread * kSlots3D * 4;
  b->smem3b = (size_t)kThreads3D * kCellsPerThread * kSlots3DBaryon * 4;
  b->smem_rows = prep_rows_smem(b->ny_cap2);
  b->smem_strip = prep_strip_smem(b->strip_cap2);
  // the kernels index their dynamic shared memory by these capacities
  if (n3 && b->smem3 == 0) {
    set_last_error("internal error: dynamic shared memory below the staged tables");
    return FSM_ERR_CUDA;
  }
  std::memcpy(H + o_ev2, b->ev2.data(), n2 * sizeof(Ev2D));
  std::memcpy(H + o_ev3, b->ev3.data(), n3 * sizeof(Ev3D));
  std::memcpy(H + o_evl, b->evl.data(), n * sizeof(EvLandau));
  std::memcpy(H + o_tiles, tiles.data(), tiles.size() * sizeof(Tile2D));
  std::memcpy(H + o_rows, rows.data(), rows.size() * sizeof(LineBlock));
  std::memcpy(H + o_cols, cols.data(), cols.size() * sizeof(LineBlock));
  std::memcpy(H + o_rows_l, rows_l.data(), rows_l.size() * sizeof(LineBlock));
  std::memcpy(H + o_cols_l, cols_l.data(), cols_l.size() * sizeof(LineBlock));
  std::memcpy(H + o_prep3, prep3.data(), prep3.size() * sizeof(CellBlock));
  std::memcpy(H + o_tiles3, tiles3.data(), tiles3.size() * sizeof(Tile3D));
  std::memcpy(H + o_bl, bl.data(), bl.size() * sizeof(CellBlock));
  b->d_ev2 = reinterpret_cast<Ev2D*>(D + o_ev2);
  b->d_ev3 = reinterpret_cast<Ev3D*>(D + o_ev3);
  b->d_evl = reinterpret_cast<EvLandau*>(D + o_evl);
  b->d_tiles = reinterpret_cast<Tile2D*>(D + o_tiles);
  b->d_rows = reinterpret_cast<LineBlock*>(D + o_rows);
  b->d_cols = reinterpret_cast<LineBlock*>(D + o_cols);
  b->d_rows_l = reinterpret_cast<LineBlock*>(D + o_rows_l);
  b->d_cols_l = reinterpret_cast<LineBlock*>(D + o_cols_l);
  b->d_prep3 = reinterpret_cast<CellBlock*>(D + o_prep3);
  b->d_tiles3 = reinterpret_cast<Tile3D*>(D + o_tiles3);
  b->d_bl = reinterpret_cast<CellBlock*>(D + o_bl);
  b->d_ctr = reinterpret_cast<Counters*>(D + o_ctr);
  b->d_err = reinterpret_cast<int*>(D + o_err);
  b->ntiles = (int)tiles.size();
  b->nrows = (int)rows.size();
  b->ncols = (int)cols.size();
  b->nrows_l = (int)rows_l.size();
  b->ncols_l = (int)cols_l.size();
  b->nprep3 = (int)prep3.size();
  b->ntiles3 = (int)tiles3.size();
  b->nbl = (int)bl.size();
  if (mem && mem->dev)
    FSM_CUDA_TRY(cudaMemcpyAsync(D, H, upload_bytes, cudaMemcpyHostToDevice, mem->stream));
  else
    FSM_CUDA_TRY(cudaMemcpy(D, H, upload_bytes, cudaMemcpyHostToDevice));
  // ---- launch geometry
  if (b->nrows) {
    fsm_status ss = ensure_dyn_smem((const void*)fsm_prep2d_rows_kernel, ctx->device, b->smem_strip,
                                    &g_smem_srows[ctx->device & 63]);
    if (ss != FSM_OK) return ss;
    ss = ensure_dyn_smem((const void*)fsm_prep2d_cols_kernel, ctx->device, b->smem_strip,
                         &g_smem_scols[ctx->device & 63]);
    if (ss != FSM_OK) return ss;
  }
  if (b->nrows_l) {
    fsm_status ss = ensure_dyn_smem((const void*)fsm_prep2d_rows_long_kernel, ctx->device,
                                    b->smem_rows, &g_smem_rows[ctx->device & 63]);
    if (ss != FSM_OK) return ss;
  }
  if (b->ntiles) {
    fsm_status ss = ensure_dyn_smem((const void*)fsm_stream2d_kernel, ctx->device, b->smem2,
                                    &g_smem2[ctx->device & 63]);
    if (ss != FSM_OK) return ss;
    int occ = 0;
    FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fsm_stream2d_kernel, kThreads2D,
                                                               b->smem2));
    b->grid2 = std::max(1, std::min(b->ntiles, ctx->num_sms * std::max(occ, 1)));
  }
  if (b->ntiles3 > b->ntiles3b) {
    fsm_status ss = ensure_dyn_smem((const void*)fsm_stream3d_kernel, ctx->device, b->smem3,
                                    &g_smem3[ctx->device & 63]);
    if (ss != FSM_OK) return ss;
    int occ = 0;
    FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fsm_stream3d_kernel, kThreads3D,
                                                               b->smem3));
    b->grid3 = std::max(1, std::min((b->ntiles3 - b->ntiles3b) * kParts3D, ctx->num_sms * std::max(occ, 1)));
  }
  if (b->ntiles3b) {
    fsm_status ss = ensure_dyn_smem((const void*)fsm_stream3d_baryon_kernel, ctx->device, b->smem3b,
                                    &g_smem3b[ctx->device & 63]);
    if (ss != FSM_OK) return ss;
    int occ = 0;
    FSM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fsm_stream3d_baryon_kernel,
                                                               kThreads3D, b->smem3b));
    b->grid3b = std::max(1, std::min(b->ntiles3b * kParts3D, ctx->num_sms * std::max(occ, 1)));
  }
  if (mem && mem->dev)
    FSM_CUDA_TRY(cudaMemsetAsync(b->d_err, 0, sizeof(int) * 4, mem->stream));
  else
    FSM_CUDA_TRY(cudaMemset(b->d_err, 0, sizeof(int) * 4));
  *out = b.release();
  return FSM_OK;
}

cudaEvent_t pool_event(fsm_ctx* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// The six-launch sequence.  With `timing`, CUDA events bracket the prep,
// stream and Landau groups on the launching stream.
fsm_status enqueue(fsm_batch* b, cudaStream_t s, bool timing) {
  fsm_ctx* ctx = b->ctx;
  TimingSet ts{};
  if (timing) {
    for (int k = 0; k < 4; ++k) ts.ev[k] = pool_event(ctx);
    ts.samples = b->samples;
    cudaEventRecord(ts.ev[0], s);
  }
  FSM_CUDA_TRY(cudaMemsetAsync(b->d_ctr, 0, sizeof(Counters), s));
  if (b->nrows) fsm_prep2d_rows_kernel<<<b->nrows, kPrepThreads, b->smem_strip, s>>>(b->d_ev2, b->d_rows);
  if (b->nrows_l)
    fsm_prep2d_rows_long_kernel<<<b->nrows_l, kPrepRows * 32, b->smem_rows, s>>>(
        b->d_ev2, b->d_rows_l, b->ny_cap2);
  if (b->ncols) fsm_prep2d_cols_kernel<<<b->ncols, kPrepThreads, b->smem_strip, s>>>(b->d_ev2, b->d_cols);
  if (b->ncols_l) fsm_prep2d_cols_long_kernel<<<b->ncols_l, 128, 0, s>>>(b->d_ev2, b->d_cols_l);
  if (b->nprep3) fsm_prep3d_kernel<<<b->nprep3, 256, 0, s>>>(b->d_ev3, b->d_prep3);
  if (timing) cudaEventRecord(ts.ev[1], s);
  if (b->ntiles)
    fsm_stream2d_kernel<<<b->grid2, kThreads2D, b->smem2, s>>>(b->d_ev2, b->d_tiles, b->ntiles,
                                                               b->box_cap2, b->d_ctr, b->d_err,
                                                               b->wait_polls);
  if (b->ntiles3b)
    fsm_stream3d_baryon_kernel<<<b->grid3b, kThreads3D, b->smem3b, s>>>(b->d_ev3, b->d_tiles3,
                                                                       b->ntiles3b, b->d_ctr);
  if (b->ntiles3 > b->ntiles3b)
    fsm_stream3d_kernel<<<b->grid3, kThreads3D, b->smem3, s>>>(
        b->d_ev3, b->d_tiles3 + b->ntiles3b, b->ntiles3 - b->ntiles3b, b->d_ctr);
  if (timing) cudaEventRecord(ts.ev[2], s);
  if (b->nbl2) fsm_landau_kernel<<<b->nbl2, kThreadsLandau, 0, s>>>(b->d_evl, b->d_bl, b->d_ctr);
  if (b->nbl > b->nbl2)
    fsm_landau3d_kernel<<<b->nbl - b->nbl2, kThreadsLandau, 0, s>>>(b->d_evl, b->d_bl + b->nbl2,
                                                                    b->d_ctr);
  if (timing) {
    cudaEventRecord(ts.ev[3], s);
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->pending.push_back(ts);
  }
  FSM_CUDA_TRY(cudaGetLastError());
  return FSM_OK;
}

bool same_params(const fsm_params& a, const fsm_params& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }
fsm_status launch(fsm_batch* b, cudaStream_t s);

// A batch with E_DEP_FS events: the sums of every such event's converted
// profile in one launch (one thread per event, the reference's order), one
// sync, then DTAU per event and the inner batch planned with it (reused while
// every DTAU stays the same), launched on the same stream.
fsm_status launch_deferred(fsm_batch* b, cudaStream_t s) {
  const int ne = (int)b->edep.size();
  const float* const* d_ptr = reinterpret_cast<const float* const*>(b->d_edep);
  const int* d_cells = reinterpret_cast<const int*>(b->d_edep + align_up(ne * sizeof(float*)));
  float* d_sums = reinterpret_cast<float*>(b->d_edep + align_up(ne * sizeof(float*)) +
                                           align_up(ne * sizeof(int)));
  fsm_edep_sums_kernel<<<ne, 256, 0, s>>>(d_ptr, d_cells, ne, d_sums);  // a block per event
  FSM_CUDA_TRY(cudaGetLastError());
  FSM_CUDA_TRY(cudaMemcpyAsync(b->h_sums, d_sums, 2 * ne * sizeof(float), cudaMemcpyDeviceToHost, s));
  FSM_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<fsm_params> res = b->raw;
  for (int k = 0; k < ne; ++k) {
    fsm_params& p = res[b->edep[k]];
    p.DTAU = edep_dtau(p, b->h_sums[2 * k], b->h_sums[2 * k + 1]);
    p.E_DEP_FS = 0;
    fsm_params_derive(&p);
  }
  bool same = b->inner && res.size() == b->inner_params.size();
  for (size_t i = 0; same && i < res.size(); ++i) same = same_params(res[i], b->inner_params[i]);
  if (!same) {
    batch_free(b->inner);
    b->inner = nullptr;
    const int n = (int)res.size();
    std::vector<const float*> ie(b->d_in_e.begin(), b->d_in_e.end()),
        inb(b->d_in_nB.begin(), b->d_in_nB.end());
    fsm_status st = batch_build(b->ctx, n, res.data(), nullptr, ie.data(), inb.data(), b->d_out.data(),
                                &b->inner);
    if (st != FSM_OK) return st;
    b->inner_params = res;
  }
  b->samples = b->inner->samples;
  return launch(b->inner, s);
}

fsm_status launch(fsm_batch* b, cudaStream_t s) {
  fsm_ctx* ctx = b->ctx;
  b->last_stream = s;
  if (!b->edep.empty()) return launch_deferred(b, s);
  if (ctx->timing) return enqueue(b, s, true);
  if (!b->graph || b->graph_stream != s) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    FSM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    fsm_status st = enqueue(b, s, false);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (st != FSM_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (ce != cudaSuccess) {
      set_last_error(std::string("graph capture: ") + cudaGetErrorString(ce));
      return FSM_ERR_CUDA;
    }
    ce = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      set_last_error(std::string("graph instantiate: ") + cudaGetErrorString(ce));
      b->graph = nullptr;
      return FSM_ERR_CUDA;
    }
    b->graph_stream = s;
  }
  FSM_CUDA_TRY(cudaGraphLaunch(b->graph, s));
  return FSM_OK;
}

// Reads the kernels' error counters in stream order on the batch's last
// stream and waits for it, so every copy enqueued before has completed.
fsm_status check_kernel_errors(fsm_batch* b) {
  if (b->inner) {  // the launches of an E_DEP_FS batch ran its inner batch
    b->inner->last_stream = b->last_stream ? b->last_stream : b->inner->last_stream;
    return check_kernel_errors(b->inner);
  }
  int err[4] = {0, 0, 0, 0};
  cudaStream_t s = b->last_stream ? b->last_stream : b->ctx->stream;
  FSM_CUDA_TRY(cudaMemcpyAsync(err, b->d_err, sizeof(err), cudaMemcpyDeviceToHost, s));
  FSM_CUDA_TRY(cudaStreamSynchronize(s));
  if (err[0]) {
    set_last_error("stream kernel: " + std::to_string(err[0]) +
                   " samples fell outside the staged footprint");
    return FSM_ERR_CUDA;
  }
  if (err[1]) {
    set_last_error("stream kernel: " + std::to_string(err[1]) +
                   " staged copies did not complete within the bounded wait");
    return FSM_ERR_TIMEOUT;
  }
  return FSM_OK;
}


fsm_status fill_info(const EventPlan& P, fsm_run_info* info) {
  if (!info) return FSM_OK;
  info->dim_phip = P.p.DIM_PHIP;
  info->dtau = P.p.DTAU;
  info->tau = P.p.TAU;
  info->live_rap_lo = P.r_lo;
  info->live_rap_hi = P.r_hi;
  info->samples = P.samples;
  return FSM_OK;
}

cudaStream_t pick_stream(fsm_ctx* ctx, void* stream) {
  return stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream;
}

}  // namespace rt
}  // namespace fsm

// ====================================================================== C ABI
extern "C" fsm_status fsm_device_count(int* n) {
  if (!n) return FSM_ERR_INVALID_ARG;
  *n = 0;
  if (cudaGetDeviceCount(n) != cudaSuccess) {
    cudaGetLastError();
    *n = 0;
  }
  return FSM_OK;
}

extern "C" fsm_status fsm_ctx_create(fsm_ctx** out, const fsm_ctx_opts* opts) {
  if (!out) return FSM_ERR_INVALID_ARG;
  *out = nullptr;
  if (!has_device()) {
    set_last_error("no CUDA device visible; the library has no CPU fallback");
    return FSM_ERR_NO_DEVICE;
  }
  std::unique_ptr<fsm_ctx> c(new fsm_ctx());
  if (opts) {
    c->device = opts->device;
    c->timing = opts->enable_timing != 0;
  }
  FSM_CUDA_TRY(cudaSetDevice(c->device));
  FSM_CUDA_TRY(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
  FSM_CUDA_TRY(cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  FSM_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  *out = c.release();
  return FSM_OK;
}

extern "C" void fsm_ctx_destroy(fsm_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  batch_free(ctx->single_host);
  batch_free(ctx->single_dev);
  for (auto& t : ctx->pending)
    for (int k = 0; k < 4; ++k) cudaEventDestroy(t.ev[k]);
  for (auto e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->d_sums) cudaFree(ctx->d_sums);
  if (ctx->h_sums) cudaFreeHost(ctx->h_sums);
  if (ctx->spare_dev) cudaFree(ctx->spare_dev);
  if (ctx->spare_host) cudaFreeHost(ctx->spare_host);
  if (ctx->pin_stage) cudaFreeHost(ctx->pin_stage);
  for (auto e : ctx->pin_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

extern "C" fsm_status fsm_ctx_timing(fsm_ctx* ctx, fsm_timing* t, int reset) {
  if (!ctx) return FSM_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  for (auto& ts : ctx->pending) {
    FSM_CUDA_TRY(cudaEventSynchronize(ts.ev[3]));
    float a = 0, b = 0, c = 0;
    cudaEventElapsedTime(&a, ts.ev[0], ts.ev[1]);
    cudaEventElapsedTime(&b, ts.ev[1], ts.ev[2]);
    cudaEventElapsedTime(&c, ts.ev[2], ts.ev[3]);
    ctx->acc.prep_ms += a;
    ctx->acc.stream_ms += b;
    ctx->acc.landau_ms += c;
    ctx->acc.prep_launches += 1;
    ctx->acc.stream_launches += 1;
    ctx->acc.landau_launches += 1;
    ctx->acc.stream_samples += ts.samples;
    for (int k = 0; k < 4; ++k) ctx->event_pool.push_back(ts.ev[k]);
  }
  ctx->pending.clear();
  if (t) *t = ctx->acc;
  if (reset) ctx->acc = fsm_timing{};
  return FSM_OK;
}

namespace {
// Copies between caller host buffers and the device on the context's stream.
// Pinned caller buffers are copied directly.  Pageable ones go through the
// context's two pinned chunks: a pageable cudaMemcpy is staged by the driver
// one bounce buffer at a time on one thread (~15 GB/s); here the host copy of
// one chunk (several threads) overlaps the device copy of the next.  Returns
// once every copy has completed.
struct HostSeg {
  char* h;        // caller host memory
  char* d;        // device memory
  size_t bytes;
};
constexpr size_t kPinChunk = size_t(8) << 20;

bool is_pinned(const void* h) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

fsm_status ensure_pin_stage(fsm_ctx* ctx) {
  if (ctx->pin_stage) return FSM_OK;
  FSM_CUDA_TRY(cudaMallocHost(&ctx->pin_stage, 2 * kPinChunk));
  for (auto& e : ctx->pin_ev) FSM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return FSM_OK;
}

fsm_status copy_staged(fsm_ctx* ctx, cudaStream_t st, const std::vector<HostSeg>& segs, bool to_device) {
  const cudaMemcpyKind kind = to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  struct Piece {
    char* h;
    char* d;
    size_t n;
  };
  std::vector<Piece> pieces;
  for (const HostSeg& g : segs) {
    if (!g.h || !g.d || !g.bytes) continue;
    if (is_pinned(g.h)) {
      FSM_CUDA_TRY(cudaMemcpyAsync(to_device ? g.d : g.h, to_device ? g.h : g.d, g.bytes, kind, st));
      continue;
    }
    for (size_t o = 0; o < g.bytes; o += kPinChunk)
      pieces.push_back(Piece{g.h + o, g.d + o, std::min(kPinChunk, g.bytes - o)});
  }
  if (!pieces.empty()) {
    fsm_status s = ensure_pin_stage(ctx);
    if (s != FSM_OK) return s;
    // a call that failed half-way may have left a copy into a chunk in flight
    FSM_CUDA_TRY(cudaStreamSynchronize(st));
  }
  const int np = (int)pieces.size();
  if (to_device) {
    // host copy of piece i into chunk i % 2 once that chunk's previous upload
    // has left it, then its upload
    for (int i = 0; i < np; ++i) {
      char* buf = ctx->pin_stage + (i & 1) * kPinChunk;
      if (i >= 2) FSM_CUDA_TRY(cudaEventSynchronize(ctx->pin_ev[i & 1]));
      parallel_copy(buf, pieces[i].h, pieces[i].n);
      FSM_CUDA_TRY(cudaMemcpyAsync(pieces[i].d, buf, pieces[i].n, kind, st));
      FSM_CUDA_TRY(cudaEventRecord(ctx->pin_ev[i & 1], st));
    }
  } else {
    // download of piece i into chunk i % 2 once the host has copied piece
    // i - 2 out of it; the host copies piece i - 1 while piece i downloads
    for (int i = 0; i <= np; ++i) {
      if (i >= 1) {
        const int j = i - 1;  // download issued last round: copy it out
        FSM_CUDA_TRY(cudaEventSynchronize(ctx->pin_ev[j & 1]));
        if (i < np) {
          char* buf = ctx->pin_stage + (i & 1) * kPinChunk;
          FSM_CUDA_TRY(cudaMemcpyAsync(buf, pieces[i].d, pieces[i].n, kind, st));
          FSM_CUDA_TRY(cudaEventRecord(ctx->pin_ev[i & 1], st));
        }
        parallel_copy(pieces[j].h, ctx->pin_stage + (j & 1) * kPinChunk, pieces[j].n);
      } else if (np > 0) {
        FSM_CUDA_TRY(cudaMemcpyAsync(ctx->pin_stage, pieces[0].d, pieces[0].n, kind, st));
        FSM_CUDA_TRY(cudaEventRecord(ctx->pin_ev[0], st));
      }
    }
  }
  FSM_CUDA_TRY(cudaStreamSynchronize(st));
  return FSM_OK;
}

// One event, host buffers in and out; fm4: the energy profile is already in
// fm^-4 (otherwise GeV/fm^3, converted as src/FreestreamMilne.cpp:266-267).
fsm_status run_event_host(fsm_ctx* ctx, const fsm_params* p, const float* e_gev, const float* nB,
                          const fsm_outputs* host_out, fsm_run_info* info, bool fm4) {
  if (!ctx || !p || !e_gev || !host_out) return FSM_ERR_INVALID_ARG;
  if (p->BARYON && !nB) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(ctx->device));
  fsm_status s;
  fsm_batch* b = ctx->single_host;
  // the cached batch serves the same parameters (and input units) again
  // without planning (an energy-dependent DTAU depends on the profile, so
  // those events re-plan)
  if (!b || p->E_DEP_FS != 0 || !same_params(ctx->single_host_raw, *p) || ctx->single_host_fm4 != fm4) {
    EventPlan P;
    std::string why;
    int window = 0, chunk = 0;
    bool tail = true;
    event_tuning(ctx, *p, &window, &chunk, &tail);
    s = plan_event(*p, e_gev, &P, &why, window, fm4, tail);
    if (s != FSM_OK) {
      set_last_error(why);
      return s;
    }
    if (!b || !same_params(b->plans[0].p, P.p) || ctx->single_host_fm4 != fm4) {
      batch_free(ctx->single_host);
      ctx->single_host = nullptr;
      const float* he[1] = {e_gev};
      BatchMem units;
      units.input_fm4 = fm4;
      s = batch_build(ctx, 1, p, he, nullptr, nullptr, nullptr, &ctx->single_host, &units);
      if (s != FSM_OK) return s;
      b = ctx->single_host;
    }
    ctx->single_host_raw = *p;
    ctx->single_host_fm4 = fm4;
  }
  const EventPlan& P = b->plans[0];
  cudaStream_t st = ctx->stream;
  const size_t DIM = P.DIM;
  auto seg = [&](const float* h, const float* dv, size_t comps) {
    return HostSeg{const_cast<char*>(reinterpret_cast<const char*>(h)),
                   const_cast<char*>(reinterpret_cast<const char*>(dv)), comps * DIM * 4};
  };
  std::vector<HostSeg> up{seg(e_gev, b->d_in_e[0], 1)};
  if (P.baryon) up.push_back(seg(nB, b->d_in_nB[0], 1));
  if ((s = copy_staged(ctx, st, up, true)) != FSM_OK) return s;
  s = launch(b, st);
  if (s != FSM_OK) return s;
  const fsm_outputs& d = b->d_out[0];
  std::vector<HostSeg> down{seg(host_out->T, d.T, 10), seg(host_out->e, d.e, 1), seg(host_out->P, d.P, 1),
                            seg(host_out->Pi, d.Pi, 1), seg(host_out->u, d.u, 4), seg(host_out->pi, d.pi, 10)};
  if (P.baryon) {
    down.push_back(seg(host_out->J, d.J, 4));
    down.push_back(seg(host_out->nB, d.nB, 1));
    down.push_back(seg(host_out->V, d.V, 4));
  }
  if ((s = copy_staged(ctx, st, down, false)) != FSM_OK) return s;
  if ((s = check_kernel_errors(b)) != FSM_OK) return s;
  return fill_info(P, info);
}
}  // namespace

extern "C" fsm_status fsm_run_event(fsm_ctx* ctx, const fsm_params* p, const float* e_gev,
                                    const float* nB, const fsm_outputs* host_out,
                                    fsm_run_info* info) {
  return run_event_host(ctx, p, e_gev, nB, host_out, info, false);
}

extern "C" fsm_status fsm_run_event_fm4(fsm_ctx* ctx, const fsm_params* p, const float* e_fm4,
                                        const float* nB, const fsm_outputs* host_out,
                                        fsm_run_info* info) {
  return run_event_host(ctx, p, e_fm4, nB, host_out, info, true);
}

extern "C" fsm_status fsm_run_event_device(fsm_ctx* ctx, const fsm_params* p, const float* d_e_gev,
                                           const float* d_nB, const fsm_outputs* dev_out,
                                           void* stream, fsm_run_info* info) {
  if (!ctx || !p || !d_e_gev || !dev_out) return FSM_ERR_INVALID_ARG;
  if (p->BARYON && !d_nB) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t st = pick_stream(ctx, stream);
  fsm_params pe = *p;
  if (pe.E_DEP_FS == 1) {
    // the free-streaming time depends on the profile: its sums are taken on
    // the device in the reference's order and read back before planning
    fsm_params_derive(&pe);
    if (pe.DIM <= 0) return FSM_ERR_INVALID_ARG;
    // device block: [input pointer | cell count | sums]; pinned mirror
    if (!ctx->d_sums) {
      FSM_CUDA_TRY(cudaMalloc(&ctx->d_sums, 64));
      FSM_CUDA_TRY(cudaMallocHost(&ctx->h_sums, 64));
    }
    char* hb = reinterpret_cast<char*>(ctx->h_sums);
    char* db = reinterpret_cast<char*>(ctx->d_sums);
    FSM_CUDA_TRY(cudaStreamSynchronize(st));  // the pinned block may be in use by a previous call
    *reinterpret_cast<const float**>(hb) = d_e_gev;
    *reinterpret_cast<int*>(hb + 16) = pe.DIM;
    FSM_CUDA_TRY(cudaMemcpyAsync(db, hb, 32, cudaMemcpyHostToDevice, st));
    fsm_edep_sums_kernel<<<1, 256, 0, st>>>(reinterpret_cast<const float* const*>(db),
                                           reinterpret_cast<const int*>(db + 16), 1,
                                           reinterpret_cast<float*>(db + 32));
    FSM_CUDA_TRY(cudaGetLastError());
    FSM_CUDA_TRY(cudaMemcpyAsync(hb + 32, db + 32, 2 * sizeof(float), cudaMemcpyDeviceToHost, st));
    FSM_CUDA_TRY(cudaStreamSynchronize(st));
    const float* sums = reinterpret_cast<const float*>(hb + 32);
    pe.DTAU = edep_dtau(pe, sums[0], sums[1]);
    pe.E_DEP_FS = 0;
  }
  p = &pe;
  EventPlan P;
  std::string why;
  int window = 0, chunk = 0;
  bool tail = true;
  event_tuning(ctx, *p, &window, &chunk, &tail);
  fsm_status s = plan_event(*p, nullptr, &P, &why, window, false, tail);
  if (s != FSM_OK) {
    set_last_error(why);
    return s;
  }
  fsm_batch* b = ctx->single_dev;
  const bool same_io = b && b->d_in_e[0] == d_e_gev && b->d_in_nB[0] == d_nB &&
                       std::memcmp(&b->d_out[0], dev_out, sizeof(fsm_outputs)) == 0;
  if (!b || !same_params(b->plans[0].p, P.p) || !same_io) {
    if (b) cudaStreamSynchronize(b->graph_stream ? b->graph_stream : st);
    batch_free(ctx->single_dev);
    ctx->single_dev = nullptr;
    const float* ie[1] = {d_e_gev};
    const float* inb[1] = {d_nB};
    s = batch_build(ctx, 1, p, nullptr, ie, inb, dev_out, &ctx->single_dev);
    if (s != FSM_OK) return s;
    b = ctx->single_dev;
  }
  s = launch(b, st);
  if (s != FSM_OK) return s;
  return fill_info(b->plans[0], info);
}

extern "C" fsm_status fsm_batch_create(fsm_ctx* ctx, int n, const fsm_params* params,
                                       fsm_batch** out) {
  return fsm_batch_create_ex(ctx, n, params, 0, out);
}

extern "C" fsm_status fsm_batch_create_ex(fsm_ctx* ctx, int n, const fsm_params* params,
                                          int grouped_outputs, fsm_batch** out) {
  if (!ctx || !params || !out || n <= 0) return FSM_ERR_INVALID_ARG;
  *out = nullptr;
  FSM_CUDA_TRY(cudaSetDevice(ctx->device));
  BatchMem layout;  // no pools: only the output layout
  layout.grouped_out = grouped_outputs != 0;
  std::vector<int> edep;
  for (int i = 0; i < n; ++i)
    if (params[i].E_DEP_FS == 1) edep.push_back(i);
  if (edep.empty()) return batch_build(ctx, n, params, nullptr, nullptr, nullptr, nullptr, out, &layout);
  // E_DEP_FS events: this batch holds the slabs (laid out from provisional
  // parameters, which fix only the event sizes); its launches run an inner
  // batch planned with the DTAUs of the uploaded profiles
  std::vector<fsm_params> prov(params, params + n);
  for (int i : edep) prov[i].E_DEP_FS = 0;
  layout.io_only = true;
  fsm_batch* b = nullptr;
  fsm_status st = batch_build(ctx, n, prov.data(), nullptr, nullptr, nullptr, nullptr, &b, &layout);
  if (st != FSM_OK) return st;
  std::unique_ptr<fsm_batch, void (*)(fsm_batch*)> hold(b, batch_free);
  b->edep = edep;
  b->raw.assign(params, params + n);
  for (auto& p : b->raw) fsm_params_derive(&p);
  const int ne = (int)edep.size();
  const size_t o_cells = align_up(ne * sizeof(float*)), o_sums = o_cells + align_up(ne * sizeof(int));
  FSM_CUDA_TRY(cudaMalloc(&b->d_edep, o_sums + 2 * ne * sizeof(float)));
  FSM_CUDA_TRY(cudaMallocHost(&b->h_sums, 2 * ne * sizeof(float)));
  std::vector<char> h(o_sums, 0);
  for (int k = 0; k < ne; ++k) {
    reinterpret_cast<const float**>(h.data())[k] = b->d_in_e[edep[k]];
    reinterpret_cast<int*>(h.data() + o_cells)[k] = b->plans[edep[k]].DIM;
  }
  FSM_CUDA_TRY(cudaMemcpy(b->d_edep, h.data(), o_sums, cudaMemcpyHostToDevice));
  *out = hold.release();
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_group_offset(fsm_batch* b, unsigned mask, int group, int ev,
                                             size_t* elem) {
  if (!b || !elem || !b->own_io || !b->grouped_out || group < 0 || group >= kOutGroups || ev < 0 ||
      ev >= (int)b->plans.size() || !(mask & (1u << group)))
    return FSM_ERR_INVALID_ARG;
  if (group >= 6 && !b->plans[ev].baryon) return FSM_ERR_INVALID_ARG;
  size_t before = 0;
  for (int g = 0; g < group; ++g)
    if (mask & (1u << g)) before += b->group_elems[g];
  *elem = before + (b->out_goff[ev][group] - b->group_off[group]);
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_download_groups(fsm_batch* b, unsigned mask, void* host_out,
                                                void* stream) {
  if (!b || !b->own_io || !b->grouped_out || !host_out) return FSM_ERR_INVALID_ARG;
  b->last_stream = pick_stream(b->ctx, stream);
  char* h = static_cast<char*>(host_out);
  for (int g = 0; g < kOutGroups; ++g) {
    if (!(mask & (1u << g)) || b->group_elems[g] == 0) continue;
    FSM_CUDA_TRY(cudaMemcpyAsync(h, b->d_mem + b->out_slab_off + b->group_off[g] * 4,
                                 b->group_elems[g] * 4, cudaMemcpyDeviceToHost, b->last_stream));
    h += b->group_elems[g] * 4;
  }
  return FSM_OK;
}

namespace {

// Components of a boost-invariant event that vanish by symmetry, per output
// group (bit c: component c): T^{tau eta}, T^{x eta}, T^{y eta}, T^{eta eta};
// u^eta; pi^{tau eta}, pi^{x eta}, pi^{y eta}; J^eta; V^eta.
constexpr unsigned kZeroEta2D[kOutGroups] = {(1u << 3) | (1u << 6) | (1u << 8) | (1u << 9), 0, 0, 0,
                                             1u << 3, (1u << 3) | (1u << 6) | (1u << 8), 1u << 3, 0,
                                             1u << 3};

bool pack_keeps(const fsm_batch* b, unsigned flags, int g, int c, int ev) {
  const EventPlan& P = b->plans[ev];
  if (g >= 6 && !P.baryon) return false;
  if ((flags & FSM_PACK_SKIP_ETA) && !P.is3d && ((kZeroEta2D[g] >> c) & 1u)) return false;
  return true;
}

// Walks the packed layout (groups in mask, events in order, kept components
// in order); f(g, c, ev, src, dst, len) per component, in packed order.
template <class F>
size_t pack_walk(const fsm_batch* b, unsigned mask, unsigned flags, F f) {
  size_t dst = 0;
  const size_t base = b->out_slab_off / 4;
  for (int g = 0; g < kOutGroups; ++g) {
    if (!(mask & (1u << g))) continue;
    for (int i = 0; i < (int)b->plans.size(); ++i) {
      const size_t dim = (size_t)b->plans[i].DIM;
      for (int c = 0; c < kOutGroupComps[g]; ++c) {
        if (!pack_keeps(b, flags, g, c, i)) continue;
        f(g, c, i, base + b->out_goff[i][g] + (size_t)c * dim, dst, dim);
        dst += dim;
      }
    }
  }
  return dst;
}

// Copy list of (mask, flags) on the device (built on first use).
fsm_status pack_prepare(fsm_batch* b, unsigned mask, unsigned flags) {
  if (b->pack_ready && b->pack_mask == mask && b->pack_flags == flags) return FSM_OK;
  std::vector<CopySeg> segs;
  const size_t total = pack_walk(b, mask, flags, [&](int, int, int, size_t src, size_t dst, size_t len) {
    if (!segs.empty()) {  // extend the previous run when both sides continue it
      CopySeg& l = segs.back();
      if ((size_t)l.src + l.len == src && (size_t)l.dst + l.len == dst && l.len < kMaxCopySeg) {
        const size_t add = std::min(len, (size_t)(kMaxCopySeg - l.len));
        l.len += (int)add;
        src += add;
        dst += add;
        len -= add;
      }
    }
    for (size_t o = 0; o < len; o += kMaxCopySeg)
      segs.push_back(CopySeg{(long long)(src + o), (long long)(dst + o),
                             (int)std::min((size_t)kMaxCopySeg, len - o), 0});
  });
  if (segs.size() > b->seg_cap) {
    if (b->d_segs) cudaFree(b->d_segs);
    b->d_segs = nullptr;
    b->seg_cap = 0;
    FSM_CUDA_TRY(cudaMalloc(&b->d_segs, segs.size() * sizeof(CopySeg)));
    b->seg_cap = segs.size();
  }
  if (total > b->pack_cap) {
    if (b->d_pack) cudaFree(b->d_pack);
    b->d_pack = nullptr;
    b->pack_cap = 0;
    FSM_CUDA_TRY(cudaMalloc(&b->d_pack, std::max<size_t>(total, 1) * 4));
    b->pack_cap = total;
  }
  if (!segs.empty())
    FSM_CUDA_TRY(cudaMemcpy(b->d_segs, segs.data(), segs.size() * sizeof(CopySeg),
                            cudaMemcpyHostToDevice));
  b->nsegs = (int)segs.size();
  b->pack_elems = total;
  b->pack_mask = mask;
  b->pack_flags = flags;
  b->pack_ready = true;
  return FSM_OK;
}

}  // namespace

extern "C" size_t fsm_batch_packed_bytes(fsm_batch* b, unsigned mask, unsigned flags) {
  if (!b || !b->own_io) return 0;
  return pack_walk(b, mask, flags, [](int, int, int, size_t, size_t, size_t) {}) * 4;
}

extern "C" fsm_status fsm_batch_packed_offset(fsm_batch* b, unsigned mask, unsigned flags, int group,
                                              int comp, int ev, size_t* elem) {
  if (!b || !elem || !b->own_io || group < 0 || group >= kOutGroups || comp < 0 ||
      comp >= kOutGroupComps[group] || ev < 0 || ev >= (int)b->plans.size() ||
      !(mask & (1u << group)) || !pack_keeps(b, flags, group, comp, ev))
    return FSM_ERR_INVALID_ARG;
  bool found = false;
  pack_walk(b, mask, flags, [&](int g, int c, int i, size_t, size_t dst, size_t) {
    if (g == group && c == comp && i == ev) {
      *elem = dst;
      found = true;
    }
  });
  return found ? FSM_OK : FSM_ERR_INVALID_ARG;
}

extern "C" fsm_status fsm_batch_packed_offsets(fsm_batch* b, unsigned mask, unsigned flags,
                                               size_t* elems, size_t n) {
  const size_t need = b ? b->plans.size() * kOutGroups * 10 : 0;
  if (!b || !elems || !b->own_io || n < need) return FSM_ERR_INVALID_ARG;
  for (size_t i = 0; i < need; ++i) elems[i] = (size_t)-1;
  pack_walk(b, mask, flags, [&](int g, int c, int i, size_t, size_t dst, size_t) {
    elems[((size_t)i * kOutGroups + g) * 10 + c] = dst;
  });
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_download_packed(fsm_batch* b, unsigned mask, unsigned flags,
                                                void* host_out, void* stream) {
  if (!b || !b->own_io || !host_out) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(b->ctx->device));
  fsm_status s = pack_prepare(b, mask, flags);
  if (s != FSM_OK) return s;
  b->last_stream = pick_stream(b->ctx, stream);
  if (b->nsegs == 0) return FSM_OK;
  fsm_pack_kernel<<<b->nsegs, 256, 0, b->last_stream>>>(reinterpret_cast<const float*>(b->d_mem), b->d_pack,
                                                        b->d_segs);
  FSM_CUDA_TRY(cudaGetLastError());
  FSM_CUDA_TRY(cudaMemcpyAsync(host_out, b->d_pack, b->pack_elems * 4, cudaMemcpyDeviceToHost,
                               b->last_stream));
  return FSM_OK;
}

extern "C" size_t fsm_batch_groups_bytes(fsm_batch* b, unsigned mask) {
  if (!b) return 0;
  size_t n = 0;
  for (int g = 0; g < kOutGroups; ++g)
    if (mask & (1u << g)) n += b->group_elems[g] * 4;
  return n;
}

extern "C" void fsm_batch_destroy(fsm_batch* b) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  cudaDeviceSynchronize();
  batch_free(b);
}

extern "C" fsm_status fsm_batch_views(fsm_batch* b, int ev, float** d_e, float** d_nB,
                                      fsm_outputs* dev_out) {
  if (!b || ev < 0 || ev >= (int)b->plans.size()) return FSM_ERR_INVALID_ARG;
  if (d_e) *d_e = b->d_in_e[ev];
  if (d_nB) *d_nB = b->d_in_nB[ev];
  if (dev_out) *dev_out = b->d_out[ev];
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_launch(fsm_batch* b, void* stream) {
  if (!b) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(b->ctx->device));
  return launch(b, pick_stream(b->ctx, stream));
}

extern "C" fsm_status fsm_batch_run_host(fsm_batch* b, const float* const* e_gev,
                                         const float* const* nB, const fsm_outputs* host_out,
                                         void* stream) {
  if (!b || !e_gev) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(b->ctx->device));
  cudaStream_t st = pick_stream(b->ctx, stream);
  const int n = (int)b->plans.size();
  for (int i = 0; i < n; ++i) {
    const EventPlan& P = b->plans[i];
    if (!e_gev[i]) return FSM_ERR_INVALID_ARG;
    FSM_CUDA_TRY(cudaMemcpyAsync(b->d_in_e[i], e_gev[i], (size_t)P.DIM * 4, cudaMemcpyHostToDevice, st));
    if (P.baryon) {
      if (!nB || !nB[i]) return FSM_ERR_INVALID_ARG;
      FSM_CUDA_TRY(cudaMemcpyAsync(b->d_in_nB[i], nB[i], (size_t)P.DIM * 4, cudaMemcpyHostToDevice, st));
    }
  }
  fsm_status s = launch(b, st);
  if (s != FSM_OK) return s;
  if (host_out) {
    for (int i = 0; i < n; ++i) {
      const size_t DIM = b->plans[i].DIM;
      const fsm_outputs& d = b->d_out[i];
      const fsm_outputs& h = host_out[i];
      auto dl = [&](float* hp, const float* dp, size_t comps) -> fsm_status {
        if (hp && dp) FSM_CUDA_TRY(cudaMemcpyAsync(hp, dp, comps * DIM * 4, cudaMemcpyDeviceToHost, st));
        return FSM_OK;
      };
      if ((s = dl(h.T, d.T, 10)) || (s = dl(h.e, d.e, 1)) || (s = dl(h.P, d.P, 1)) ||
          (s = dl(h.Pi, d.Pi, 1)) || (s = dl(h.u, d.u, 4)) || (s = dl(h.pi, d.pi, 10)) ||
          (s = dl(h.J, d.J, 4)) || (s = dl(h.nB, d.nB, 1)) || (s = dl(h.V, d.V, 4)))
        return s;
    }
  }
  FSM_CUDA_TRY(cudaStreamSynchronize(st));
  return check_kernel_errors(b);
}

extern "C" fsm_status fsm_batch_info(fsm_batch* b, int ev, fsm_run_info* info) {
  if (!b || ev < 0 || ev >= (int)b->plans.size()) return FSM_ERR_INVALID_ARG;
  if (!b->edep.empty()) {
    if (!b->inner) {
      set_last_error("E_DEP_FS batch: the run values are known after the first launch");
      return FSM_ERR_PENDING;
    }
    return fill_info(b->inner->plans[ev], info);
  }
  return fill_info(b->plans[ev], info);
}

extern "C" double fsm_batch_samples(fsm_batch* b) { return b ? b->samples : 0.0; }

extern "C" fsm_status fsm_batch_slabs(fsm_batch* b, size_t* in_bytes, size_t* out_bytes) {
  if (!b || !b->own_io) return FSM_ERR_INVALID_ARG;
  if (in_bytes) *in_bytes = b->in_slab_bytes;
  if (out_bytes) *out_bytes = b->out_slab_bytes;
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_event_offsets(fsm_batch* b, int ev, size_t* in_elem,
                                              size_t* out_elem) {
  if (!b || !b->own_io || ev < 0 || ev >= (int)b->plans.size()) return FSM_ERR_INVALID_ARG;
  if (in_elem) *in_elem = b->in_off[ev];
  if (out_elem) *out_elem = b->grouped_out ? (size_t)-1 : b->out_off[ev];
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_upload(fsm_batch* b, const void* host_in, void* stream) {
  if (!b || !b->own_io || !host_in) return FSM_ERR_INVALID_ARG;
  b->last_stream = pick_stream(b->ctx, stream);
  FSM_CUDA_TRY(cudaMemcpyAsync(b->d_mem + b->in_slab_off, host_in, b->in_slab_bytes,
                               cudaMemcpyHostToDevice, b->last_stream));
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_download(fsm_batch* b, void* host_out, void* stream) {
  if (!b || !b->own_io || !host_out) return FSM_ERR_INVALID_ARG;
  b->last_stream = pick_stream(b->ctx, stream);
  FSM_CUDA_TRY(cudaMemcpyAsync(host_out, b->d_mem + b->out_slab_off, b->out_slab_bytes,
                               cudaMemcpyDeviceToHost, b->last_stream));
  return FSM_OK;
}

extern "C" fsm_status fsm_batch_check(fsm_batch* b) {
  if (!b) return FSM_ERR_INVALID_ARG;
  return check_kernel_errors(b);
}

// ============================================================ diagnostics
extern "C" fsm_status fsm_diagnostics_device(const fsm_params* p, const fsm_outputs* in,
                                             const fsm_diagnostics* out, void* stream) {
  if (!p || !in || !out || !in->e || !in->P || !in->Pi || !in->u || !in->pi)
    return FSM_ERR_INVALID_ARG;
  const long long n = (long long)p->DIM_X * p->DIM_Y * p->DIM_ETA;
  if (p->DIM_X < 1 || p->DIM_Y < 1 || p->DIM_ETA < 1 || n > (1ll << 30)) return FSM_ERR_INVALID_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int blocks = (int)((n + 255) / 256);
  fsm_diag_kernel<<<blocks, 256, 0, s>>>(p->DIM_X, p->DIM_Y, p->DIM_ETA, p->DX, p->DY, p->TAU, in->e,
                                         in->P, in->Pi, in->u, in->pi, out->R_Pi_Inv,
                                         out->R_pimunu_Inv, out->pi_dot_u, out->pi_mu_mu, out->beta,
                                         out->omega);
  FSM_CUDA_TRY(cudaGetLastError());
  return FSM_OK;
}

extern "C" fsm_status fsm_diagnostics_host(fsm_ctx* ctx, const fsm_params* p, const fsm_outputs* hin,
                                           const fsm_diagnostics* hout) {
  if (!ctx || !p || !hin || !hout || !hin->e || !hin->P || !hin->Pi || !hin->u || !hin->pi)
    return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(ctx->device));
  const size_t n = (size_t)p->DIM_X * p->DIM_Y * p->DIM_ETA;
  // inputs e P Pi u(4) pi(10), outputs 17 components
  float* d = nullptr;
  FSM_CUDA_TRY(cudaMalloc(&d, (17 + 17) * n * 4));
  cudaStream_t st = ctx->stream;
  fsm_status s = FSM_OK;
  auto up = [&](float* dst, const float* src, size_t comps) {
    if (cudaMemcpyAsync(dst, src, comps * n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
      s = FSM_ERR_CUDA;
  };
  fsm_outputs din{};
  din.e = d;
  din.P = d + n;
  din.Pi = d + 2 * n;
  din.u = d + 3 * n;
  din.pi = d + 7 * n;
  up(din.e, hin->e, 1);
  up(din.P, hin->P, 1);
  up(din.Pi, hin->Pi, 1);
  up(din.u, hin->u, 4);
  up(din.pi, hin->pi, 10);
  float* o = d + 17 * n;
  fsm_diagnostics dout{o, o + n, o + 2 * n, o + 6 * n, o + 7 * n, o + 11 * n};
  if (s == FSM_OK) s = fsm_diagnostics_device(p, &din, &dout, st);
  auto down = [&](float* dst, const float* src, size_t comps) {
    if (dst && s == FSM_OK &&
        cudaMemcpyAsync(dst, src, comps * n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      s = FSM_ERR_CUDA;
  };
  down(hout->R_Pi_Inv, dout.R_Pi_Inv, 1);
  down(hout->R_pimunu_Inv, dout.R_pimunu_Inv, 1);
  down(hout->pi_dot_u, dout.pi_dot_u, 4);
  down(hout->pi_mu_mu, dout.pi_mu_mu, 1);
  down(hout->beta, dout.beta, 4);
  down(hout->omega, dout.omega, 6);
  if (cudaStreamSynchronize(st) != cudaSuccess && s == FSM_OK) s = FSM_ERR_CUDA;
  cudaFree(d);
  if (s != FSM_OK) set_last_error(std::string("fsm_diagnostics_host: ") + cudaGetErrorString(cudaGetLastError()));
  return s;
}

// ============================================================== autotuning
extern "C" fsm_status fsm_ctx_set_tuning(fsm_ctx* ctx, const fsm_tuning* t) {
  if (!ctx || !t) return FSM_ERR_INVALID_ARG;
  const int minimum = (kTileX + 3) * (kTileY + 3) * 16;
  if (t->window_bytes < minimum || t->window_bytes > 96 * 1024) {
    set_last_error("fsm_ctx_set_tuning: window_bytes outside [" + std::to_string(minimum) + ", 98304]");
    return FSM_ERR_INVALID_ARG;
  }
  ctx->window_budget = t->window_bytes;
  // cached one-event batches were planned with the old windows
  batch_free(ctx->single_host);
  ctx->single_host = nullptr;
  batch_free(ctx->single_dev);
  ctx->single_dev = nullptr;
  return FSM_OK;
}

extern "C" fsm_status fsm_ctx_set_wait_limit(fsm_ctx* ctx, int polls) {
  if (!ctx || polls < 0) return FSM_ERR_INVALID_ARG;
  ctx->wait_polls = polls;
  // the cached one-event batches were built with the old bound
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  batch_free(ctx->single_host);
  batch_free(ctx->single_dev);
  ctx->single_host = ctx->single_dev = nullptr;
  return FSM_OK;
}

extern "C" fsm_status fsm_autotune(fsm_ctx* ctx, int n, const fsm_params* params,
                                   const float* const* host_e, const float* const* host_nB,
                                   fsm_tuning* out) {
  if (!ctx || n <= 0 || !params || !out) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(ctx->device));
  static const int cand_kb[] = {20, 24, 28, 32, 40, 48};
  const int saved = ctx->window_budget;
  double best_ms = 0.0;
  int best = saved;
  cudaStream_t st = ctx->stream;
  cudaEvent_t e0, e1;
  FSM_CUDA_TRY(cudaEventCreate(&e0));
  FSM_CUDA_TRY(cudaEventCreate(&e1));
  fsm_status status = FSM_OK;
  for (int kb : cand_kb) {
    ctx->window_budget = kb * 1024;
    fsm_batch* b = nullptr;
    fsm_status s = batch_build(ctx, n, params, host_e, nullptr, nullptr, nullptr, &b);
    if (s != FSM_OK) {
      batch_free(b);
      continue;  // e.g. too many runs for this window: not a candidate
    }
    // inputs: the caller's profiles (or zeros) in the batch's own input slab
    for (int i = 0; i < n && host_e; ++i) {
      const size_t dim = (size_t)b->plans[i].DIM;
      cudaMemcpyAsync(b->d_in_e[i], host_e[i], dim * 4, cudaMemcpyHostToDevice, st);
      if (b->plans[i].baryon && host_nB && host_nB[i])
        cudaMemcpyAsync(b->d_in_nB[i], host_nB[i], dim * 4, cudaMemcpyHostToDevice, st);
    }
    if (!host_e) cudaMemsetAsync(b->d_mem + b->in_slab_off, 0, b->in_slab_bytes, st);
    double ms = 0.0;
    for (int rep = 0; rep < 4 && s == FSM_OK; ++rep) {
      cudaEventRecord(e0, st);
      s = enqueue(b, st, false);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) s = FSM_ERR_CUDA;
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep >= 1) ms += t;  // the first launch warms up
    }
    if (s == FSM_OK) s = check_kernel_errors(b);
    batch_free(b);
    if (s != FSM_OK) {
      status = s;
      break;
    }
    ms /= 3.0;
    if (best_ms == 0.0 || ms < best_ms) {
      best_ms = ms;
      best = kb * 1024;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->window_budget = saved;
  if (status != FSM_OK) return status;
  if (best_ms == 0.0) {
    set_last_error("fsm_autotune: no candidate window could be planned");
    return FSM_ERR_INVALID_ARG;
  }
  out->window_bytes = best;
  out->ms = best_ms;
  return fsm_ctx_set_tuning(ctx, out);
}

// ====================================================== per-bucket tuning
namespace {
void drop_single_batches(fsm_ctx* ctx) {  // they were planned with the old tuning
  batch_free(ctx->single_host);
  ctx->single_host = nullptr;
  batch_free(ctx->single_dev);
  ctx->single_dev = nullptr;
}
}  // namespace

extern "C" fsm_status fsm_ctx_set_tuning_buckets(fsm_ctx* ctx, const fsm_tuning_bucket* table) {
  if (!ctx || !table) return FSM_ERR_INVALID_ARG;
  for (int k = 0; k < FSM_TUNING_BUCKETS; ++k) {
    const fsm_tuning_bucket& t = table[k];
    const bool ok = (t.window_bytes == 0 || (t.window_bytes >= (kTileX + 3) * (kTileY + 3) * 16 &&
                                             t.window_bytes <= 96 * 1024)) &&
                    (t.phi_chunk == 0 || t.phi_chunk == 16 || t.phi_chunk == 32) &&
                    (t.tile_shapes >= FSM_TILES_DEFAULT && t.tile_shapes <= FSM_TILES_SQUARE);
    if (!ok) {
      set_last_error("fsm_ctx_set_tuning_buckets: bucket " + std::to_string(k) +
                     " has a window outside [4900, 98304] bytes, a chunk other than 16 or 32"
                     " or an unknown tile_shapes value");
      return FSM_ERR_INVALID_ARG;
    }
  }
  std::copy(table, table + FSM_TUNING_BUCKETS, ctx->buckets);
  drop_single_batches(ctx);
  return FSM_OK;
}

extern "C" fsm_status fsm_autotune_buckets(fsm_ctx* ctx, int n, const fsm_params* params,
                                           const float* const* host_e, const float* const* host_nB,
                                           fsm_tuning_bucket* out) {
  if (!ctx || n <= 0 || !params || !out) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(ctx->device));
  constexpr int kPerBucket = 64;  // events timed per bucket at most
  // windows up to 40 KB: a batch sizes its shared memory by its largest
  // window, and above that one bucket would drop the whole launch to one CTA
  // per SM (measured: 48 KB in one bucket made a 512-event batch 1.5x
  // slower).  The chunk stays 16: 32 was measured past the e tolerance
  // against FP64 on a 201^2 event (1.05e-4); callers may still set it.
  static const int cand_kb[] = {24, 28, 32, 36, 40};
  static const int cand_chunk[] = {16};
  static const int cand_tiles[] = {FSM_TILES_TAIL, FSM_TILES_SQUARE};
  std::vector<int> members[FSM_TUNING_BUCKETS];
  for (int i = 0; i < n; ++i)
    if (params[i].DIM_ETA == 1) {
      auto& m = members[tuning_bucket(params[i])];
      if ((int)m.size() < kPerBucket) m.push_back(i);
    }
  fsm_tuning_bucket saved[FSM_TUNING_BUCKETS], result[FSM_TUNING_BUCKETS] = {};
  std::copy(ctx->buckets, ctx->buckets + FSM_TUNING_BUCKETS, saved);
  cudaStream_t st = ctx->stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FSM_CUDA_TRY(cudaEventCreate(&e0));
  FSM_CUDA_TRY(cudaEventCreate(&e1));
  fsm_status status = FSM_OK;
  for (int k = 0; k < FSM_TUNING_BUCKETS && status == FSM_OK; ++k) {
    const int m = (int)members[k].size();
    if (!m) continue;
    std::vector<fsm_params> ps(m);
    std::vector<const float*> he(m, nullptr), hb(m, nullptr);
    for (int j = 0; j < m; ++j) {
      ps[j] = params[members[k][j]];
      if (host_e) he[j] = host_e[members[k][j]];
      if (host_nB) hb[j] = host_nB[members[k][j]];
    }
    // narrow tail tiles are a candidate only where some event has a partial
    // last strip they would cover
    bool any_tail = false;
    for (int j = 0; j < m; ++j)
      any_tail = any_tail || y_tail_shape(ps[j].DIM_Y) >= 0 || x_tail_shape(ps[j].DIM_X) >= 0;
    fsm_tuning_bucket best{};
    for (int kb : cand_kb)
      for (int chunk : cand_chunk)
        for (int tiles : cand_tiles) {
        if (tiles == FSM_TILES_SQUARE && !any_tail) continue;
        ctx->buckets[k] = fsm_tuning_bucket{kb * 1024, chunk, 0.0, 0, tiles};
        fsm_batch* b = nullptr;
        fsm_status s = batch_build(ctx, m, ps.data(), host_e ? he.data() : nullptr, nullptr, nullptr,
                                   nullptr, &b);
        if (s != FSM_OK) {
          batch_free(b);
          continue;  // e.g. too many runs for this window: not a candidate
        }
        for (int j = 0; j < m; ++j) {
          const size_t dim = (size_t)b->plans[j].DIM;
          if (host_e && he[j]) cudaMemcpyAsync(b->d_in_e[j], he[j], dim * 4, cudaMemcpyHostToDevice, st);
          if (b->plans[j].baryon && hb[j])
            cudaMemcpyAsync(b->d_in_nB[j], hb[j], dim * 4, cudaMemcpyHostToDevice, st);
        }
        if (!host_e) cudaMemsetAsync(b->d_mem + b->in_slab_off, 0, b->in_slab_bytes, st);
        double ms = 0.0;
        for (int rep = 0; rep < 4 && s == FSM_OK; ++rep) {
          cudaEventRecord(e0, st);
          s = enqueue(b, st, false);
          cudaEventRecord(e1, st);
          if (cudaEventSynchronize(e1) != cudaSuccess) s = FSM_ERR_CUDA;
          float t = 0.f;
          cudaEventElapsedTime(&t, e0, e1);
          if (rep >= 1) ms += t;  // the first launch warms up
        }
        if (s == FSM_OK) s = check_kernel_errors(b);
        batch_free(b);
        if (s != FSM_OK) {
          status = s;
          break;
        }
        ms /= 3.0;
        if (best.ms == 0.0 || ms < best.ms) best = fsm_tuning_bucket{kb * 1024, chunk, ms, m, tiles};
        }
    result[k] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::copy(saved, saved + FSM_TUNING_BUCKETS, ctx->buckets);
  if (status != FSM_OK) return status;
  std::copy(result, result + FSM_TUNING_BUCKETS, out);
  return fsm_ctx_set_tuning_buckets(ctx, result);
}

extern "C" fsm_status fsm_tuning_save(fsm_ctx* ctx, const char* path) {
  if (!ctx || !path) return FSM_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "w");
  if (!f) {
    set_last_error(std::string("fsm_tuning_save: cannot open ") + path);
    return FSM_ERR_FILE;
  }
  std::fprintf(f, "# bucket window_bytes phi_chunk ms events tile_shapes\n");
  for (int k = 0; k < FSM_TUNING_BUCKETS; ++k) {
    const fsm_tuning_bucket& t = ctx->buckets[k];
    if (t.window_bytes > 0)
      std::fprintf(f, "%d %d %d %.6f %d %d\n", k, t.window_bytes, t.phi_chunk, t.ms, t.events,
                   t.tile_shapes);
  }
  return std::fclose(f) == 0 ? FSM_OK : FSM_ERR_FILE;
}

extern "C" fsm_status fsm_tuning_load(fsm_ctx* ctx, const char* path) {
  if (!ctx || !path) return FSM_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "r");
  if (!f) {
    set_last_error(std::string("fsm_tuning_load: cannot open ") + path);
    return FSM_ERR_FILE;
  }
  fsm_tuning_bucket table[FSM_TUNING_BUCKETS] = {};
  char line[256];
  fsm_status st = FSM_OK;
  while (std::fgets(line, sizeof(line), f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    int k = -1, w = 0, c = 0, ev = 0, tiles = FSM_TILES_DEFAULT;
    double ms = 0.0;
    // tables written before the tile_shapes column read as the default shapes
    const int got = std::sscanf(line, "%d %d %d %lf %d %d", &k, &w, &c, &ms, &ev, &tiles);
    if (got < 5 || k < 0 || k >= FSM_TUNING_BUCKETS) {
      set_last_error(std::string("fsm_tuning_load: malformed line: ") + line);
      st = FSM_ERR_INVALID_ARG;
      break;
    }
    table[k] = fsm_tuning_bucket{w, c, ms, ev, tiles};
  }
  std::fclose(f);
  if (st != FSM_OK) return st;
  return fsm_ctx_set_tuning_buckets(ctx, table);
}

// ==================================================== energy bookkeeping
extern "C" fsm_status fsm_batch_energy(fsm_batch* b, fsm_energy* out, void* stream) {
  if (!b || !out) return FSM_ERR_INVALID_ARG;
  FSM_CUDA_TRY(cudaSetDevice(b->ctx->device));
  // an E_DEP_FS batch ran its inner batch: its plans hold the run values
  const fsm_batch* pb = b->inner ? b->inner : b;
  if (!b->edep.empty() && !b->inner) {
    set_last_error("fsm_batch_energy: the batch has not been launched");
    return FSM_ERR_PENDING;
  }
  const int n = (int)b->plans.size();
  const size_t o_sums = align_up((size_t)n * sizeof(fsm::EvEnergy));
  if (!b->d_energy) {
    FSM_CUDA_TRY(cudaMalloc(&b->d_energy, o_sums + (size_t)n * 3 * sizeof(float)));
    FSM_CUDA_TRY(cudaMallocHost(&b->h_energy, (size_t)n * 3 * sizeof(float)));
  }
  std::vector<fsm::EvEnergy> ev(n);
  for (int i = 0; i < n; ++i) {
    const EventPlan& P = pb->plans[i];
    ev[i] = fsm::EvEnergy{b->d_in_e[i], b->d_out[i].T ? b->d_out[i].T : b->d_T[i], b->d_out[i].e, P.DIM,
                          P.input_fm4 ? 1 : 0, P.p.E_FREEZE};
    if (!ev[i].T00 || !ev[i].e) {
      set_last_error("fsm_batch_energy: the batch has no T or e output for event " + std::to_string(i));
      return FSM_ERR_INVALID_ARG;
    }
  }
  cudaStream_t s = pick_stream(b->ctx, stream);
  FSM_CUDA_TRY(cudaMemcpyAsync(b->d_energy, ev.data(), (size_t)n * sizeof(fsm::EvEnergy),
                               cudaMemcpyHostToDevice, s));
  fsm_energy_sums_kernel<<<n, 256, 0, s>>>(reinterpret_cast<const fsm::EvEnergy*>(b->d_energy),
                                                         n, reinterpret_cast<float*>(b->d_energy + o_sums));
  FSM_CUDA_TRY(cudaGetLastError());
  FSM_CUDA_TRY(cudaMemcpyAsync(b->h_energy, b->d_energy + o_sums, (size_t)n * 3 * sizeof(float),
                               cudaMemcpyDeviceToHost, s));
  FSM_CUDA_TRY(cudaStreamSynchronize(s));
  for (int i = 0; i < n; ++i) {
    const fsm_params& p = pb->plans[i].p;
    float before = b->h_energy[3 * i], after = b->h_energy[3 * i + 1], inside = b->h_energy[3 * i + 2];
    // volume factors as src/FreestreamMilne.cpp:351-353, 533-544
    if (p.DIM_ETA > 1) before *= (p.TAU0 * p.DX * p.DY * p.DETA);
    else before *= (p.DX * p.DY);
    if (p.DIM_ETA > 1) after *= (p.TAU * p.DX * p.DY * p.DETA);
    else after *= (p.TAU * p.DX * p.DY);
    if (p.DIM_ETA > 1) inside *= (p.TAU * p.DX * p.DY * p.DETA);
    else inside *= (p.TAU * p.DX * p.DY);
    out[i] = fsm_energy{before, after, inside, inside / after};
  }
  return FSM_OK;
}
