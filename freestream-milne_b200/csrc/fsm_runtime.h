// fsm_runtime.h -- internal: context and batch objects and the batch
// build/launch functions shared by the C ABI (fsm_runtime.cu) and the request
// server (fsm_server.cu).  Not installed; the public interface is fsm.h.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <thread>
#include <string>
#include <vector>

#include "../../include/fsm.h"
#include "fsm_internal.h"
#include "fsm_plan.h"

#define FSM_CUDA_TRY(call)                                                        \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));         \
      return (e_ == cudaErrorMemoryAllocation) ? FSM_ERR_OUT_OF_MEMORY : FSM_ERR_CUDA; \
    }                                                                             \
  } while (0)

namespace fsm {
namespace rt {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v, size_t a = kAlign) { return (v + a - 1) / a * a; }

struct TimingSet {
  cudaEvent_t ev[4];
  double samples;
};

}  // namespace rt
}  // namespace fsm

using fsm::CellBlock;
using fsm::Counters;
using fsm::Ev2D;
using fsm::Ev3D;
using fsm::EvLandau;
using fsm::EventPlan;
using fsm::LineBlock;
using fsm::Tile2D;
using fsm::Tile3D;
using fsm::PhiEntry3D;
using fsm::CombW;

namespace fsm {
namespace rt {
// Output component groups of a batch's output slab, in slab order:
// T(10) e P Pi u(4) pi(10) J(4) nB V(4); J, nB and V only for baryon events.
constexpr int kOutGroups = 9;
constexpr int kOutGroupComps[kOutGroups] = {10, 1, 1, 1, 4, 10, 4, 1, 4};
}  // namespace rt
}  // namespace fsm

struct fsm_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool timing = false;
  int num_sms = 0;
  int smem_optin = 0;
  fsm_timing acc{};
  std::vector<fsm::rt::TimingSet> pending;
  std::vector<cudaEvent_t> event_pool;
  std::mutex mu;
  int window_budget = fsm::kWindowBudget2D;  // staged window of a 2D phi_p run (autotuned)
  int wait_polls = fsm::kWaitPolls;  // bounded waits of batches built from now on
  // per-bucket tuning of 2D events (window_bytes 0: the context's window)
  fsm_tuning_bucket buckets[FSM_TUNING_BUCKETS] = {};
  // energy-dependent DTAU of device profiles: sums on the device, read back
  float* d_sums = nullptr;
  float* h_sums = nullptr;
  // cached one-event batches (single_host_raw: the caller's parameters it was built for)
  fsm_batch* single_host = nullptr;
  fsm_batch* single_dev = nullptr;
  fsm_params single_host_raw{};
  bool single_host_fm4 = false;  // units the cached one-event host batch was built for
  // the device and pinned allocations of the last batch destroyed, kept for
  // the next batch that fits (a stream of event sets then allocates nothing)
  std::mutex spare_mu;
  char* spare_dev = nullptr;
  size_t spare_dev_cap = 0;
  char* spare_host = nullptr;
  size_t spare_host_cap = 0;
  // two pinned chunks and their events: copies between pageable caller
  // buffers and the device go through them, chunk by chunk, the host copy
  // of one chunk overlapping the device copy of the next
  char* pin_stage = nullptr;
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  // plans of 3D events by their parameters and tuning (a 3D plan takes
  // milliseconds of host work; its shift table is shared, not copied, by the
  // batches that use it); at most kPlanCacheEntries holding at most
  // kPlanCacheBytes of shift tables, oldest dropped first; a plan whose table
  // alone exceeds kPlanCacheMaxPlan is not kept
  std::mutex plan_mu;
  std::unordered_map<std::string, std::shared_ptr<const EventPlan>> plan_cache;
  std::vector<std::string> plan_order;
  size_t plan_bytes = 0;
};
constexpr size_t kPlanCacheEntries = 32;
constexpr size_t kPlanCacheBytes = (size_t)512 << 20;
constexpr size_t kPlanCacheMaxPlan = (size_t)64 << 20;

struct fsm_batch {
  fsm_ctx* ctx = nullptr;
  std::vector<EventPlan> plans;
  bool own_io = true;
  bool ext_mem = false;  // d_mem / h_stage belong to the caller (BatchMem)
  // device allocation
  char* d_mem = nullptr;
  size_t bytes = 0;
  size_t dev_cap = 0, host_cap = 0;  // sizes of the own allocations (may exceed the need)
  // staging for descriptor uploads (pinned)
  char* h_stage = nullptr;
  size_t stage_bytes = 0;
  size_t desc_off = 0, desc_bytes = 0;
  // per-event device views
  std::vector<float*> d_in_e, d_in_nB;
  std::vector<fsm_outputs> d_out;
  std::vector<size_t> in_off, out_off;  // element offsets inside the slabs
  // element offset of event i's component group g inside the output slab; with
  // grouped_out the slab holds group by group (all events' T, then all e, ...)
  std::vector<std::array<size_t, fsm::rt::kOutGroups>> out_goff;
  bool grouped_out = false;
  size_t group_off[fsm::rt::kOutGroups] = {}, group_elems[fsm::rt::kOutGroups] = {};
  size_t in_slab_off = 0, in_slab_bytes = 0, out_slab_off = 0, out_slab_bytes = 0;
  std::vector<float*> d_T, d_J;         // moment buffers the Landau kernel reads
  // host copies of descriptors
  std::vector<Ev2D> ev2;
  std::vector<Ev3D> ev3;
  std::vector<EvLandau> evl;
  std::vector<int> ev2_of, ev3_of;      // event -> index in ev2/ev3 (or -1)
  std::vector<int> evq_of;              // 2D baryon event -> its charge pass in ev2 (or -1)
  // device descriptor arrays and work lists
  Ev2D* d_ev2 = nullptr;
  Ev3D* d_ev3 = nullptr;
  EvLandau* d_evl = nullptr;
  Tile2D* d_tiles = nullptr;
  LineBlock *d_rows = nullptr, *d_cols = nullptr, *d_rows_l = nullptr, *d_cols_l = nullptr;
  CellBlock *d_prep3 = nullptr, *d_bl = nullptr;
  fsm::Tile3D* d_tiles3 = nullptr;
  Counters* d_ctr = nullptr;
  int* d_err = nullptr;
  int ntiles = 0, nrows = 0, ncols = 0, nrows_l = 0, ncols_l = 0, nprep3 = 0, ntiles3 = 0, nbl = 0;
  int ntiles3b = 0;  // the first ntiles3b 3D tiles belong to events with baryon charge
  int nbl2 = 0;      // the first nbl2 Landau blocks belong to boost-invariant events
  int cs_cap2 = 0, cs_cap3 = 0, box_cap2 = 0, ny_cap2 = 0, strip_cap2 = 0;
  size_t smem2 = 0, smem3 = 0, smem3b = 0, smem_rows = 0, smem_strip = 0;
  int grid2 = 0, grid3 = 0, grid3b = 0;
  int wait_polls = fsm::kWaitPolls;  // polls of one bounded wait in the stream kernel
  double samples = 0;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  cudaStream_t last_stream = nullptr;  // stream of the most recent upload/launch/download
  // packed downloads: copy list of the last (mask, flags) and the staging buffer
  unsigned pack_mask = 0, pack_flags = 0;
  bool pack_ready = false;
  fsm::CopySeg* d_segs = nullptr;
  int nsegs = 0;
  size_t seg_cap = 0;
  float* d_pack = nullptr;
  size_t pack_elems = 0, pack_cap = 0;
  // Events with E_DEP_FS = 1 (free-streaming time from the profile,
  // src/FreeStream.cpp:389-417) cannot be planned before their inputs exist.
  // Such a batch holds the slabs only; each launch takes every such event's
  // profile sums on the device (one launch, one sync), resolves DTAU, and runs
  // `inner`, a batch planned with the resolved parameters that reads and
  // writes this batch's slabs (rebuilt only when a DTAU changes).
  std::vector<int> edep;              // indices of the E_DEP_FS events
  std::vector<fsm_params> raw;        // the caller's parameters
  fsm_batch* inner = nullptr;
  std::vector<fsm_params> inner_params;
  char* d_edep = nullptr;             // device: input pointers, cell counts, sums
  float* h_sums = nullptr;            // pinned: the sums read back
  char* d_energy = nullptr;           // device: energy-bookkeeping descriptors and sums
  float* h_energy = nullptr;          // pinned: those sums read back
};

namespace fsm {
namespace rt {

// Memory for a batch supplied by its owner instead of cudaMalloc /
// cudaMallocHost (the server's pools).  dev/host return at least `bytes`
// (256-byte aligned) or nullptr when the pool is exhausted; the descriptor
// upload is then enqueued on `stream` instead of copied synchronously.  With
// dev null the batch allocates its own memory and only grouped_out applies.
struct BatchMem {
  void* user = nullptr;
  char* (*dev)(void* user, size_t bytes) = nullptr;
  char* (*host)(void* user, size_t bytes) = nullptr;
  cudaStream_t stream = nullptr;
  bool grouped_out = false;  // output slab laid out group by group
  // only the input/output slabs and the tables: no stream-kernel scratch (a
  // batch whose launches run an inner batch planned later, see fsm_batch::inner)
  bool io_only = false;
  // the energy profiles are already in fm^-4 (fsm_run_event_fm4)
  bool input_fm4 = false;
};

bool has_device();
void batch_free(fsm_batch* b);
fsm_status batch_build(fsm_ctx* ctx, int n, const fsm_params* params, const float* const* host_e,
                       const float* const* ext_in_e, const float* const* ext_in_nB,
                       const fsm_outputs* ext_out, fsm_batch** out, const BatchMem* mem = nullptr);
fsm_status enqueue(fsm_batch* b, cudaStream_t s, bool timing);
// Tuning bucket of a 2D event (grid side class x shift-length class) and the
// staged-window bound / phi_p chunk the context's tuning gives an event.
int tuning_bucket(const fsm_params& p);
void event_tuning(const fsm_ctx* ctx, const fsm_params& p, int* window, int* chunk, bool* tail);
// Raises (never lowers) a kernel's dynamic shared-memory limit: the limit is a
// process-wide attribute other launches (and captured graphs) rely on.
// `slot` records the largest value set so far for that kernel on `device`;
// every caller of the library uses the slots below, under one mutex.
fsm_status ensure_dyn_smem(const void* fn, int device, size_t bytes, int* slot);
extern int g_smem2[64], g_smem3[64], g_smem3b[64], g_smem_rows[64], g_smem_srows[64], g_smem_scols[64];
fsm_status check_kernel_errors(fsm_batch* b);
fsm_status fill_info(const EventPlan& P, fsm_run_info* info);

}  // namespace rt
}  // namespace fsm
