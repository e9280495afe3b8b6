// fsm_noalloc.cu -- a single-event 2D entry point that allocates nothing.
//
// Some callers cannot allocate device memory at the point where they run the
// free streaming: a host framework that owns every device allocation through
// its own memory pool or budget, a process that must not grow its device
// footprint after start-up, or code that runs while another component forbids
// allocation calls.  fsm_run_event_2d_noalloc serves them: it runs the same
// kernels as fsm_run_event_device on caller-owned inputs and outputs, with all
// of its scratch (spline derivatives, node array, the internal T^{mu nu}
// buffer, the per-event tables and work lists) in one file-scope device array,
// g_noalloc_scratch, of fixed size.  Because the array is a static __device__
// object, every GPU that loads this library holds it until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
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
__global__ void fsm_stream2d_kernel(const Ev2D*, const Tile2D*, int, int, Counters*, int*, int);
__global__ void fsm_landau_kernel(const EvLandau*, const CellBlock*, Counters*);
}  // namespace fsm

using namespace fsm;

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB
constexpr int kNoAllocMaxCells = 301 * 301;               // DIM_X * DIM_Y
constexpr int kNoAllocMaxPhi = 1024;                      // DIM_PHIP after the arc-length rule
// Fixed header of the scratch: the launch counters and the stream kernel's
// error words sit at the same offsets for every event, so that
// fsm_run_event_2d_noalloc_check can read them without knowing the event.
constexpr size_t kHdrCtr = 0;
constexpr size_t kHdrErr = 256;
constexpr size_t kHdrBytes = 512;

}  // namespace

// The scratch array.  Host code must not use this name as an address: on the
// host it is only a stand-in, and the device address comes from
// cudaGetSymbolAddress (see noalloc_scratch_address).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the first call on each device does the lookup).
fsm_status noalloc_scratch_address(char** out) {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return FSM_ERR_CUDA;
  }
  if (dev < 0 || dev >= 64) return FSM_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
      return FSM_ERR_CUDA;
    }
    addr[dev] = p;
  }
  *out = static_cast<char*>(addr[dev]);
  return FSM_OK;
}

struct Region {
  size_t off = kHdrBytes;
  size_t take(size_t bytes) {
    size_t o = off;
    off = (off + bytes + 255) / 256 * 256;
    return o;
  }
};

}  // namespace

extern "C" fsm_status fsm_run_event_2d_noalloc(const fsm_params* p, const float* d_e_gev,
                                               const fsm_outputs* dev_out, void* stream) {
  if (!p || !d_e_gev || !dev_out) return FSM_ERR_INVALID_ARG;
  if (p->DIM_ETA != 1 || p->BARYON != 0) {
    set_last_error("fsm_run_event_2d_noalloc handles boost-invariant events without baryons");
    return FSM_ERR_UNSUPPORTED;
  }
  if ((long long)p->DIM_X * p->DIM_Y > kNoAllocMaxCells) {
    set_last_error("fsm_run_event_2d_noalloc: DIM_X*DIM_Y above its fixed scratch limit of " +
                   std::to_string(kNoAllocMaxCells) + " cells");
    return FSM_ERR_TOO_LARGE;
  }
  EventPlan P;
  std::string why;
  fsm_status st = plan_event(*p, nullptr, &P, &why);
  if (st != FSM_OK) {
    set_last_error(why);
    return st;
  }
  if (P.p.DIM_PHIP > kNoAllocMaxPhi) {
    set_last_error("fsm_run_event_2d_noalloc: DIM_PHIP " + std::to_string(P.p.DIM_PHIP) +
                   " above its fixed scratch limit of " + std::to_string(kNoAllocMaxPhi));
    return FSM_ERR_TOO_LARGE;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  {
    // the call uploads its tables from host memory that is gone when it
    // returns, so a graph replaying the upload would read freed memory
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
      set_last_error("fsm_run_event_2d_noalloc: cudaStreamIsCapturing failed");
      return FSM_ERR_CUDA;
    }
    if (cap != cudaStreamCaptureStatusNone) {
      set_last_error("fsm_run_event_2d_noalloc cannot be captured into a CUDA graph");
      return FSM_ERR_UNSUPPORTED;
    }
  }
  char* D = nullptr;
  if ((st = noalloc_scratch_address(&D)) != FSM_OK) return st;
  const int NX = P.p.DIM_X, NY = P.p.DIM_Y, DIM = P.DIM;

  // work lists (as the batch path builds them for one event)
  // one event of at most kNoAllocMaxCells cells has fewer 32 x 32 tiles than
  // the GPU has SMs: square tiles (see tiles_2d)
  std::vector<Tile2D> tiles;
  tiles_2d(P, 0, tiles, true);
  std::vector<LineBlock> rows, cols;
  const bool strip = NX <= kMaxStrip && NY <= kMaxStrip;
  if (strip) {
    for (int x = 0; x < NX; x += 32) rows.push_back(LineBlock{0, x, 0});
    for (int y = 0; y < NY; y += 32) cols.push_back(LineBlock{0, y, 0});
  } else {
    for (int x = 0; x < NX; x += kPrepRows) rows.push_back(LineBlock{0, x, 0});
    for (int y = 0; y < NY; y += 32)
      for (int g = 0; g < (NX + kSegP - 1) / kSegP; g += 4) cols.push_back(LineBlock{0, y, g});
  }
  std::vector<CellBlock> bl;
  for (int b = 0; b < DIM; b += kThreadsLandau) bl.push_back(CellBlock{0, b});

  // scratch layout: the fixed header (counters, error words), the uploaded
  // part, then the device-written scratch
  Region R;
  const size_t o_cs = R.take(P.cs.size() * sizeof(FSM_FLOAT2));
  const size_t o_tab = R.take(P.tab2.size() * sizeof(PhiEntry2D));
  const size_t o_chunks = R.take(P.chunks2.size() * sizeof(Chunk2D));
  const size_t o_axx = R.take(P.axx.size() * sizeof(AxisNode));
  const size_t o_axy = R.take(P.axy.size() * sizeof(AxisNode));
  const size_t o_ev2 = R.take(sizeof(Ev2D)), o_evl = R.take(sizeof(EvLandau));
  const size_t o_tiles = R.take(tiles.size() * sizeof(Tile2D));
  const size_t o_rows = R.take(rows.size() * sizeof(LineBlock));
  const size_t o_cols = R.take(cols.size() * sizeof(LineBlock));
  const size_t o_bl = R.take(bl.size() * sizeof(CellBlock));
  const size_t o_up = kHdrBytes, upload_bytes = R.off - o_up;
  const size_t o_ctr = kHdrCtr, o_err = kHdrErr;
  const size_t o_fa = R.take((size_t)DIM * 4), o_sy = R.take((size_t)DIM * 4);
  const size_t o_nodes = R.take((size_t)DIM * 16);
  const size_t o_T = R.take((size_t)DIM * 10 * 4);
  if (R.off > kNoAllocScratchBytes) {
    set_last_error("fsm_run_event_2d_noalloc: event needs " + std::to_string(R.off) +
                   " scratch bytes, above the fixed " + std::to_string(kNoAllocScratchBytes));
    return FSM_ERR_TOO_LARGE;
  }

  // descriptors (the same fields the batch path fills)
  Ev2D e{};
  e.NX = NX;
  e.NY = NY;
  e.NPHI = P.p.DIM_PHIP;
  e.NR = P.p.DIM_RAP;
  e.DX = P.p.DX;
  e.DY = P.p.DY;
  e.DTAU = P.p.DTAU;
  e.TAU = P.p.TAU;
  e.xmin = P.xmin;
  e.ymin = P.ymin;
  e.xmax_i = P.xmax_i;
  e.ymax_i = P.ymax_i;
  e.d_phip = P.d_phip;
  e.tab = reinterpret_cast<const PhiEntry2D*>(D + o_tab);
  e.chunks = reinterpret_cast<const Chunk2D*>(D + o_chunks);
  for (int sh = 0; sh < kShapes2D; ++sh) {
    e.choff[sh] = P.choff[sh];
    e.nch[sh] = P.nch[sh];
  }
  e.e_gev = d_e_gev;
  e.ax = reinterpret_cast<const AxisNode*>(D + o_axx) + kPadLo;
  e.ay = reinterpret_cast<const AxisNode*>(D + o_axy) + kPadLo;
  e.fa = reinterpret_cast<float*>(D + o_fa);
  e.sy = reinterpret_cast<float*>(D + o_sy);
  e.nodes = reinterpret_cast<FSM_FLOAT4*>(D + o_nodes);
  e.T = dev_out->T ? dev_out->T : reinterpret_cast<float*>(D + o_T);
  e.charge = 0;
  e.fb_scale = 1.0f;
  e.chunk = kPhiChunk;
  EvLandau l{};
  l.DIM = DIM;
  l.is3d = 0;
  l.baryon = 0;
  l.eos = P.p.EOS_TYPE;
  l.viscous = P.p.VISCOUS_MATCHING;
  l.TAU = P.p.TAU;
  l.T = e.T;
  l.J = nullptr;
  l.e = dev_out->e;
  l.P = dev_out->P;
  l.Pi = dev_out->Pi;
  l.u = dev_out->u;
  l.pi = dev_out->pi;

  // host image of the uploaded part (ordinary host memory; no pinned staging)
  std::vector<char> H(upload_bytes, 0);
  auto put = [&](size_t off, const void* src, size_t n) {
    if (n) std::memcpy(H.data() + (off - o_up), src, n);
  };
  put(o_cs, P.cs.data(), P.cs.size() * sizeof(FSM_FLOAT2));
  put(o_tab, P.tab2.data(), P.tab2.size() * sizeof(PhiEntry2D));
  put(o_chunks, P.chunks2.data(), P.chunks2.size() * sizeof(Chunk2D));
  put(o_axx, P.axx.data(), P.axx.size() * sizeof(AxisNode));
  put(o_axy, P.axy.data(), P.axy.size() * sizeof(AxisNode));
  put(o_ev2, &e, sizeof(e));
  put(o_evl, &l, sizeof(l));
  put(o_tiles, tiles.data(), tiles.size() * sizeof(Tile2D));
  put(o_rows, rows.data(), rows.size() * sizeof(LineBlock));
  put(o_cols, cols.data(), cols.size() * sizeof(LineBlock));
  put(o_bl, bl.data(), bl.size() * sizeof(CellBlock));

  // launch geometry of the stream kernel (as the batch path computes it); the
  // dynamic shared-memory limits go through the library's one raise-only
  // helper, so that no caller ever lowers a limit another launch relies on
  auto cu = [&](cudaError_t ce, const char* what) -> fsm_status {
    if (ce == cudaSuccess) return FSM_OK;
    set_last_error(std::string(what) + ": " + cudaGetErrorString(ce));
    return FSM_ERR_CUDA;
  };
  int dev = 0, sms = 0, occ = 0;
  if ((st = cu(cudaGetDevice(&dev), "cudaGetDevice")) != FSM_OK) return st;
  const int slot = dev & 63;
  const int box_cap = (P.box_elems + 7) & ~7;
  const size_t smem2 = stream2d_smem(box_cap);
  if ((st = rt::ensure_dyn_smem((const void*)fsm_stream2d_kernel, dev, smem2, &rt::g_smem2[slot])) != FSM_OK)
    return st;
  const size_t smem_rows = strip ? prep_strip_smem(std::max(NX, NY)) : prep_rows_smem(NY);
  if (strip) {
    if ((st = rt::ensure_dyn_smem((const void*)fsm_prep2d_rows_kernel, dev, smem_rows,
                                  &rt::g_smem_srows[slot])) != FSM_OK)
      return st;
    if ((st = rt::ensure_dyn_smem((const void*)fsm_prep2d_cols_kernel, dev, smem_rows,
                                  &rt::g_smem_scols[slot])) != FSM_OK)
      return st;
  } else if ((st = rt::ensure_dyn_smem((const void*)fsm_prep2d_rows_long_kernel, dev, smem_rows,
                                       &rt::g_smem_rows[slot])) != FSM_OK) {
    return st;
  }
  if ((st = cu(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute")) !=
      FSM_OK)
    return st;
  if ((st = cu(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fsm_stream2d_kernel, kThreads2D, smem2),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor")) != FSM_OK)
    return st;
  if (sms <= 0 || occ <= 0) {
    set_last_error("fsm_run_event_2d_noalloc: the stream kernel cannot be resident on this device");
    return FSM_ERR_CUDA;
  }
  const int ntiles = (int)tiles.size();
  const int grid2 = std::max(1, std::min(ntiles, sms * occ));

  // upload (pageable source: returns once the bytes are staged), reset the
  // counters this call reads, then the same launch sequence as the batch path
  if ((st = cu(cudaMemcpyAsync(D + o_up, H.data(), upload_bytes, cudaMemcpyHostToDevice, s), "upload")) !=
      FSM_OK)
    return st;
  if ((st = cu(cudaMemsetAsync(D + o_ctr, 0, sizeof(Counters), s), "memset")) != FSM_OK) return st;
  if ((st = cu(cudaMemsetAsync(D + o_err, 0, 4 * sizeof(int), s), "memset")) != FSM_OK) return st;
  const Ev2D* d_ev2 = reinterpret_cast<const Ev2D*>(D + o_ev2);
  const LineBlock* d_rows = reinterpret_cast<const LineBlock*>(D + o_rows);
  const LineBlock* d_cols = reinterpret_cast<const LineBlock*>(D + o_cols);
  if (strip) {
    fsm_prep2d_rows_kernel<<<(int)rows.size(), kPrepThreads, smem_rows, s>>>(d_ev2, d_rows);
    fsm_prep2d_cols_kernel<<<(int)cols.size(), kPrepThreads, smem_rows, s>>>(d_ev2, d_cols);
  } else {
    fsm_prep2d_rows_long_kernel<<<(int)rows.size(), kPrepRows * 32, smem_rows, s>>>(d_ev2, d_rows, NY);
    fsm_prep2d_cols_long_kernel<<<(int)cols.size(), 128, 0, s>>>(d_ev2, d_cols);
  }
  fsm_stream2d_kernel<<<grid2, kThreads2D, smem2, s>>>(d_ev2, reinterpret_cast<const Tile2D*>(D + o_tiles), ntiles,
                                                       box_cap, reinterpret_cast<Counters*>(D + o_ctr),
                                                       reinterpret_cast<int*>(D + o_err), kWaitPolls);
  fsm_landau_kernel<<<(int)bl.size(), kThreadsLandau, 0, s>>>(reinterpret_cast<const EvLandau*>(D + o_evl),
                                                            reinterpret_cast<const CellBlock*>(D + o_bl),
                                                            reinterpret_cast<Counters*>(D + o_ctr));
  return cu(cudaGetLastError(), "launch");
}

// Reads the error words the stream kernel of the last fsm_run_event_2d_noalloc
// call on this device left in the scratch header, after waiting for `stream`
// (the stream that call used).  The copy goes into a stack array: nothing is
// allocated.  Samples outside the staged footprint -> FSM_ERR_CUDA; a staged
// copy that did not land within the bounded wait -> FSM_ERR_TIMEOUT (the
// affected tiles were not computed, so the outputs of that call are invalid).
extern "C" fsm_status fsm_run_event_2d_noalloc_check(void* stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int err[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyFromSymbolAsync(err, g_noalloc_scratch, sizeof(err), kHdrErr,
                                            cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_last_error(std::string("fsm_run_event_2d_noalloc_check: ") + cudaGetErrorString(e));
    return FSM_ERR_CUDA;
  }
  if (err[0]) {
    set_last_error("fsm_run_event_2d_noalloc: " + std::to_string(err[0]) +
                   " samples fell outside the staged footprint");
    return FSM_ERR_CUDA;
  }
  if (err[1]) {
    set_last_error("fsm_run_event_2d_noalloc: " + std::to_string(err[1]) +
                   " staged copies did not complete within the bounded wait");
    return FSM_ERR_TIMEOUT;
  }
  return FSM_OK;
}
