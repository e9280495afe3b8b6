/* fsm.h -- C ABI of the B200 free-streaming + Landau-matching library (libfsm.so).
 *
 * This is the drop-in boundary for the hot path of freestream-milne's
 * FREESTREAMMILNE class (reference src/FreestreamMilne.cpp:28-136).  Every entry
 * point takes plain pointers and sizes; CUDA streams are passed as `void*`
 * (a cudaStream_t, NULL = the context's own stream).  Device work runs on one
 * GPU with hand-written sm_100a kernels; there is no CPU fallback: every
 * compute entry point returns FSM_ERR_NO_DEVICE when no GPU is present.
 *
 * Array conventions (identical to the reference):
 *   cell index  is = (DIM_Y*DIM_ETA)*ix + DIM_ETA*iy + ieta
 *               (src/FreeStream.cpp:23-25, FileIO.cpp:132)
 *   tensors are component-major: T[c*DIM + is], components in the order
 *   tt tx ty tn xx xy xn yy yn nn (src/LandauMatch.cpp:46-55), vectors t x y n.
 *   Units: inputs e in GeV/fm^3 as initialize_from_vector takes them
 *   (src/FreestreamMilne.cpp:43-46); nB as the IC_BARYON=3 file gives it
 *   (read by src/FileIO.cpp:133-164, no conversion); float outputs are in the
 *   reference's internal units (fm^-4, fm^-3) -- the compat class applies the
 *   hbar*c factor of src/FreestreamMilne.cpp:700-716 when filling its vectors.
 */
#ifndef FSM_H_
#define FSM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes replace the reference's printf+return / exit() paths. */
typedef enum fsm_status {
  FSM_OK = 0,
  FSM_ERR_INVALID_ARG = 1,   /* NULL pointer, non-positive size, malformed params   */
  FSM_ERR_SIZE_MISMATCH = 2, /* input length != DIM: reference exit(-1), FreestreamMilne.cpp:259-264 */
  FSM_ERR_INVALID_IC = 3,    /* unknown IC_ENERGY/IC_BARYON: FreestreamMilne.cpp:277-281,302-306 */
  FSM_ERR_UNSUPPORTED = 4,   /* parameter combination outside the implemented path  */
  FSM_ERR_CUDA = 5,          /* a CUDA runtime call failed (see fsm_last_error)     */
  FSM_ERR_NO_DEVICE = 6,     /* no CUDA device: there is no CPU fallback            */
  FSM_ERR_OUT_OF_MEMORY = 7, /* device allocation failed                            */
  FSM_ERR_FILE = 8,          /* params/IC file missing: FileIO.cpp:150-154,178-181  */
  FSM_ERR_BUSY = 9,          /* server: request does not fit the HBM budget now     */
  FSM_ERR_TIMEOUT = 10,      /* a bounded wait ran out                              */
  FSM_ERR_PENDING = 11,      /* server: request admitted, result not ready yet      */
  FSM_ERR_TOO_LARGE = 12,    /* request can never fit (budget / fixed limits)       */
  FSM_ERR_CANCELLED = 13     /* server stopped before the request ran               */
} fsm_status;

const char* fsm_status_str(fsm_status s);
/* Human-readable detail of the last error raised on the calling thread. */
const char* fsm_last_error(void);

/* Parameters: same fields, order and meaning as `struct parameters`
 * (src/Parameter.h:2-33).  DIM and TAU are derived (FreestreamMilne.cpp:177-178). */
typedef struct fsm_params {
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
} fsm_params;

/* Defaults of src/FreestreamMilne.cpp:149-171 (E_R, TAU_R, ALPHA: 1, 1, 0). */
void fsm_params_default(fsm_params* p);
/* Positional parse of a freestream_input file (src/FileIO.cpp:166-245): 26
 * "KEY<ws>value" lines in fixed order, the key text is ignored.  A missing
 * file returns FSM_ERR_FILE and leaves *p untouched (the reference prints and
 * keeps its defaults, FileIO.cpp:178-181). */
fsm_status fsm_params_read_file(const char* path, fsm_params* p);
/* Fills DIM and TAU (FreestreamMilne.cpp:177-178). */
void fsm_params_derive(fsm_params* p);

/* ------------------------------------------------------------------ context */
typedef struct fsm_ctx fsm_ctx;

typedef struct fsm_ctx_opts {
  int device;          /* CUDA device ordinal                                    */
  int enable_timing;   /* record CUDA events around every kernel (fsm_ctx_timing) */
} fsm_ctx_opts;

fsm_status fsm_ctx_create(fsm_ctx** ctx, const fsm_ctx_opts* opts /* NULL = defaults */);
/* Number of visible CUDA devices (0 when there is none or no driver); no
 * counterpart in the reference, which has no device. */
fsm_status fsm_device_count(int* n);
void fsm_ctx_destroy(fsm_ctx* ctx);

/* Accumulated device time per kernel family since the last reset, measured
 * with CUDA events on the launching stream (enable_timing must be set). */
typedef struct fsm_timing {
  double prep_ms;      /* input conversion + spline node construction          */
  double stream_ms;    /* fused free-streaming + moment quadrature             */
  double landau_ms;    /* Landau matching + EoS + viscous/baryon decomposition */
  long long prep_launches, stream_launches, landau_launches;
  double stream_samples; /* cell x momentum samples processed by stream launches */
} fsm_timing;
fsm_status fsm_ctx_timing(fsm_ctx* ctx, fsm_timing* t, int reset);

/* --------------------------------------------------------------- outputs */
/* Output views; host pointers for fsm_run_event, device pointers for the
 * *_device entry points.  Any pointer may be NULL to skip that output. */
typedef struct fsm_outputs {
  float* T;   /* 10*DIM  T^{mu nu}                                            */
  float* J;   /* 4*DIM   J^mu (BARYON)                                        */
  float* e;   /* DIM     energy density                                       */
  float* P;   /* DIM     pressure                                             */
  float* Pi;  /* DIM     bulk pressure                                        */
  float* u;   /* 4*DIM   flow velocity u^mu                                   */
  float* pi;  /* 10*DIM  shear stress pi^{mu nu}                              */
  float* nB;  /* DIM     baryon density (BARYON)                              */
  float* V;   /* 4*DIM   baryon diffusion V^mu (BARYON)                        */
} fsm_outputs;

/* Effective run values (after E_DEP_FS and the phi_p rule of
 * src/FreestreamMilne.cpp:316-332); n_fallback counts cells where Landau
 * matching found no acceptable eigenvector (LandauMatch.cpp:283-291). */
typedef struct fsm_run_info {
  int dim_phip;
  float dtau;
  float tau;   /* tau_LandauMatch (FreestreamMilne.cpp:326) */
  int live_rap_lo, live_rap_hi; /* 3D: rapidity nodes that can reach the grid */
  double samples;               /* cell x momentum samples evaluated            */
} fsm_run_info;

/* ------------------------------------------------------------ plain path */
/* One event, host buffers in and out (replaces run_freestream_milne's
 * compute, src/FreestreamMilne.cpp:251-506).  Synchronous. */
fsm_status fsm_run_event(fsm_ctx* ctx, const fsm_params* p, const float* e_gev,
                         const float* nB, const fsm_outputs* host_out, fsm_run_info* info);

/* One event on device-resident buffers, enqueued on `stream`; returns without
 * synchronising, except with E_DEP_FS = 1: the free-streaming time depends on
 * the profile, so its sums (src/FreeStream.cpp:389-417) are taken on the
 * device and read back before the event is planned. */
fsm_status fsm_run_event_device(fsm_ctx* ctx, const fsm_params* p, const float* d_e_gev,
                                const float* d_nB, const fsm_outputs* dev_out, void* stream,
                                fsm_run_info* info);

/* --------------------------------------------------------------- batches */
/* Many 2D/3D events of uneven size in one persistent launch per kernel family,
 * captured into a CUDA graph on first launch.  The batch owns device input
 * and output slabs; per-event views come from fsm_batch_views.
 * Events with E_DEP_FS = 1 (free-streaming time from the profile,
 * src/FreeStream.cpp:389-417, src/FreestreamMilne.cpp:316-332) are planned at
 * launch: each fsm_batch_launch of such a batch first sums every such event's
 * uploaded profile on the device (one launch, in the reference's order, so
 * DTAU is bit-identical to the reference's) and synchronises the stream once,
 * then runs the batch planned with those DTAUs (re-planned only when one
 * changes).  fsm_batch_info reports their run values after the first launch
 * (FSM_ERR_PENDING before). */
typedef struct fsm_batch fsm_batch;

fsm_status fsm_batch_create(fsm_ctx* ctx, int n_events, const fsm_params* params,
                            fsm_batch** batch);
/* As fsm_batch_create; grouped_outputs != 0 lays the output slab out group by
 * group (all events' T, then all events' e, ... in FSM_OUT_* order, events in
 * batch order inside a group) so that a caller can copy back only the groups
 * it reads with fsm_batch_download_groups.  fsm_batch_event_offsets then
 * reports (size_t)-1 as the output offset; use fsm_batch_group_offset. */
fsm_status fsm_batch_create_ex(fsm_ctx* ctx, int n_events, const fsm_params* params,
                               int grouped_outputs, fsm_batch** batch);
void fsm_batch_destroy(fsm_batch* b);
/* Device views of event `ev`: input slots (d_e, d_nB) and outputs. */
fsm_status fsm_batch_views(fsm_batch* b, int ev, float** d_e, float** d_nB,
                           fsm_outputs* dev_out);
/* Enqueue the whole batch on `stream` (graph replay after the first call). */
fsm_status fsm_batch_launch(fsm_batch* b, void* stream);
/* Host round trip: copy every event's input from host, launch, copy the
 * outputs named in host_out[ev] back, synchronise.  nB may be NULL. */
fsm_status fsm_batch_run_host(fsm_batch* b, const float* const* e_gev, const float* const* nB,
                              const fsm_outputs* host_out, void* stream);
fsm_status fsm_batch_info(fsm_batch* b, int ev, fsm_run_info* info);
/* Slab interface: the batch keeps every event's inputs in one contiguous
 * device slab (per event: e[DIM] then nB[DIM] when BARYON) and every event's
 * outputs in another (per event: T(10) e P Pi u(4) pi(10), then J(4) nB V(4)
 * when BARYON; each component DIM floats).  Offsets are in floats. */
fsm_status fsm_batch_slabs(fsm_batch* b, size_t* in_bytes, size_t* out_bytes);
fsm_status fsm_batch_event_offsets(fsm_batch* b, int ev, size_t* in_elem, size_t* out_elem);
/* One host->device copy of the whole input slab / device->host copy of the
 * whole output slab, enqueued on `stream` (pinned host memory makes them async). */
fsm_status fsm_batch_upload(fsm_batch* b, const void* host_in, void* stream);
fsm_status fsm_batch_download(fsm_batch* b, void* host_out, void* stream);
/* Grouped batches only: copies the groups in `mask` (an OR of FSM_OUT_*
 * values, defined below) back to host_out, packed in group order, one copy per
 * group.  Bytes written: fsm_batch_groups_bytes(b, mask).  Offset (in floats)
 * of event ev's part of group g (FSM_OUT_* == 1 << g) inside that packed
 * buffer: fsm_batch_group_offset. */
fsm_status fsm_batch_download_groups(fsm_batch* b, unsigned mask, void* host_out, void* stream);
size_t fsm_batch_groups_bytes(fsm_batch* b, unsigned mask);
fsm_status fsm_batch_group_offset(fsm_batch* b, unsigned mask, int group, int ev, size_t* elem);
/* Packed copy of the fields a caller reads, for either slab layout: the groups
 * in `mask` one after the other, events in batch order, components in order,
 * gathered on the device into one buffer and copied to host_out with one
 * device->host copy on `stream`.  flags FSM_PACK_SKIP_ETA leaves out the
 * components of boost-invariant (DIM_ETA = 1) events that vanish by symmetry:
 * T^{tau eta}, T^{x eta}, T^{y eta}, T^{eta eta}, u^eta, pi^{tau eta},
 * pi^{x eta}, pi^{y eta}, J^eta, V^eta (pi^{eta eta} does not vanish and is
 * kept).  The first call for a (mask, flags) pair allocates the device copy
 * list and the staging buffer.  Offsets are in floats; a left-out component
 * has none (FSM_ERR_INVALID_ARG). */
enum { FSM_PACK_SKIP_ETA = 1 };
fsm_status fsm_batch_download_packed(fsm_batch* b, unsigned mask, unsigned flags, void* host_out,
                                     void* stream);
size_t fsm_batch_packed_bytes(fsm_batch* b, unsigned mask, unsigned flags);
fsm_status fsm_batch_packed_offset(fsm_batch* b, unsigned mask, unsigned flags, int group, int comp,
                                   int ev, size_t* elem);
/* All offsets at once: elems[(ev * 9 + g) * 10 + c] for event ev, group g
 * (FSM_OUT_* == 1 << g) and component c, (size_t)-1 where the packed buffer
 * has none; n >= n_events * 90. */
fsm_status fsm_batch_packed_offsets(fsm_batch* b, unsigned mask, unsigned flags, size_t* elems,
                                    size_t n);
/* Waits for the stream the batch last used (upload, launch or download) and
 * checks the kernels' internal error counters. */
fsm_status fsm_batch_check(fsm_batch* b);
/* The reference's energy bookkeeping per event of the last launch
 * (src/FreestreamMilne.cpp:349-354, 531-545): total energy on the grid before
 * streaming (the initial profile in fm^-4 times DX DY, times TAU0 DETA in 3D),
 * after streaming (T^{tau tau} times TAU DX DY [DETA]), the part of it in
 * cells with e hbar*c > E_FREEZE, and that fraction; the running float sums
 * are taken on the device in the reference's cell order (one thread per
 * event, all events in one launch), so they equal the reference's.  Enqueued
 * on `stream` after the launch and waited for; out has one entry per event. */
typedef struct fsm_energy {
  float before, after, inside, fraction;
} fsm_energy;
fsm_status fsm_batch_energy(fsm_batch* b, fsm_energy* out, void* stream);
/* Total cell x momentum samples of one launch of the batch. */
double fsm_batch_samples(fsm_batch* b);

/* --------------------------------------------------------- no allocation */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory when they run the free streaming (a framework that owns all device
 * memory through its own pool or budget, or code running where allocation
 * calls are not allowed): one boost-invariant event (DIM_ETA = 1, BARYON = 0,
 * E_DEP_FS = 0) on caller-owned device input and outputs, enqueued on
 * `stream`, calling no cudaMalloc/cudaFree or other allocating routine.  Its
 * scratch lives in one fixed 8 MiB file-scope device array that every GPU
 * loading the library holds until the process exits; limits: DIM_X*DIM_Y <=
 * 90601 (e.g. 301 x 301) and DIM_PHIP <= 1024 after the arc-length rule, larger
 * events return FSM_ERR_TOO_LARGE.  The call cannot be captured into a CUDA
 * graph (it uploads its tables from host memory that is released when it
 * returns): on a capturing stream it returns FSM_ERR_UNSUPPORTED.
 * All calls share the array, so calls that overlap on the GPU race: run them in
 * one stream or serialise them.  The call returns once its work is enqueued;
 * the outputs are valid once fsm_run_event_2d_noalloc_check returns FSM_OK. */
fsm_status fsm_run_event_2d_noalloc(const fsm_params* p, const float* d_e_gev,
                                    const fsm_outputs* dev_out, void* stream);
/* No counterpart in the reference.  Waits for `stream` and reports the
 * kernel-side errors of the last fsm_run_event_2d_noalloc call on the current
 * device, read from the fixed header of the same scratch array into host
 * stack memory (no allocation): FSM_ERR_TIMEOUT when a staged copy did not
 * land within its bounded wait (some tiles were not computed), FSM_ERR_CUDA
 * when samples fell outside the staged footprint. */
fsm_status fsm_run_event_2d_noalloc_check(void* stream);

/* ------------------------------------------------------------- autotuning */
/* Launch-shape tuning of a context (no counterpart in the reference).  The 2D
 * stream kernel stages, per output tile, one source window per run of
 * consecutive phi_p; window_bytes bounds a window (larger windows: fewer runs
 * and barriers, more shared memory per block and possibly fewer blocks per
 * SM).  fsm_autotune times the full launch sequence of the given events for a
 * set of candidate sizes, keeps the fastest for every later batch and event of
 * ctx and returns it; the result can be stored and restored with
 * fsm_ctx_set_tuning.  host_e / host_nB may be NULL (zero profiles). */
typedef struct fsm_tuning {
  int window_bytes;  /* staged window bound of a 2D phi_p run (default 32768)   */
  double ms;         /* measured launch-sequence time with it (fsm_autotune)    */
} fsm_tuning;
fsm_status fsm_autotune(fsm_ctx* ctx, int n, const fsm_params* params, const float* const* host_e,
                        const float* const* host_nB, fsm_tuning* out);
fsm_status fsm_ctx_set_tuning(fsm_ctx* ctx, const fsm_tuning* t);

/* Per-bucket tuning of boost-invariant events.  An event's bucket is
 * side_class * 4 + shift_class, side_class from max(DIM_X, DIM_Y) (0: < 128,
 * 1: < 192, 2: < 256, 3: larger) and shift_class from the shift length in
 * cells DTAU / min(DX, DY) (0: < 8, 1: < 16, 2: < 24, 3: larger).  Per bucket
 * the 2D stream kernel's staged-window bound, its phi_p chunk (phi_p per
 * FP32 partial sum of the two-level moment sum: 16, or 32 -- about 2 % faster
 * and with a larger summation error: e against FP64 reached 1.05e-4 on a 201^2
 * event, so the tuner keeps 16) and its output tile shapes: 32 x 32 tiles
 * everywhere, or narrow tiles (64 x 16, 128 x 8 along a last partial y strip
 * of at most 16 / 8 cells; 16 x 64, 8 x 128 along such an x strip) so that
 * fewer lanes and warps run past the grid edge.  fsm_autotune_buckets times,
 * for every bucket the given events fall in, the launch sequence of those
 * events (at most 64 of them) for windows of 24-40 KB (larger windows would
 * lower the occupancy of every batch holding such an event) with and without
 * the narrow tiles, keeps the fastest per bucket for ctx and writes the
 * FSM_TUNING_BUCKETS entries (window_bytes 0 for buckets without events: they
 * keep the context's window, chunk 16 and narrow tail tiles).  The table can
 * be stored and restored as text with fsm_tuning_save / fsm_tuning_load (one
 * "bucket window_bytes phi_chunk ms events tile_shapes" line per tuned
 * bucket).  Results do not depend on the window or the tile shapes. */
#define FSM_TUNING_BUCKETS 16
enum {
  FSM_TILES_DEFAULT = 0, /* narrow tiles on partial last strips              */
  FSM_TILES_TAIL = 1,    /* the same, chosen by the tuner                    */
  FSM_TILES_SQUARE = 2   /* 32 x 32 tiles only                               */
};
typedef struct fsm_tuning_bucket {
  int window_bytes;  /* staged window bound (0: the context's)               */
  int phi_chunk;     /* 16 or 32 (0: 16)                                       */
  double ms;         /* measured launch-sequence time of the bucket's events   */
  int events;        /* events the measurement used                            */
  int tile_shapes;   /* FSM_TILES_*                                            */
} fsm_tuning_bucket;
fsm_status fsm_autotune_buckets(fsm_ctx* ctx, int n, const fsm_params* params,
                                const float* const* host_e, const float* const* host_nB,
                                fsm_tuning_bucket* out);
fsm_status fsm_ctx_set_tuning_buckets(fsm_ctx* ctx, const fsm_tuning_bucket* table);
fsm_status fsm_tuning_save(fsm_ctx* ctx, const char* path);
fsm_status fsm_tuning_load(fsm_ctx* ctx, const char* path);

/* Polls of one bounded wait on a staged copy in the 2D stream kernel for the
 * batches (and one-event batches) of ctx built after the call; default 1 << 20,
 * 0 makes every such wait give up at once.  No counterpart in the reference,
 * whose CPU loops have nothing to wait on: it exists so that the time-out path
 * (FSM_ERR_TIMEOUT from fsm_batch_check, the context staying usable) can be
 * exercised without a fault.  After a time-out the kernel always waits, with
 * the default bound, for the copies it has in flight before it exits. */
fsm_status fsm_ctx_set_wait_limit(fsm_ctx* ctx, int polls);

/* ---------------------------------------------------------- request server */
/* No counterpart in the reference, which computes one event per call.  A
 * continuous-batching server: fsm_server_submit queues one event (host
 * buffers, copied in); a scheduler thread admits queued requests into launch
 * waves whenever one of its streams is idle and its device / pinned-host
 * budgets have room, so requests arriving while others run join the next
 * wave, and waves on different streams overlap on the device.  A request's
 * results are identical to fsm_run_event's on the same event.  The server's
 * functions may be called from any thread, except that fsm_server_stop must
 * not race with the others. */
typedef struct fsm_server fsm_server;

/* Output groups a server returns (fsm_server_opts.output_mask; 0 = all). */
enum {
  FSM_OUT_T = 1u << 0,     /* T^{mu nu}                 */
  FSM_OUT_E = 1u << 1,     /* e                         */
  FSM_OUT_P = 1u << 2,     /* P                         */
  FSM_OUT_BULK = 1u << 3,  /* Pi                        */
  FSM_OUT_U = 1u << 4,     /* u^mu                      */
  FSM_OUT_SHEAR = 1u << 5, /* pi^{mu nu}                */
  FSM_OUT_J = 1u << 6,     /* J^mu (baryon events)      */
  FSM_OUT_NB = 1u << 7,    /* n_B (baryon events)       */
  FSM_OUT_V = 1u << 8,     /* V^mu (baryon events)      */
  FSM_OUT_ALL = 0x1ffu
};

typedef struct fsm_server_opts {
  int device;                /* CUDA device ordinal                                 */
  size_t hbm_budget_bytes;   /* device memory held for waves in flight (0: 8 GiB)   */
  size_t host_budget_bytes;  /* pinned host memory for inputs/outputs (0: 2 GiB)    */
  int max_wave_events;       /* events per launch wave (0: 512)                     */
  int streams;               /* waves in flight (0: 4)                              */
  unsigned output_mask;      /* FSM_OUT_* groups copied back (0: all); fields of
                                fsm_server_poll's host_out outside it are left as
                                they are                                            */
  int stream_2d;             /* 1: one more stream whose waves hold boost-invariant
                                requests only, so that they never queue behind 3D
                                waves (0: none)                                     */
} fsm_server_opts;

typedef struct fsm_server_stats {
  long long submitted, completed, failed, waves;
  double p50_ms, p99_ms, max_ms;  /* latency submit -> outputs in host memory         */
  double events_per_s;            /* completed / (last completion - first submission) */
} fsm_server_stats;

/* Allocates both budgets up front (one device and one pinned allocation). */
fsm_status fsm_server_start(fsm_server** s, const fsm_server_opts* opts /* NULL = defaults */);
fsm_status fsm_server_submit(fsm_server* s, const fsm_params* p, const float* e_gev,
                             const float* nB, long long* id);
/* Waits up to timeout_ms (< 0: until done, 0: no wait).  done = 1: the request
 * finished, its outputs are copied into host_out (NULL fields skipped), it is
 * forgotten, and the return value is its own status (FSM_ERR_TOO_LARGE when it
 * cannot fit the budgets, FSM_ERR_CANCELLED when the server stopped first). */
fsm_status fsm_server_poll(fsm_server* s, long long id, const fsm_outputs* host_out,
                           fsm_run_info* info, double timeout_ms, int* done);
/* Zero-copy variant: on done = 1 the fields of `views` point at the request's
 * outputs inside the server's pinned memory (NULL for groups outside the
 * output mask), valid until fsm_server_release(s, id); the request stays
 * known until then. */
fsm_status fsm_server_poll_view(fsm_server* s, long long id, fsm_outputs* views,
                                fsm_run_info* info, double timeout_ms, int* done);
fsm_status fsm_server_release(fsm_server* s, long long id);
fsm_status fsm_server_stats_get(fsm_server* s, fsm_server_stats* st);
/* Where a server's time goes, averaged over the waves retired so far (no
 * counterpart in the reference): host time to plan a wave (tables, runs, work
 * lists) and to stage its inputs into pinned memory; device time of its input
 * copy, its kernels and its output copies (CUDA events on the wave's stream);
 * the mean time a request waited in the queue before a wave took it; and the
 * device time of all waves (copies + kernels, and kernels alone) per
 * wall-clock time from the first submission to the last completion (above 1
 * when waves on different streams overlap). */
typedef struct fsm_server_breakdown {
  long long waves;
  double events_per_wave;
  double plan_ms, stage_ms;          /* host, per wave                        */
  double h2d_ms, kernels_ms, d2h_ms; /* device, per wave                      */
  double queue_ms;                   /* per request: submit -> taken by a wave */
  double device_busy, kernel_busy;   /* device time / wall time               */
} fsm_server_breakdown;
fsm_status fsm_server_breakdown_get(fsm_server* s, fsm_server_breakdown* bd);
/* Finishes the waves in flight, cancels queued requests, frees everything. */
fsm_status fsm_server_stop(fsm_server* s);

/* ------------------------------------------------------------- diagnostics */
/* Hydro-validity and thermal-vorticity fields of Landau-matched outputs, as the
 * reference computes them before writing its *_projection / beta / w_xy files
 * (src/HydroValidity.cpp:8-101, src/LandauMatch.cpp:395-489,
 * src/FreestreamMilne.cpp:561-611).  Any field may be NULL. */
typedef struct fsm_diagnostics {
  float* R_Pi_Inv;      /* [DIM]     Pi / max(P, 1e-5)                          */
  float* R_pimunu_Inv;  /* [DIM]     sqrt|pi_{mu nu} pi^{mu nu}| / sqrt(e^2+3P^2) */
  float* pi_dot_u;      /* [4][DIM]  pi^{mu nu} u_nu                            */
  float* pi_mu_mu;      /* [DIM]     pi^mu_mu                                   */
  float* beta;          /* [4][DIM]  u_mu / T on interior (ix, iy), else 0      */
  float* omega;         /* [6][DIM]  thermal vorticity; only w_xy is non-zero   */
} fsm_diagnostics;

/* From device outputs (e, P, Pi, u, pi of fsm_outputs) on `stream`; p->TAU is
 * the Landau-matching time (fsm_run_info.tau). */
fsm_status fsm_diagnostics_device(const fsm_params* p, const fsm_outputs* dev_in,
                                  const fsm_diagnostics* dev_out, void* stream);
/* Same from host arrays (copied to the device and back; synchronous). */
fsm_status fsm_diagnostics_host(fsm_ctx* ctx, const fsm_params* p, const fsm_outputs* host_in,
                                const fsm_diagnostics* host_out);

/* ------------------------------------------------------------- text output */
/* One per-cell field in the reference's text formats (src/FileIO.cpp:11-131,
 * replacing writeScalarToFile / writeVectorToFile for one component when
 * projection = 0: "x y eta value" per cell with coordinates rounded to the
 * spacing; writeScalarToFileProjection / writeVectorToFileProjection when
 * projection = 1: the eta-centre slice, rows = y, columns = x).  Formatted by
 * nthreads host threads (0 = all hardware threads).  Unlike the reference,
 * which fails silently, an unwritable path returns FSM_ERR_FILE. */
fsm_status fsm_write_field(const char* path, const float* var, const fsm_params* p, int projection,
                           int nthreads);
/* Every per-cell file the reference writes after Landau matching
 * (src/FreestreamMilne.cpp:561-673 via src/FileIO.cpp:11-131), byte-identical,
 * into directory `dir` under the reference's file names (<dir>/e.dat,
 * <dir>/e_projection.dat, ... the reference writes them into output/): from
 * `diag` the hydro-validity projections (R_Pi_Inv, R_pimunu_Inv, pi_dot_u_*,
 * pi_mu_mu) and beta_x, beta_y, w_xy (full and projection); from `out` e, p,
 * bulk_PI, u^mu, pi^{mu nu} (full and projection) and with BARYON nB (both)
 * and V_x, V_y, V_eta.  Host arrays; NULL fields (and a NULL diag) are
 * skipped.  The files are formatted concurrently by nthreads host threads
 * (0 = all hardware threads), largest first. */
fsm_status fsm_write_outputs(const char* dir, const fsm_params* p, const fsm_outputs* out,
                             const fsm_diagnostics* diag, int nthreads);

/* ------------------------------------------------------ initial conditions */
/* The reference's initial conditions other than the caller's vector
 * (src/FreestreamMilne.cpp:225-306), as host profiles in fm^-4 -- the units
 * the reference computes with; pass them to fsm_run_event_fm4.  IC_ENERGY: 1
 * smooth elliptical Gaussian, 2 the same times a rand() draw per cell, 3 an
 * "x y eta value" file <dir>/e.dat, 4 a CPU-VH file <dir>/e.dat, 6 two
 * Gaussians times rand() draws (the reference's norm is 0: a zero profile);
 * IC_BARYON: 1, 2 as energy 1, 2 with the baryon widths, 3 <dir>/nB.dat.  dir
 * NULL: "initial_profiles" (the reference's directory).  The Monte-Carlo
 * profiles draw from the C library's rand() in the reference's order.
 * Missing files return FSM_ERR_FILE (the reference exits for IC 3 and prints
 * for IC 4); IC_ENERGY 5 and unknown values FSM_ERR_INVALID_IC. */
fsm_status fsm_initial_energy(const fsm_params* p, const char* dir, float* e_fm4);
fsm_status fsm_initial_baryon(const fsm_params* p, const char* dir, float* nB);
/* One profile file of DIM floats in fm^-4 in one of the reference's formats:
 * "x y eta value" lines (src/FileIO.cpp:133-164), CPU-VH "d d d value" lines in
 * eta, y, x order plus 1e-7 (src/InitialConditions.cpp:316-355), superMC and
 * TRENTO transverse blocks times the reference's eta plateau plus 1e-3
 * (:127-236; TRENTO skips a 12-line header, rows are y), and TRENTO 3D blocks
 * plus 1e-3 (:274-314).  The reference has these block readers but does not
 * reach them from run_freestream_milne; they are here for callers that read
 * such files. */
enum {
  FSM_PROFILE_XYEV = 0,
  FSM_PROFILE_CPUVH = 1,
  FSM_PROFILE_SUPERMC_BLOCK = 2,
  FSM_PROFILE_TRENTO_BLOCK = 3,
  FSM_PROFILE_TRENTO3D_BLOCK = 4
};
fsm_status fsm_read_profile(const char* path, const fsm_params* p, int format, float* out);
/* fsm_run_event for a profile already in fm^-4 (IC_ENERGY other than 5: the
 * reference then uses the profile as it is, src/FreestreamMilne.cpp:231-281,
 * and takes the E_DEP_FS sums over it, src/FreeStream.cpp:389-417). */
fsm_status fsm_run_event_fm4(fsm_ctx* ctx, const fsm_params* p, const float* e_fm4, const float* nB,
                             const fsm_outputs* host_out, fsm_run_info* info);

/* ------------------------------------------------------------ diagnostics */
/* Measured FP32 FMA throughput of `device` in TFLOP/s (a short FMA-chain
 * kernel timed with CUDA events): the peak the stream kernels' roofline
 * fraction is quoted against. */
fsm_status fsm_probe_fp32_tflops(int device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* FSM_H_ */
