"""ctypes binding of libfsm.so, the C ABI declared in include/fsm.h.

This module is a thin Python mirror of the C entry points for tests and the
benchmark; the product is the C ABI itself (and the C++ FREESTREAMMILNE
compatibility class built on it).  Loading fails loudly when the library has
not been built: there is no Python or CPU fallback for the compute path.
"""
import ctypes
import os
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libfsm.so"

FSM_OK = 0
STATUS = {0: "FSM_OK", 1: "FSM_ERR_INVALID_ARG", 2: "FSM_ERR_SIZE_MISMATCH", 3: "FSM_ERR_INVALID_IC",
          4: "FSM_ERR_UNSUPPORTED", 5: "FSM_ERR_CUDA", 6: "FSM_ERR_NO_DEVICE",
          7: "FSM_ERR_OUT_OF_MEMORY", 8: "FSM_ERR_FILE", 9: "FSM_ERR_BUSY", 10: "FSM_ERR_TIMEOUT",
          11: "FSM_ERR_PENDING", 12: "FSM_ERR_TOO_LARGE", 13: "FSM_ERR_CANCELLED"}

# fsm_params (field order of the reference's struct parameters,
# src/Parameter.h:2-33), shared with the library-free workload generators
from fsm_params import PARAM_FIELDS, Params  # noqa: E402,F401


_FP = ctypes.POINTER(ctypes.c_float)


class Outputs(ctypes.Structure):
    _fields_ = [("T", ctypes.c_void_p), ("J", ctypes.c_void_p), ("e", ctypes.c_void_p),
                ("P", ctypes.c_void_p), ("Pi", ctypes.c_void_p), ("u", ctypes.c_void_p),
                ("pi", ctypes.c_void_p), ("nB", ctypes.c_void_p), ("V", ctypes.c_void_p)]


class RunInfo(ctypes.Structure):
    _fields_ = [("dim_phip", ctypes.c_int), ("dtau", ctypes.c_float), ("tau", ctypes.c_float),
                ("live_rap_lo", ctypes.c_int), ("live_rap_hi", ctypes.c_int),
                ("samples", ctypes.c_double)]


class CtxOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("enable_timing", ctypes.c_int)]


class Timing(ctypes.Structure):
    _fields_ = [("prep_ms", ctypes.c_double), ("stream_ms", ctypes.c_double),
                ("landau_ms", ctypes.c_double), ("prep_launches", ctypes.c_longlong),
                ("stream_launches", ctypes.c_longlong), ("landau_launches", ctypes.c_longlong),
                ("stream_samples", ctypes.c_double)]


# Every symbol include/fsm.h declares, with (restype, argtypes).
_VP = ctypes.c_void_p
_ST = ctypes.c_int
class Tuning(ctypes.Structure):
    _fields_ = [("window_bytes", ctypes.c_int), ("ms", ctypes.c_double)]


class Energy(ctypes.Structure):
    _fields_ = [("before", ctypes.c_float), ("after", ctypes.c_float), ("inside", ctypes.c_float),
                ("fraction", ctypes.c_float)]


class TuningBucket(ctypes.Structure):
    _fields_ = [("window_bytes", ctypes.c_int), ("phi_chunk", ctypes.c_int), ("ms", ctypes.c_double),
                ("events", ctypes.c_int), ("tile_shapes", ctypes.c_int)]


TUNING_BUCKETS = 16
TILES_DEFAULT, TILES_TAIL, TILES_SQUARE = 0, 1, 2  # FSM_TILES_*


class ServerOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t),
                ("host_budget_bytes", ctypes.c_size_t), ("max_wave_events", ctypes.c_int),
                ("streams", ctypes.c_int), ("output_mask", ctypes.c_uint), ("stream_2d", ctypes.c_int)]


# output groups of the server (FSM_OUT_* in fsm.h), in slab order
OUT_GROUPS = ["T", "e", "P", "Pi", "u", "pi", "J", "nB", "V"]
PACK_SKIP_ETA = 1  # FSM_PACK_SKIP_ETA


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("waves", ctypes.c_longlong),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("events_per_s", ctypes.c_double)]


class ServerBreakdown(ctypes.Structure):
    _fields_ = [("waves", ctypes.c_longlong), ("events_per_wave", ctypes.c_double),
                ("plan_ms", ctypes.c_double), ("stage_ms", ctypes.c_double),
                ("h2d_ms", ctypes.c_double), ("kernels_ms", ctypes.c_double),
                ("d2h_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("device_busy", ctypes.c_double), ("kernel_busy", ctypes.c_double)]


class Diagnostics(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in
                ("R_Pi_Inv", "R_pimunu_Inv", "pi_dot_u", "pi_mu_mu", "beta", "omega")]


DIAG_COMPS = {"R_Pi_Inv": 1, "R_pimunu_Inv": 1, "pi_dot_u": 4, "pi_mu_mu": 1, "beta": 4, "omega": 6}


SIGNATURES = {
    "fsm_status_str": (ctypes.c_char_p, [ctypes.c_int]),
    "fsm_last_error": (ctypes.c_char_p, []),
    "fsm_params_default": (None, [ctypes.POINTER(Params)]),
    "fsm_params_read_file": (_ST, [ctypes.c_char_p, ctypes.POINTER(Params)]),
    "fsm_params_derive": (None, [ctypes.POINTER(Params)]),
    "fsm_ctx_create": (_ST, [ctypes.POINTER(_VP), ctypes.POINTER(CtxOpts)]),
    "fsm_device_count": (_ST, [ctypes.POINTER(ctypes.c_int)]),
    "fsm_ctx_destroy": (None, [_VP]),
    "fsm_ctx_timing": (_ST, [_VP, ctypes.POINTER(Timing), ctypes.c_int]),
    "fsm_run_event": (_ST, [_VP, ctypes.POINTER(Params), _VP, _VP, ctypes.POINTER(Outputs),
                            ctypes.POINTER(RunInfo)]),
    "fsm_run_event_device": (_ST, [_VP, ctypes.POINTER(Params), _VP, _VP,
                                   ctypes.POINTER(Outputs), _VP, ctypes.POINTER(RunInfo)]),
    "fsm_batch_create": (_ST, [_VP, ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(_VP)]),
    "fsm_batch_destroy": (None, [_VP]),
    "fsm_batch_views": (_ST, [_VP, ctypes.c_int, ctypes.POINTER(_VP), ctypes.POINTER(_VP),
                              ctypes.POINTER(Outputs)]),
    "fsm_batch_launch": (_ST, [_VP, _VP]),
    "fsm_batch_run_host": (_ST, [_VP, ctypes.POINTER(_VP), ctypes.POINTER(_VP),
                                 ctypes.POINTER(Outputs), _VP]),
    "fsm_batch_info": (_ST, [_VP, ctypes.c_int, ctypes.POINTER(RunInfo)]),
    "fsm_batch_samples": (ctypes.c_double, [_VP]),
    "fsm_batch_slabs": (_ST, [_VP, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "fsm_batch_event_offsets": (_ST, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                                      ctypes.POINTER(ctypes.c_size_t)]),
    "fsm_batch_upload": (_ST, [_VP, _VP, _VP]),
    "fsm_batch_download": (_ST, [_VP, _VP, _VP]),
    "fsm_batch_create_ex": (_ST, [_VP, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int,
                                  ctypes.POINTER(_VP)]),
    "fsm_batch_download_groups": (_ST, [_VP, ctypes.c_uint, _VP, _VP]),
    "fsm_batch_groups_bytes": (ctypes.c_size_t, [_VP, ctypes.c_uint]),
    "fsm_batch_group_offset": (_ST, [_VP, ctypes.c_uint, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_size_t)]),
    "fsm_batch_download_packed": (_ST, [_VP, ctypes.c_uint, ctypes.c_uint, _VP, _VP]),
    "fsm_batch_packed_bytes": (ctypes.c_size_t, [_VP, ctypes.c_uint, ctypes.c_uint]),
    "fsm_batch_packed_offset": (_ST, [_VP, ctypes.c_uint, ctypes.c_uint, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "fsm_batch_packed_offsets": (_ST, [_VP, ctypes.c_uint, ctypes.c_uint, _VP, ctypes.c_size_t]),
    "fsm_batch_check": (_ST, [_VP]),
    "fsm_batch_energy": (_ST, [_VP, ctypes.POINTER(Energy), _VP]),
    "fsm_probe_fp32_tflops": (_ST, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "fsm_run_event_2d_noalloc": (_ST, [ctypes.POINTER(Params), _VP, ctypes.POINTER(Outputs), _VP]),
    "fsm_run_event_2d_noalloc_check": (_ST, [_VP]),
    "fsm_ctx_set_wait_limit": (_ST, [_VP, ctypes.c_int]),
    "fsm_write_field": (_ST, [ctypes.c_char_p, _VP, ctypes.POINTER(Params), ctypes.c_int,
                              ctypes.c_int]),
    "fsm_initial_energy": (_ST, [ctypes.POINTER(Params), ctypes.c_char_p, _VP]),
    "fsm_initial_baryon": (_ST, [ctypes.POINTER(Params), ctypes.c_char_p, _VP]),
    "fsm_read_profile": (_ST, [ctypes.c_char_p, ctypes.POINTER(Params), ctypes.c_int, _VP]),
    "fsm_run_event_fm4": (_ST, [_VP, ctypes.POINTER(Params), _VP, _VP, ctypes.POINTER(Outputs),
                                ctypes.POINTER(RunInfo)]),
    "fsm_write_outputs": (_ST, [ctypes.c_char_p, ctypes.POINTER(Params), ctypes.POINTER(Outputs),
                                ctypes.POINTER(Diagnostics), ctypes.c_int]),
    "fsm_diagnostics_device": (_ST, [ctypes.POINTER(Params), ctypes.POINTER(Outputs),
                                     ctypes.POINTER(Diagnostics), _VP]),
    "fsm_diagnostics_host": (_ST, [_VP, ctypes.POINTER(Params), ctypes.POINTER(Outputs),
                                   ctypes.POINTER(Diagnostics)]),
    "fsm_autotune": (_ST, [_VP, ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(_VP),
                           ctypes.POINTER(_VP), ctypes.POINTER(Tuning)]),
    "fsm_ctx_set_tuning": (_ST, [_VP, ctypes.POINTER(Tuning)]),
    "fsm_autotune_buckets": (_ST, [_VP, ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(_VP),
                                   ctypes.POINTER(_VP), ctypes.POINTER(TuningBucket)]),
    "fsm_ctx_set_tuning_buckets": (_ST, [_VP, ctypes.POINTER(TuningBucket)]),
    "fsm_tuning_save": (_ST, [_VP, ctypes.c_char_p]),
    "fsm_tuning_load": (_ST, [_VP, ctypes.c_char_p]),
    "fsm_server_start": (_ST, [ctypes.POINTER(_VP), ctypes.POINTER(ServerOpts)]),
    "fsm_server_submit": (_ST, [_VP, ctypes.POINTER(Params), _VP, _VP,
                                ctypes.POINTER(ctypes.c_longlong)]),
    "fsm_server_poll": (_ST, [_VP, ctypes.c_longlong, ctypes.POINTER(Outputs),
                              ctypes.POINTER(RunInfo), ctypes.c_double, ctypes.POINTER(ctypes.c_int)]),
    "fsm_server_poll_view": (_ST, [_VP, ctypes.c_longlong, ctypes.POINTER(Outputs),
                                   ctypes.POINTER(RunInfo), ctypes.c_double,
                                   ctypes.POINTER(ctypes.c_int)]),
    "fsm_server_release": (_ST, [_VP, ctypes.c_longlong]),
    "fsm_server_stats_get": (_ST, [_VP, ctypes.POINTER(ServerStats)]),
    "fsm_server_stop": (_ST, [_VP]),
    "fsm_server_breakdown_get": (_ST, [_VP, ctypes.POINTER(ServerBreakdown)]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built (run `make -C freestream-milne_b200`); "
                               "the compute path has no fallback")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class FsmError(RuntimeError):
    def __init__(self, status, where):
        msg = lib().fsm_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS.get(status, status)} ({msg})")
        self.status = status


def check(status, where):
    if status != FSM_OK:
        raise FsmError(status, where)


def default_params(**kw):
    p = Params()
    lib().fsm_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    lib().fsm_params_derive(ctypes.byref(p))
    return p


def read_params_file(path, base=None):
    p = base if base is not None else default_params()
    check(lib().fsm_params_read_file(str(path).encode(), ctypes.byref(p)), "fsm_params_read_file")
    return p


OUT_COMPS = dict(T=10, J=4, e=1, P=1, Pi=1, u=4, pi=10, nB=1, V=4)
SLAB_ORDER = ["T", "e", "P", "Pi", "u", "pi"]
SLAB_ORDER_BARYON = SLAB_ORDER + ["J", "nB", "V"]


def run_event_2d_noalloc(params, d_e, dev_out, stream=None):
    """The allocation-free single-event 2D entry point; device pointers (ints)."""
    o = Outputs(**{k: v for k, v in dev_out.items()})
    check(lib().fsm_run_event_2d_noalloc(ctypes.byref(params), d_e, ctypes.byref(o), stream),
          "fsm_run_event_2d_noalloc")


def run_event_2d_noalloc_check(stream=None):
    """Waits for `stream` and raises if the last allocation-free call's
    kernels reported an error."""
    check(lib().fsm_run_event_2d_noalloc_check(stream), "fsm_run_event_2d_noalloc_check")


def probe_fp32_tflops(device=0):
    v = ctypes.c_double()
    check(lib().fsm_probe_fp32_tflops(device, ctypes.byref(v)), "fsm_probe_fp32_tflops")
    return v.value


class Context:
    def __init__(self, device=0, timing=False):
        self.h = ctypes.c_void_p()
        opts = CtxOpts(device, int(timing))
        check(lib().fsm_ctx_create(ctypes.byref(self.h), ctypes.byref(opts)), "fsm_ctx_create")

    def close(self):
        if self.h:
            lib().fsm_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def timing(self, reset=False):
        t = Timing()
        check(lib().fsm_ctx_timing(self.h, ctypes.byref(t), int(reset)), "fsm_ctx_timing")
        return {k: getattr(t, k) for k, _ in Timing._fields_}

    def run_event(self, params, e_gev, nB=None, outputs=None, into=None, fm4=False):
        """Plain per-event path with host buffers; returns {name: ndarray}
        (written into the arrays of `into`, a previous result of the same
        shape, when given).  fm4: the profile is already in fm^-4
        (fsm_run_event_fm4, the reference's initial conditions other than the
        vector); otherwise in GeV/fm^3."""
        e_gev = np.ascontiguousarray(e_gev, dtype=np.float32).ravel()
        dim = params.DIM_X * params.DIM_Y * params.DIM_ETA
        if e_gev.size != dim:
            raise ValueError(f"input has {e_gev.size} cells, grid has {dim}")
        baryon = bool(params.BARYON)
        names = outputs or (list(OUT_COMPS) if baryon else [k for k in OUT_COMPS if k not in ("J", "nB", "V")])
        arrs = {}
        o = Outputs()
        for k in names:
            if into is not None and k in into:
                a = into[k]
            else:
                a = np.zeros((OUT_COMPS[k], dim) if OUT_COMPS[k] > 1 else (dim,), dtype=np.float32)
            arrs[k] = a
            setattr(o, k, a.ctypes.data)
        nb_ptr = None
        if baryon:
            nB = np.ascontiguousarray(nB, dtype=np.float32).ravel()
            nb_ptr = nB.ctypes.data
        info = RunInfo()
        fn = lib().fsm_run_event_fm4 if fm4 else lib().fsm_run_event
        check(fn(self.h, ctypes.byref(params), e_gev.ctypes.data, nb_ptr, ctypes.byref(o),
                 ctypes.byref(info)), "fsm_run_event_fm4" if fm4 else "fsm_run_event")
        arrs["info"] = {k: getattr(info, k) for k, _ in RunInfo._fields_}
        return arrs

    def autotune(self, params_list, inputs=None):
        """Times the candidate staged-window sizes on these events (inputs: list
        of (e, nB) or None for zeros) and keeps the fastest for this context."""
        n = len(params_list)
        arr = (Params * n)(*params_list)
        keep, pe, pn = [], None, None
        if inputs is not None:
            pe, pn = (_VP * n)(), (_VP * n)()
            for i, (e, nb) in enumerate(inputs):
                a = np.ascontiguousarray(e, dtype=np.float32).ravel()
                keep.append(a)
                pe[i] = a.ctypes.data
                if nb is not None:
                    b = np.ascontiguousarray(nb, dtype=np.float32).ravel()
                    keep.append(b)
                    pn[i] = b.ctypes.data
        t = Tuning()
        check(lib().fsm_autotune(self.h, n, arr, pe, pn, ctypes.byref(t)), "fsm_autotune")
        return {"window_bytes": t.window_bytes, "ms": t.ms}

    def set_wait_limit(self, polls):
        """Polls of one bounded wait in batches built from now on (0: give up at once)."""
        check(lib().fsm_ctx_set_wait_limit(self.h, int(polls)), "fsm_ctx_set_wait_limit")

    def autotune_buckets(self, params_list, inputs=None):
        """Per-bucket tuning (window, phi_p chunk, tile shapes) on these events;
        returns the 16 bucket entries as dicts (window_bytes 0: bucket not
        tuned)."""
        n = len(params_list)
        arr = (Params * n)(*params_list)
        keep = []
        he = hb = None
        if inputs is not None:
            he = (_VP * n)()
            hb = (_VP * n)()
            for i, (e, nb) in enumerate(inputs):
                e = np.ascontiguousarray(e, dtype=np.float32)
                keep.append(e)
                he[i] = e.ctypes.data
                if nb is not None:
                    nb = np.ascontiguousarray(nb, dtype=np.float32)
                    keep.append(nb)
                    hb[i] = nb.ctypes.data
        out = (TuningBucket * TUNING_BUCKETS)()
        check(lib().fsm_autotune_buckets(self.h, n, arr, he, hb, out), "fsm_autotune_buckets")
        return [{k: getattr(t, k) for k, _ in TuningBucket._fields_} for t in out]

    def set_tuning_buckets(self, table):
        arr = (TuningBucket * TUNING_BUCKETS)(*[TuningBucket(t["window_bytes"], t["phi_chunk"],
                                                             t.get("ms", 0.0), t.get("events", 0),
                                                             t.get("tile_shapes", TILES_DEFAULT))
                                                for t in table])
        check(lib().fsm_ctx_set_tuning_buckets(self.h, arr), "fsm_ctx_set_tuning_buckets")

    def save_tuning(self, path):
        check(lib().fsm_tuning_save(self.h, str(path).encode()), "fsm_tuning_save")

    def load_tuning(self, path):
        check(lib().fsm_tuning_load(self.h, str(path).encode()), "fsm_tuning_load")

    def set_tuning(self, window_bytes):
        t = Tuning(int(window_bytes), 0.0)
        check(lib().fsm_ctx_set_tuning(self.h, ctypes.byref(t)), "fsm_ctx_set_tuning")

    def diagnostics(self, params, result):
        """Hydro-validity and vorticity fields of a run_event result (TAU taken
        from its info); returns {name: ndarray}."""
        p = Params.from_buffer_copy(params)
        F_ = lib()
        F_.fsm_params_derive(ctypes.byref(p))
        p.TAU = result["info"]["tau"]
        dim = p.DIM_X * p.DIM_Y * p.DIM_ETA
        o = Outputs()
        keep = []
        for k in ("e", "P", "Pi", "u", "pi"):
            a = np.ascontiguousarray(result[k], dtype=np.float32)
            keep.append(a)
            setattr(o, k, a.ctypes.data)
        arrs, dg = {}, Diagnostics()
        for k, c in DIAG_COMPS.items():
            a = np.zeros((c, dim) if c > 1 else (dim,), dtype=np.float32)
            arrs[k] = a
            setattr(dg, k, a.ctypes.data)
        check(F_.fsm_diagnostics_host(self.h, ctypes.byref(p), ctypes.byref(o), ctypes.byref(dg)),
              "fsm_diagnostics_host")
        return arrs

    def run_event_device(self, params, d_e, d_nB, dev_out, stream=None):
        """Device path; d_e/d_nB/dev_out values are raw device pointers (ints)."""
        o = Outputs(**{k: v for k, v in dev_out.items()})
        info = RunInfo()
        check(lib().fsm_run_event_device(self.h, ctypes.byref(params), d_e, d_nB, ctypes.byref(o),
                                         stream, ctypes.byref(info)), "fsm_run_event_device")
        return {k: getattr(info, k) for k, _ in RunInfo._fields_}


def out_mask(groups):
    """OR of the FSM_OUT_* bits of the named output groups (OUT_GROUPS names)."""
    m = 0
    for k in groups:
        m |= 1 << OUT_GROUPS.index(k)
    return m


class Batch:
    def __init__(self, ctx, params_list, grouped=False):
        self.ctx = ctx
        n = len(params_list)
        arr = (Params * n)(*params_list)
        self.params = list(params_list)
        self.grouped = bool(grouped)
        self.h = ctypes.c_void_p()
        check(lib().fsm_batch_create_ex(ctx.h, n, arr, int(self.grouped), ctypes.byref(self.h)),
              "fsm_batch_create_ex")
        self.n = n
        ib, ob = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib().fsm_batch_slabs(self.h, ctypes.byref(ib), ctypes.byref(ob)), "fsm_batch_slabs")
        self.in_bytes, self.out_bytes = ib.value, ob.value

    def close(self):
        if self.h:
            lib().fsm_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def offsets(self, ev):
        a, b = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib().fsm_batch_event_offsets(self.h, ev, ctypes.byref(a), ctypes.byref(b)),
              "fsm_batch_event_offsets")
        return a.value, b.value

    def info(self, ev):
        info = RunInfo()
        check(lib().fsm_batch_info(self.h, ev, ctypes.byref(info)), "fsm_batch_info")
        return {k: getattr(info, k) for k, _ in RunInfo._fields_}

    def samples(self):
        return lib().fsm_batch_samples(self.h)

    def upload(self, host_ptr, stream=None):
        check(lib().fsm_batch_upload(self.h, host_ptr, stream), "fsm_batch_upload")

    def download(self, host_ptr, stream=None):
        check(lib().fsm_batch_download(self.h, host_ptr, stream), "fsm_batch_download")

    def launch(self, stream=None):
        check(lib().fsm_batch_launch(self.h, stream), "fsm_batch_launch")

    def groups_bytes(self, groups):
        return lib().fsm_batch_groups_bytes(self.h, out_mask(groups))

    def download_groups(self, groups, host_ptr, stream=None):
        """Grouped batches: copy back only `groups`, packed in OUT_GROUPS order."""
        check(lib().fsm_batch_download_groups(self.h, out_mask(groups), host_ptr, stream),
              "fsm_batch_download_groups")

    def group_offset(self, groups, group, ev):
        o = ctypes.c_size_t()
        check(lib().fsm_batch_group_offset(self.h, out_mask(groups), OUT_GROUPS.index(group), ev,
                                           ctypes.byref(o)), "fsm_batch_group_offset")
        return o.value

    def packed_bytes(self, groups, skip_eta=False):
        return lib().fsm_batch_packed_bytes(self.h, out_mask(groups), PACK_SKIP_ETA if skip_eta else 0)

    def download_packed(self, groups, host_ptr, skip_eta=False, stream=None):
        """Gather `groups` on the device and copy them back with one copy; with
        skip_eta the components of 2D events that vanish by symmetry are left out."""
        check(lib().fsm_batch_download_packed(self.h, out_mask(groups),
                                              PACK_SKIP_ETA if skip_eta else 0, host_ptr, stream),
              "fsm_batch_download_packed")

    def packed_offset(self, groups, group, comp, ev, skip_eta=False):
        """Offset (floats) of component `comp` of `group` of event `ev` in a
        packed download, or None when the component is left out."""
        o = ctypes.c_size_t()
        st = lib().fsm_batch_packed_offset(self.h, out_mask(groups), PACK_SKIP_ETA if skip_eta else 0,
                                           OUT_GROUPS.index(group), comp, ev, ctypes.byref(o))
        return o.value if st == 0 else None

    def packed_offsets(self, groups, skip_eta=False):
        """(events, 9 groups, 10 components) array of packed-buffer offsets,
        -1 where a component is not in the packed buffer (cached)."""
        key = (tuple(groups), bool(skip_eta))
        cache = self.__dict__.setdefault("_pack_offsets", {})
        if key not in cache:
            a = np.empty(self.n * len(OUT_GROUPS) * 10, np.uint64)
            check(lib().fsm_batch_packed_offsets(self.h, out_mask(groups),
                                                 PACK_SKIP_ETA if skip_eta else 0,
                                                 a.ctypes.data, a.size), "fsm_batch_packed_offsets")
            cache[key] = a.astype(np.int64).reshape(self.n, len(OUT_GROUPS), 10)
        return cache[key]

    def unpack_packed(self, packed, groups, ev, skip_eta=False):
        """Per-event dict of the `groups` arrays from a packed download; left-out
        components (zero by symmetry) come back as zeros."""
        p = self.params[ev]
        dim = p.DIM_X * p.DIM_Y * p.DIM_ETA
        offs = self.packed_offsets(groups, skip_eta)[ev]
        res = {}
        for k in OUT_GROUPS:
            if k not in groups or (k in ("J", "nB", "V") and not p.BARYON):
                continue
            c = OUT_COMPS[k]
            a = np.zeros((c, dim), np.float32)
            for m in range(c):
                off = int(offs[OUT_GROUPS.index(k), m])
                if off >= 0:
                    a[m] = packed[off:off + dim]
            res[k] = a if c > 1 else a[0]
        return res

    def unpack_groups(self, packed, groups, ev):
        """Per-event dict of the `groups` arrays from a download_groups buffer."""
        p = self.params[ev]
        dim = p.DIM_X * p.DIM_Y * p.DIM_ETA
        res = {}
        for k in OUT_GROUPS:
            if k not in groups or (k in ("J", "nB", "V") and not p.BARYON):
                continue
            c = OUT_COMPS[k]
            off = self.group_offset(groups, k, ev)
            a = packed[off:off + c * dim]
            res[k] = a.reshape(c, dim) if c > 1 else a
        return res

    def check_errors(self):
        check(lib().fsm_batch_check(self.h), "fsm_batch_check")

    def energy(self, stream=None):
        """Per event: total energy before / after streaming, the part inside
        E_FREEZE and its fraction (fsm_batch_energy)."""
        out = (Energy * self.n)()
        check(lib().fsm_batch_energy(self.h, out, stream), "fsm_batch_energy")
        return [{k: getattr(x, k) for k, _ in Energy._fields_} for x in out]

    def pack_inputs(self, inputs):
        """inputs: list of (e_gev, nB or None) -> float32 host slab."""
        slab = np.zeros(self.in_bytes // 4, dtype=np.float32)
        for ev, (e, nb) in enumerate(inputs):
            off, _ = self.offsets(ev)
            e = np.ascontiguousarray(e, dtype=np.float32).ravel()
            slab[off:off + e.size] = e
            if self.params[ev].BARYON:
                slab[off + e.size:off + 2 * e.size] = np.ascontiguousarray(nb, np.float32).ravel()
        return slab

    def unpack_outputs(self, slab, ev):
        """Per-event dict of output arrays from a downloaded output slab."""
        if self.grouped:
            return self.unpack_groups(slab, OUT_GROUPS, ev)
        p = self.params[ev]
        dim = p.DIM_X * p.DIM_Y * p.DIM_ETA
        _, off = self.offsets(ev)
        res = {}
        order = SLAB_ORDER_BARYON if p.BARYON else SLAB_ORDER
        for k in order:
            c = OUT_COMPS[k]
            a = slab[off:off + c * dim]
            res[k] = a.reshape(c, dim) if c > 1 else a
            off += c * dim
        return res

    def run_host(self, inputs):
        """Upload, launch, download, synchronise; returns per-event output dicts."""
        import torch  # pinned staging only
        ins = torch.from_numpy(self.pack_inputs(inputs)).pin_memory()
        outs = torch.empty(self.out_bytes // 4, dtype=torch.float32).pin_memory()
        self.upload(ins.data_ptr())
        self.launch()
        self.download(outs.data_ptr())
        self.check_errors()  # synchronises
        o = outs.numpy()
        return [{k: v.copy() for k, v in self.unpack_outputs(o, ev).items()} for ev in range(self.n)]


def write_field(path, var, params, projection=False, nthreads=0):
    """One per-cell field in the reference's text format (src/FileIO.cpp:11-131)."""
    v = np.ascontiguousarray(var, dtype=np.float32)
    if v.size != params.DIM_X * params.DIM_Y * params.DIM_ETA:
        raise ValueError("field size does not match the grid")
    check(lib().fsm_write_field(str(path).encode(), v.ctypes.data, ctypes.byref(params),
                                int(bool(projection)), int(nthreads)), "fsm_write_field")


def write_outputs(dirpath, params, result, diag=None, nthreads=0):
    """Every output file of one event (the reference's post-matching file set)
    from host arrays: result as returned by Context.run_event, diag as by
    Context.diagnostics (or None)."""
    keep = []

    def ptr(a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        keep.append(a)
        return a.ctypes.data

    o = Outputs(**{k: ptr(result[k]) for k in ("e", "P", "Pi", "u", "pi", "nB", "V")
                   if result.get(k) is not None})
    d = None
    if diag is not None:
        d = Diagnostics(**{k: ptr(diag[k]) for k in DIAG_COMPS if diag.get(k) is not None})
    check(lib().fsm_write_outputs(str(dirpath).encode(), ctypes.byref(params), ctypes.byref(o),
                                  ctypes.byref(d) if d is not None else None, int(nthreads)),
          "fsm_write_outputs")


PROFILE_FORMATS = {"xyev": 0, "cpuvh": 1, "supermc_block": 2, "trento_block": 3, "trento3d_block": 4}


def initial_profile(params, kind="energy", directory=None):
    """The reference's initial condition params.IC_ENERGY (or IC_BARYON) as a
    float32 profile in fm^-4 (fsm_initial_energy / fsm_initial_baryon)."""
    out = np.zeros(params.DIM_X * params.DIM_Y * params.DIM_ETA, np.float32)
    fn = lib().fsm_initial_energy if kind == "energy" else lib().fsm_initial_baryon
    check(fn(ctypes.byref(params), None if directory is None else str(directory).encode(),
             out.ctypes.data), "fsm_initial_" + kind)
    return out


def read_profile(path, params, fmt):
    out = np.zeros(params.DIM_X * params.DIM_Y * params.DIM_ETA, np.float32)
    check(lib().fsm_read_profile(str(path).encode(), ctypes.byref(params), PROFILE_FORMATS[fmt],
                                 out.ctypes.data), "fsm_read_profile")
    return out


def device_count():
    """Visible CUDA devices (0 without a GPU or driver)."""
    n = ctypes.c_int(0)
    check(lib().fsm_device_count(ctypes.byref(n)), "fsm_device_count")
    return n.value


class Server:
    """Continuous-batching request server (fsm_server_*): submit events as they
    arrive, poll for their outputs; results equal Context.run_event's."""

    def __init__(self, device=0, hbm_budget=0, host_budget=0, max_wave_events=0, streams=0,
                 outputs=None, stream_2d=False):
        self.h = ctypes.c_void_p()
        self.outputs = list(outputs) if outputs else list(OUT_GROUPS)
        mask = out_mask(self.outputs)
        opts = ServerOpts(device, int(hbm_budget), int(host_budget), int(max_wave_events),
                          int(streams), mask, int(bool(stream_2d)))
        check(lib().fsm_server_start(ctypes.byref(self.h), ctypes.byref(opts)), "fsm_server_start")
        self._pending = {}

    def submit(self, params, e_gev, nB=None):
        e_gev = np.ascontiguousarray(e_gev, dtype=np.float32).ravel()
        nb_ptr = None
        if params.BARYON:
            nB = np.ascontiguousarray(nB, dtype=np.float32).ravel()
            nb_ptr = nB.ctypes.data
        rid = ctypes.c_longlong()
        check(lib().fsm_server_submit(self.h, ctypes.byref(params), e_gev.ctypes.data, nb_ptr,
                                      ctypes.byref(rid)), "fsm_server_submit")
        dim = params.DIM_X * params.DIM_Y * params.DIM_ETA
        self._pending[rid.value] = (dim, bool(params.BARYON))
        return rid.value

    def poll(self, rid, timeout_ms=-1.0):
        """None while running; the outputs dict once done (FsmError if it failed)."""
        dim, baryon = self._pending[rid]
        names = [k for k in self.outputs if baryon or k not in ("J", "nB", "V")]
        arrs, o = {}, Outputs()
        for k in names:
            a = np.zeros((OUT_COMPS[k], dim) if OUT_COMPS[k] > 1 else (dim,), dtype=np.float32)
            arrs[k] = a
            setattr(o, k, a.ctypes.data)
        info, done = RunInfo(), ctypes.c_int(0)
        st = lib().fsm_server_poll(self.h, rid, ctypes.byref(o), ctypes.byref(info),
                                   float(timeout_ms), ctypes.byref(done))
        if not done.value:
            check(st, "fsm_server_poll")
            return None
        del self._pending[rid]
        check(st, "fsm_server_poll")
        arrs["info"] = {k: getattr(info, k) for k, _ in RunInfo._fields_}
        return arrs

    def poll_view(self, rid, timeout_ms=-1.0):
        """Zero-copy poll: None while running; once done, read-only arrays viewing
        the server's pinned memory, valid until release(rid)."""
        dim, baryon = self._pending[rid]
        o, info, done = Outputs(), RunInfo(), ctypes.c_int(0)
        st = lib().fsm_server_poll_view(self.h, rid, ctypes.byref(o), ctypes.byref(info),
                                        float(timeout_ms), ctypes.byref(done))
        if not done.value:
            check(st, "fsm_server_poll_view")
            return None
        if st != FSM_OK:
            self.release(rid)
            check(st, "fsm_server_poll_view")
        arrs = {}
        for k in self.outputs:
            ptr = getattr(o, k)
            if ptr:
                n = OUT_COMPS[k] * dim
                a = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), (n,))
                a.flags.writeable = False
                arrs[k] = a.reshape((OUT_COMPS[k], dim)) if OUT_COMPS[k] > 1 else a
        arrs["info"] = {k: getattr(info, k) for k, _ in RunInfo._fields_}
        return arrs

    def release(self, rid):
        check(lib().fsm_server_release(self.h, rid), "fsm_server_release")
        self._pending.pop(rid, None)

    def stats(self):
        st = ServerStats()
        check(lib().fsm_server_stats_get(self.h, ctypes.byref(st)), "fsm_server_stats_get")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def breakdown(self):
        """Per-wave means of where the server's time goes (fsm_server_breakdown_get)."""
        bd = ServerBreakdown()
        check(lib().fsm_server_breakdown_get(self.h, ctypes.byref(bd)), "fsm_server_breakdown_get")
        return {k: getattr(bd, k) for k, _ in ServerBreakdown._fields_}

    def stop(self):
        if self.h:
            check(lib().fsm_server_stop(self.h), "fsm_server_stop")
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
