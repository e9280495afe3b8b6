#!/usr/bin/env python
"""Benchmark of the free-streaming + Landau-matching path on B200.

Workload (one step): the batched configuration -- 512 seeded uneven 2D events
(grid side in {101,151,201,261,301}, DX in [0.05,0.1] fm, DIM_PHIP in
{64,100,200} raised by the arc-length rule, DTAU in [0.3,1.5] fm/c, conformal
or Wuppertal-Budapest EoS) run as one batch: one persistent launch per kernel
family, replayed from a CUDA graph.  Each rank runs its own 512 events
(replicas, weak scaling, no collective on the data path).

Printed JSON line (rank 0):
  value        events/s over all ranks, inputs resident in HBM
  e2e          events/s through the C ABI with the host round trip inside the
               timed region (pinned input slab H2D, launch, D2H of the fields
               the reference returns to its caller: e, P, Pi, u, pi, less the
               components that vanish by boost invariance)
  plain_*      the same events one at a time (one launch sequence per event)
  roofline     fused stream kernel, FP32 pipe: algorithmic FLOPs / measured
               launch time vs the measured FP32 FMA peak of the same GPU
  cpu_baseline the reference's own sources (or the oracle port) on host cores
  served       Poisson streams of mixed 2D/3D requests (and 2D only) through
               the continuous-batching server: burst capacity, p50/p99 at 70 %
               load, per-wave breakdown, against the one-event host path
  event_3d     one 131^2 x 51 baryon event (21 rapidities, 100 phi_p) with the
               3D stream kernel's roofline

`--impl reference` times the reference's CPU implementation on the same
workload and prints the same metric.
"""
import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "freestream-milne_b200"))

METRIC = "events/s & p99 latency, batched/served vs plain GPU path at ≤1e-5 Tμν rel err"
FLOPS_PER_SAMPLE_2D = 55  # shift 4 + bicubic 30 + bilinear 9 + 6 moments 12
# 3D with baryons, per in-grid sample: the reference's trilinear form counts
# shift 5 + 2 trilinear x 21 + 14 moments x 2 = 75; the kernel interpolates
# combined node planes (eta interpolation and rapidity weights applied once
# per node and (slice, rapidity) pair by the prep kernel), executing shift 5
# + 2 bilinear x 9 + 14 moments x 2 = 51 per sample
FLOPS_PER_SAMPLE_3D_BARYON = 51
FLOPS_PER_SAMPLE_3D_BARYON_REF = 75
# algorithmic DRAM bytes per cell of the 2D prep and Landau kernels: prep reads
# the profile (4 B), writes and re-reads F and its y-slopes (8 + 8 B) and
# writes the node array (16 B); Landau reads the 6 non-zero T components of a
# boost-invariant event (24 B) and writes e, P, Pi, u, pi (68 B)
PREP_BYTES_PER_CELL_2D = 36
LANDAU_BYTES_PER_CELL_2D = 92


def _hbm_gbs():
    """Measured copy bandwidth of this pool's B200s (GB/s), else the earlier
    measurement of 6650 GB/s."""
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0


HBM_GBS = _hbm_gbs()
# DRAM bytes per cell x phi_p sample of fsm_stream2d_kernel: (88.9 MB read +
# 167.7 MB written) / 713.26 M samples, from one ncu capture of the launch on
# the first 128 events of this workload (a full 512-event launch is above the
# capture size rule), scaled by samples
TRAFFIC_BYTES_PER_SAMPLE_2D = (88.878592e6 + 167.744512e6) / 713258674
WORKLOAD = ("uneven_batch: 512 seeded lumpy 2D events, side {101,151,201,261,301}, DX U[0.05,0.1], "
            "DIM_PHIP {64,100,200} + arc-length rule, DTAU U[0.3,1.5], EOS 1/2 50:50, TAU0 0.2")
L2_NOTE = ("no explicit flush: each step streams ~2 GB (inputs 86 MB, spline scratch, 1.6 GB "
           "outputs) through the 126 MB L2")


def config_of(args):
    """The workload both arms time (identical in the reference arm's line)."""
    return {"workload": WORKLOAD, "events": args.events, "seed": 3,
            "sample": f"all {args.events} events of the seeded list (rank r: seed 3 + 1000 r)",
            "l2": L2_NOTE}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--events", type=int, default=512)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-3d", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=160)
    ap.add_argument("--serve-load", type=float, default=0.7,
                    help="Poisson arrival rate as a fraction of the measured burst capacity")
    return ap.parse_args()


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def wait_first(self, timeout_s=5.0):
        """Waits until nvidia-smi has written its first sample (it takes a
        while to start), so that the timed region that follows is sampled."""
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < timeout_s:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0:
                return
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def cpu_baseline(events, nthreads, budget_s=20.0):
    """Times the reference's CPU implementation on a bounded sample of the
    workload: oracle/_ref (reference sources, OpenMP) when built, otherwise the
    oracle port.  Returns (events/s, kind, sample description)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py as O
    kind = "reference" if O.ref_available() else "port"
    impl = "ref" if kind == "reference" else "oracle"
    if kind == "port":
        os.environ.setdefault("OMP_NUM_THREADS", str(nthreads))
    # silence the reference's progress prints on stdout
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    done = 0
    t0 = time.perf_counter()
    try:
        for p, e, nb in events:
            O.run(O.Params(**p.as_dict()), e, nB=nb, impl=impl, nthreads=nthreads)
            done += 1
            if time.perf_counter() - t0 > budget_s:
                break
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)
    dt = time.perf_counter() - t0
    return done / dt, kind, f"first {done} events of the workload, {nthreads} OpenMP threads, {dt:.1f} s"


def serve_stream(args, F, W, local, rank, ctx, reps, frac3d=0.2, opts=None):
    """Request stream (by default 80 % 2D of sides 101-301, 20 % 3D of 131^2 x
    {25, 51} with 21/31/41 rapidities; frac3d=0: boost-invariant requests only)
    through the continuous-batching server: a burst measures capacity, then
    Poisson arrivals at serve_load x capacity give p50/p99 latency; the same
    requests one by one through fsm_run_event give the plain path."""
    import threading
    reqs = W.stream_requests(args.serve_requests, rate_hz=1.0, seed=reps.seed(4), frac3d=frac3d)
    gaps = [reqs[0][0]] + [reqs[k][0] - reqs[k - 1][0] for k in range(1, len(reqs))]
    events = [ev for _, ev in reqs]
    hydro = ["e", "P", "Pi", "u", "pi", "nB", "V"]  # the fields the reference hands to hydro
    # 12 streams (waves overlap host planning, copies and kernels; measured
    # burst capacity on one box with the current kernels 1705 / ~1770 / 1885
    # events/s with 4 / 8 / 12, p99 at 70 % load 16.9 / 11.2-13.0 / 11.5 ms)
    # and one more reserved for boost-invariant waves
    budget = dict(hbm_budget=48 << 30, host_budget=8 << 30, streams=12, stream_2d=True, outputs=hydro)
    budget.update(opts or {})

    def run(rate_hz):
        srv = F.Server(local, **budget)
        ids = []
        t0 = time.perf_counter()

        def feeder():
            t = t0
            for g, (p, e, nb) in zip(gaps, events):
                if rate_hz:
                    t += g / rate_hz
                    d = t - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                ids.append(srv.submit(p, e, nb))

        th = threading.Thread(target=feeder)
        th.start()
        k = 0
        while k < len(events):
            if k < len(ids):
                srv.poll_view(ids[k])  # zero-copy: the client reads the pinned outputs
                srv.release(ids[k])
                k += 1
            else:
                time.sleep(1e-4)
        th.join()
        st = srv.stats()
        st["breakdown"] = srv.breakdown()
        srv.stop()
        return st

    burst = run(0.0)
    cap = burst["events_per_s"]
    rate = args.serve_load * cap
    st = run(rate)
    # plain per-event path on the same requests
    bufs = {}
    t0 = time.perf_counter()
    for p, e, nb in events:
        key = (p.DIM_X, p.DIM_Y, p.DIM_ETA, p.BARYON)
        bufs[key] = ctx.run_event(p, e, nb, outputs=hydro, into=bufs.get(key))
    plain = len(events) / (time.perf_counter() - t0)
    n3 = sum(1 for p, _, _ in events if p.DIM_ETA > 1)
    # whole job: rates summed over the replicas, latencies the worst rank's
    cap_all, plain_all = reps.sum(cap), reps.sum(plain)
    return {"requests": len(events) * reps.world, "requests_3d": n3, "burst_events_per_s": cap_all,
            "rate_hz": reps.sum(rate), "load": args.serve_load,
            "events_per_s": reps.sum(st["events_per_s"]),
            "p50_ms": reps.max(st["p50_ms"]), "p99_ms": reps.max(st["p99_ms"]),
            "max_ms": reps.max(st["max_ms"]), "waves": st["waves"],
            "burst_breakdown": burst["breakdown"], "load_breakdown": st["breakdown"],
            "plain_events_per_s": plain_all, "burst_over_plain": cap_all / plain_all,
            "outputs": hydro,
            "budget": {"hbm_bytes": budget["hbm_budget"], "pinned_host_bytes": budget["host_budget"]}}


def other_kernels(tm, steps, cells):
    """The prep and Landau kernels against the measured HBM copy bandwidth
    (their algorithmic bytes per cell over their CUDA-event time); both are
    bound by FP64 latency, not by DRAM, so the fractions stay well below 1."""
    out = {}
    for name, per_cell in (("prep", PREP_BYTES_PER_CELL_2D), ("landau", LANDAU_BYTES_PER_CELL_2D)):
        ms = tm[f"{name}_ms"] / steps
        gbs = cells * per_cell / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "cells": cells, "bytes_per_cell": per_cell, "achieved_gbs": gbs,
                     "peak_gbs": HBM_GBS, "frac": gbs / HBM_GBS, "bound": "fp64 latency",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy)"}
    return out


def cpu_model():
    """The host CPU's model name and logical core count."""
    name = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                name = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{name} ({os.cpu_count()} logical cores)"


def issue_peak(torch, device, clocks):
    """FP32 FMA issue peak in TFLOP/s: SMs x 128 FP32 lanes x 2 FLOP x the
    maximum SM clock seen (nominal 148 x 128 x 2 x 1.965 GHz = 74.4)."""
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = (clocks or {}).get("sm_max_mhz") or 1965.0
    return sms * 128 * 2 * mhz * 1e6 / 1e12


def event_3d(F, W, local, sp, stream, args):
    """The 3D configuration with baryon charge, one event device-resident:
    131 x 131 x 51 cells, 21 rapidities (tan map), 100 phi_p, DTAU 0.8."""
    import torch
    p, e, nb = W.baryon3d()
    ctx = F.Context(local, timing=True)
    b = F.Batch(ctx, [p])
    h_in = torch.from_numpy(b.pack_inputs([(e, nb)])).pin_memory()
    b.upload(h_in.data_ptr(), sp)
    for _ in range(2):
        b.launch(sp)
    stream.synchronize()
    ctx.timing(reset=True)
    n = max(3, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(n):
        b.launch(sp)
    e1.record(stream)
    stream.synchronize()
    b.check_errors()
    ms = e0.elapsed_time(e1) / n
    tm = ctx.timing(reset=True)
    live = b.samples()
    ref = p.DIM_X * p.DIM_Y * p.DIM_ETA * p.DIM_RAP * b.info(0)["dim_phip"]
    stream_ms = tm["stream_ms"] / max(tm["stream_launches"], 1)
    out = {"config": "131x131x51, DIM_RAP 21 (tan map), DIM_PHIP 100, DTAU 0.8, BARYON 1, EOS 1",
           "ms_per_event": ms, "stream_ms": stream_ms, "landau_ms": tm["landau_ms"] / n,
           "live_samples": live, "reference_samples": ref,
           "live_samples_per_s": live / (stream_ms * 1e-3),
           "stream_tflops": live * FLOPS_PER_SAMPLE_3D_BARYON / (stream_ms * 1e-3) / 1e12,
           "flops_per_sample": FLOPS_PER_SAMPLE_3D_BARYON,
           "reference_form_tflops": live * FLOPS_PER_SAMPLE_3D_BARYON_REF / (stream_ms * 1e-3) / 1e12,
           "reference_form_flops_per_sample": FLOPS_PER_SAMPLE_3D_BARYON_REF}
    b.close()
    ctx.close()
    return out


def output_files(F, W, ctx):
    """Every output file of one event (the reference's post-matching file set,
    47 files for a 2D event) from host arrays: fsm_write_outputs (files
    formatted concurrently on all host threads) against the reference's own
    writers (src/FileIO.cpp:11-131, one file after another, as its
    run_freestream_milne calls them), on the outputs of the 261^2 lumpy event."""
    import shutil
    import numpy as np
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py as O
    p, e, _ = W.lumpy2d(seed=1)
    got = ctx.run_event(p, e)
    dg = ctx.diagnostics(p, got)
    p.TAU = got["info"]["tau"]
    tmp = pathlib.Path(tempfile.mkdtemp(prefix="fsm_out_"))
    try:
        ours = []
        (tmp / "ours").mkdir()
        for _ in range(3):
            t0 = time.perf_counter()
            F.write_outputs(tmp / "ours", p, got, dg)
            ours.append(time.perf_counter() - t0)
        nbytes = sum(f.stat().st_size for f in (tmp / "ours").iterdir())
        nfiles = len(list((tmp / "ours").iterdir()))
        out = {"event": "261^2 lumpy, DIM_PHIP 200, WB EoS", "files": nfiles, "bytes": nbytes,
               "ours_ms": 1e3 * min(ours), "threads": os.cpu_count()}
        if O.ref_available():
            (tmp / "ref" / "output").mkdir(parents=True)
            d17 = np.concatenate([np.asarray(dg[k], np.float32).reshape(c, -1)
                                  for k, c in F.DIAG_COMPS.items()])
            t0 = time.perf_counter()
            O.ref_write_outputs(tmp / "ref", O.Params(**p.as_dict()), got, d17)
            out["reference_ms"] = 1e3 * (time.perf_counter() - t0)
            out["reference"] = "the reference's writers, compiled from its sources (one thread)"
            out["identical_bytes"] = all((tmp / "ours" / f.name).read_bytes() == f.read_bytes()
                                         for f in (tmp / "ref" / "output").iterdir())
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def reference_arm(args):
    """The reference's CPU implementation on the same 512 events: the timed
    steps walk through the seeded event list in order, ceil(512 / steps)
    events per step, so that together they run every event of the workload
    once (a few repeat when the division is not exact).  Only the oracle
    module and the workload generators are loaded -- never libfsm.so."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import workloads as W  # library-free generators (fsm_params, numpy)
    nthreads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    events = W.uneven_batch(n=args.events, seed=3)
    n = len(events)
    per_step = -(-n // args.steps)
    kind = None
    for s in range(args.warmup):  # one event per warm-up step
        _, kind, _ = cpu_baseline([events[s % n]], nthreads, budget_s=1e9)
    times, done = [], 0
    for s in range(args.steps):
        chunk = [events[(s * per_step + k) % n] for k in range(per_step)]
        rate, kind, _ = cpu_baseline(chunk, nthreads, budget_s=1e9)
        times.append(len(chunk) / rate)
        done += len(chunk)
    total = sum(times)
    value = done / total
    sample = (f"all {n} events of the workload in order, {per_step} per step over {args.steps} "
              f"timed steps ({done} event runs), {nthreads} OpenMP threads")
    line = {"metric": METRIC, "value": value, "unit": "events/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(args),
            "setup": {"parallelism": f"cpu ({nthreads} threads)", "events_per_step": per_step},
            "cpu_baseline": {"value": value, "unit": "events/s", "cores": nthreads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)

    import numpy as np
    import torch
    import fsm_b200 as F
    import workloads as W

    from replicas import Replicas
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    reps = Replicas(backend="nccl")  # one process per GPU, own events; timing reductions only
    rank, world = reps.rank, reps.world
    barrier, max_over_ranks = reps.barrier, reps.max

    events = W.uneven_batch(n=args.events, seed=reps.seed(3))
    params = [p for p, _, _ in events]
    ctx = F.Context(local)
    tuning = ctx.autotune(params, [(e, nb) for _, e, nb in events])  # staged-window size
    # per bucket (grid side x shift length): window, phi_p chunk, tile shapes
    buckets = ctx.autotune_buckets(params, [(e, nb) for _, e, nb in events])
    tiles_name = {F.TILES_DEFAULT: "tail tiles", F.TILES_TAIL: "tail tiles",
                  F.TILES_SQUARE: "32x32 tiles"}
    bucket_choice = {k: f"{t['window_bytes'] // 1024} KB / {t['phi_chunk']} / "
                        f"{tiles_name[t['tile_shapes']]}"
                     for k, t in enumerate(buckets) if t["window_bytes"]}
    batch = F.Batch(ctx, params)
    cells_per_step = sum(p.DIM_X * p.DIM_Y for p in params)
    n = len(events)
    # host cost of a fresh event set: planning (tables, runs, work lists),
    # the batch's one device allocation and the upload of its tables
    t0 = time.perf_counter()
    fresh = F.Batch(ctx, params)
    create_cold_ms = 1e3 * (time.perf_counter() - t0)
    fresh.close()  # its allocations stay with the context for the next batch
    fresh_events = W.uneven_batch(n=args.events, seed=reps.seed(5))
    t0 = time.perf_counter()
    fresh = F.Batch(ctx, [p for p, _, _ in fresh_events])
    create_ms = 1e3 * (time.perf_counter() - t0)
    fresh.close()
    del fresh_events
    h_in = torch.from_numpy(batch.pack_inputs([(e, nb) for _, e, nb in events])).pin_memory()
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    batch.upload(h_in.data_ptr(), sp)
    torch.cuda.synchronize()

    # ---------------- device-resident batched path (graph replay)
    for _ in range(args.warmup):
        batch.launch(sp)
    stream.synchronize()
    batch.check_errors()
    step_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.wait_first()
    with torch.cuda.stream(stream):
        step_ev[0].record(stream)
        for k in range(args.steps):
            batch.launch(sp)
            step_ev[k + 1].record(stream)
    stream.synchronize()
    clocks = clk.stop()
    torch.cuda.synchronize()
    barrier()
    step_ms = [step_ev[k].elapsed_time(step_ev[k + 1]) for k in range(args.steps)]
    t_ms = max_over_ranks(sum(step_ms))
    value = world * n * args.steps / (t_ms / 1e3)

    # ---------------- end to end through the C ABI, host buffers.  Two batches
    # on two streams alternate steps, so one step's copies overlap the other's
    # kernels; each step uploads its input slab and copies back, packed on the
    # device into one transfer, the fields the reference hands its caller
    # (output_to_vectors, src/FreestreamMilne.cpp:700-716: e, P, Pi, u^mu,
    # pi^{mu nu}) without the components that vanish by symmetry in these
    # boost-invariant events (u^eta, pi^{tau eta}, pi^{x eta}, pi^{y eta}).
    e2e_groups = ["e", "P", "Pi", "u", "pi"]
    pair = [F.Batch(ctx, params) for _ in range(2)]
    e2e_streams = [stream, torch.cuda.Stream()]
    d2h_bytes = pair[0].packed_bytes(e2e_groups, skip_eta=True)
    h_outs = [torch.empty(d2h_bytes // 4, dtype=torch.float32).pin_memory() for _ in range(2)]

    def e2e_step(k):
        b, s = pair[k % 2], e2e_streams[k % 2].cuda_stream
        b.upload(h_in.data_ptr(), s)
        b.launch(s)
        b.download_packed(e2e_groups, h_outs[k % 2].data_ptr(), skip_eta=True, stream=s)

    for k in range(max(2, args.warmup)):
        e2e_step(k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(e2e_streams[0])
    e2e_streams[1].wait_event(e0)
    for k in range(args.steps):
        e2e_step(k)
    e2e_streams[0].wait_stream(e2e_streams[1])
    e1.record(e2e_streams[0])
    torch.cuda.synchronize()
    for b in pair:
        b.check_errors()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e = world * n * args.steps / (e2e_ms / 1e3)
    # the packed host copy holds the same values as the device-resident run
    got = pair[(args.steps - 1) % 2].unpack_packed(h_outs[(args.steps - 1) % 2].numpy(),
                                                   e2e_groups, 0, skip_eta=True)
    h_full = torch.empty(batch.out_bytes // 4, dtype=torch.float32).pin_memory()
    batch.download(h_full.data_ptr(), sp)
    batch.check_errors()
    ref0 = batch.unpack_outputs(h_full.numpy(), 0)
    for k in e2e_groups:
        if not np.array_equal(got[k], ref0[k]):
            raise RuntimeError(f"e2e copy of {k} differs from the device-resident result")
    del h_full
    for b in pair:
        b.close()

    # ---------------- kernel timing pass for the roofline (CUDA events per kernel family)
    tctx = F.Context(local, timing=True)
    tctx.set_tuning(tuning["window_bytes"])
    tctx.set_tuning_buckets(buckets)
    tb = F.Batch(tctx, params)
    tb.upload(h_in.data_ptr(), sp)
    for _ in range(2):
        tb.launch(sp)
    stream.synchronize()
    tctx.timing(reset=True)
    for _ in range(args.steps):
        tb.launch(sp)
    stream.synchronize()
    tm = tctx.timing(reset=True)
    samples = batch.samples()
    stream_ms = tm["stream_ms"] / max(tm["stream_launches"], 1)
    achieved = samples * FLOPS_PER_SAMPLE_2D / (stream_ms * 1e-3) / 1e12
    peak = F.probe_fp32_tflops(local)

    # ---------------- plain per-event GPU path: same events, one launch sequence each
    plain = None
    if not args.no_plain:
        singles = [F.Batch(ctx, [p]) for p in params]
        for s, (p, e, nb) in zip(singles, events):
            s.upload(torch.from_numpy(s.pack_inputs([(e, nb)])).pin_memory().data_ptr(), sp)
        for s in singles[:8]:
            s.launch(sp)
        stream.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for s in singles:
            s.launch(sp)
        p1.record(stream)
        stream.synchronize()
        plain_ms = max_over_ranks(p0.elapsed_time(p1))
        plain = world * n / (plain_ms / 1e3)
        for s in singles:
            s.close()

    # ---------------- served: Poisson stream of mixed 2D/3D requests through the server
    served = served_2d = None
    if not args.no_serve:
        served = serve_stream(args, F, W, local, rank, ctx, reps)
        served_2d = serve_stream(args, F, W, local, rank, ctx, reps, frac3d=0.0)

    # ---------------- one 3D event with baryon charge (131^2 x 51, 21 rapidities, 100 phi_p)
    ev3d = None
    if not args.no_3d:
        ev3d = event_3d(F, W, local, sp, stream, args)
        ev3d["roofline"] = {"bound": "fp32", "kernel": "fsm_stream3d_baryon_kernel",
                            "achieved": ev3d["stream_tflops"], "peak": peak, "unit": "TFLOP/s",
                            "frac": ev3d["stream_tflops"] / peak,
                            "peak_source": "measured FP32 FMA probe on this GPU",
                            "frac_of_issue_peak": ev3d["stream_tflops"] / issue_peak(torch, local, clocks),
                            "flops_per_sample": FLOPS_PER_SAMPLE_3D_BARYON,
                            "reference_form_frac": ev3d["reference_form_tflops"] / peak}

    files = None
    if rank == 0 and world == 1 and not args.no_cpu:
        files = output_files(F, W, ctx)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        rate, kind, sample = cpu_baseline(events, nthreads, budget_s=40.0)
        # the same on one thread, with the same budget (the reference's OpenMP
        # loops gain little on events of this size)
        rate1, _, sample1 = cpu_baseline(events, 1, budget_s=40.0)
        cpu = {"value": rate, "unit": "events/s", "cores": nthreads, "kind": kind, "sample": sample,
               "single_thread": {"value": rate1, "sample": sample1}, "cpu_model": cpu_model()}

    launches_per_step = 4  # prep lines, prep pack, stream2d, landau (2D-only batch)
    if rank == 0:
        sm = sorted(step_ms)
        line = {
            "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": config_of(args),
            "setup": {"events_per_step": n, "ranks": world, "parallelism": f"replicas{world}",
                      "cell_momentum_samples_per_step": samples,
                      "autotuned_window_bytes": tuning["window_bytes"],
                      "autotuned_buckets": bucket_choice},
            "p50_step_ms": sm[len(sm) // 2], "p99_step_ms": sm[min(len(sm) - 1, int(0.99 * len(sm)))],
            "plain_events_per_s": plain,
            "batched_over_plain": (value / plain) if plain else None,
            "samples_per_s": samples * world * args.steps / (t_ms / 1e3),
            "roofline": {"bound": "fp32", "kernel": "fsm_stream2d_kernel", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": "measured FP32 FMA probe on this GPU (fsm_probe_fp32_tflops)",
                         "issue_peak": issue_peak(torch, local, clocks),
                         "frac_of_issue_peak": achieved / issue_peak(torch, local, clocks),
                         "flops_per_sample": FLOPS_PER_SAMPLE_2D, "samples_per_launch": samples,
                         "launch_ms": stream_ms,
                         "traffic": TRAFFIC_BYTES_PER_SAMPLE_2D * samples,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                           "launch on the first 128 events, scaled by samples"},
            "kernel_ms_per_step": {"prep": tm["prep_ms"] / args.steps,
                                   "stream": tm["stream_ms"] / args.steps,
                                   "landau": tm["landau_ms"] / args.steps},
            "other_kernels": other_kernels(tm, args.steps, cells_per_step),
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "events/s", "h2d_bytes_per_step": batch.in_bytes,
                    "d2h_bytes_per_step": d2h_bytes, "d2h_fields": e2e_groups,
                    "d2h_omitted": "u^eta, pi^{tau eta}, pi^{x eta}, pi^{y eta} (zero by "
                                   "boost invariance)",
                    "pipeline": "2 batches on 2 streams, alternating steps; device gather "
                                "+ one copy per step"},
            "fresh_event_set": {"batch_create_ms": create_ms, "first_batch_create_ms": create_cold_ms,
                                "e2e_events_per_s_with_create": world * n / (
                                    e2e_ms / args.steps / 1e3 + create_ms / 1e3),
                                "note": "fsm_batch_create on a new 512-event list (host planning on "
                                        "the worker pool, table upload) after another batch was "
                                        "destroyed (its allocations reused); first: with fresh "
                                        "allocations; e2e above replays one planned batch"},
            "gpu_launches": launches_per_step * args.steps,
            "output_files": files,
            "served": served,
            "served_2d": served_2d,
            "event_3d": ev3d,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    tb.close()
    tctx.close()
    batch.close()
    ctx.close()
    reps.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
