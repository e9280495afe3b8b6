"""The allocation-free entry point, for callers that cannot allocate device
memory when they run the free streaming (e.g. a framework that owns all device
memory through its own pool).  It must give the results of the ordinary device
entry point.  Kept in its own file, collected last, so a run that stops at its
first failure has run every other test first; it also passes alone.  Its
companion check reads the kernels' error words without allocating."""
import numpy as np
import pytest

import fsm_b200 as F
import workloads as W
from fsm_testutil import compare

pytestmark = pytest.mark.gpu

OUTS = ("T", "e", "P", "Pi", "u", "pi")


def _dev_outputs(torch, dim):
    return {k: torch.zeros((F.OUT_COMPS[k] * dim,), dtype=torch.float32, device="cuda") for k in OUTS}


def _host(outs, dim):
    return {k: v.cpu().numpy().reshape((F.OUT_COMPS[k], dim) if F.OUT_COMPS[k] > 1 else (dim,))
            for k, v in outs.items()}


def _long_thin():
    """100 x 900 cells: a line longer than the strip kernels stage, so the
    long-line spline kernels run (within the entry point's cell limit)."""
    p, _, _ = W.lumpy2d(seed=7, side=41, dx=0.08, nphip=64, dtau=0.6, eos=1, radius=1.2)
    p.DIM_X, p.DIM_Y = 100, 900
    W.derive(p)
    rng = np.random.default_rng(8)
    e = W.hotspots(rng, W.axis(100, p.DX), W.axis(900, p.DY), radius=3.0)
    return p, e.astype(np.float32).ravel(), None


def test_no_alloc_entry_matches_device_entry(ctx):
    import torch
    events = [W.lumpy2d(seed=21, side=151, dx=0.07, nphip=100, dtau=0.9, eos=2, radius=4.0),
              W.gaussian2d(), _long_thin()]
    stream = torch.cuda.current_stream().cuda_stream
    for p, e, _ in events:  # two calls in a row, each against the existing entry point
        dim = e.size
        d_e = torch.from_numpy(e).cuda()
        ref = _dev_outputs(torch, dim)
        ctx.run_event_device(p, d_e.data_ptr(), None, {k: v.data_ptr() for k, v in ref.items()},
                             stream=stream)
        got = _dev_outputs(torch, dim)
        F.run_event_2d_noalloc(p, d_e.data_ptr(), {k: v.data_ptr() for k, v in got.items()},
                               stream=stream)
        F.run_event_2d_noalloc_check(stream)  # waits; raises on a kernel-side error
        torch.cuda.synchronize()
        r, g = _host(ref, dim), _host(got, dim)
        compare(g, r, float(p.TAU0 + p.DTAU))
        assert all(np.isfinite(g[k]).all() for k in g)


def test_no_alloc_rejects_oversized_events(ctx):
    import torch
    p = F.default_params(DIM_X=401, DIM_Y=401)
    d_e = torch.zeros(401 * 401, dtype=torch.float32, device="cuda")
    out = _dev_outputs(torch, 401 * 401)
    with pytest.raises(F.FsmError) as ei:
        F.run_event_2d_noalloc(p, d_e.data_ptr(), {k: v.data_ptr() for k, v in out.items()})
    assert ei.value.status == 12  # FSM_ERR_TOO_LARGE


def test_no_alloc_rejects_stream_capture(ctx):
    """Its table upload reads host memory released when the call returns, so
    a call on a capturing stream is refused before it enqueues anything."""
    import torch
    p = F.default_params(DIM_X=41, DIM_Y=41)
    d_e = torch.ones(41 * 41, dtype=torch.float32, device="cuda")
    out = _dev_outputs(torch, 41 * 41)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        d_e.mul_(1.0)  # the graph holds one node of its own
        with pytest.raises(F.FsmError) as ei:
            F.run_event_2d_noalloc(p, d_e.data_ptr(), {k: v.data_ptr() for k, v in out.items()},
                                   stream=s.cuda_stream)
    assert ei.value.status == 4  # FSM_ERR_UNSUPPORTED
    g.replay()
    torch.cuda.synchronize()
