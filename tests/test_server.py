"""The continuous-batching server (fsm_server_*): every request's outputs are
the same alone, in a mixed burst and through the plain per-event entry point;
the memory budget splits waves instead of failing them; a request larger than
the budget fails alone."""
import numpy as np
import pytest

import fsm_b200 as F
import workloads as W


def _mixed_requests():
    reqs = []
    p, e, _ = W.gaussian2d()
    reqs.append((p, e, None))
    p, e, _ = W.lumpy2d(seed=3, side=101, dx=0.08, nphip=64, dtau=0.7, eos=2, radius=3.0)
    reqs.append((p, e, None))
    p, e, _ = W.lumpy2d(seed=4, side=61, dx=0.1, nphip=100, dtau=0.4, eos=1, radius=2.0)
    reqs.append((p, e, None))
    p, e, nb = W.baryon3d(seed=5, side=25, neta=13, nrap=11, nphip=24)
    reqs.append((p, e, nb))
    p, e, _ = W.lumpy2d(seed=6, side=81, dx=0.07, nphip=64, dtau=1.2, eos=2, radius=2.5)
    reqs.append((p, e, None))
    p, e, _ = W.gaussian2d()
    p.E_DEP_FS, p.TAU_R, p.E_R, p.ALPHA = 1, 1.16, 4.0, 0.2
    reqs.append((p, e, None))
    return reqs


def _same(a, b):
    for k in a:
        if k == "info":
            assert a[k]["tau"] == b[k]["tau"] and a[k]["dim_phip"] == b[k]["dim_phip"]
            continue
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_server_needs_a_device():
    if F.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(F.FsmError):
        F.Server()


@pytest.mark.gpu
def test_server_results_alone_in_mix_and_plain(ctx):
    reqs = _mixed_requests()
    srv = F.Server(streams=2)
    try:
        alone = []
        for p, e, nb in reqs:
            rid = srv.submit(p, e, nb)
            alone.append(srv.poll(rid))
        ids = [srv.submit(p, e, nb) for p, e, nb in reqs * 3]   # one burst, repeated events
        mixed = [srv.poll(i) for i in ids]
        st = srv.stats()
    finally:
        srv.stop()
    for k, (p, e, nb) in enumerate(reqs):
        plain = ctx.run_event(p, e, nb)
        _same(alone[k], plain)
        for r in range(3):
            _same(mixed[r * len(reqs) + k], alone[k])
    assert st["completed"] == 4 * len(reqs) and st["failed"] == 0
    assert st["waves"] < 4 * len(reqs)          # the burst shared waves
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]


@pytest.mark.gpu
def test_server_reserved_2d_stream(ctx):
    """With a stream reserved for boost-invariant waves (and 3D events capped
    per wave), a burst of mixed requests -- several 3D ones among them --
    gives every request the plain entry point's outputs."""
    reqs = _mixed_requests()
    p3, e3, nb3 = W.baryon3d(seed=7, side=31, neta=15, nrap=11, nphip=24)
    reqs += [(p3, e3, nb3)] * 3
    srv = F.Server(streams=2, stream_2d=True)
    try:
        ids = [srv.submit(p, e, nb) for p, e, nb in reqs * 2]
        got = [srv.poll(i) for i in ids]
        st = srv.stats()
    finally:
        srv.stop()
    for k, (p, e, nb) in enumerate(reqs * 2):
        _same(got[k], ctx.run_event(p, e, nb))
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0


@pytest.mark.gpu
def test_server_budget_splits_waves_and_rejects_oversize():
    small = [W.lumpy2d(seed=10 + k, side=61, dx=0.1, nphip=64, dtau=0.5, eos=1, radius=2.0)
             for k in range(12)]
    srv = F.Server(hbm_budget=3 << 20, host_budget=3 << 20, streams=2)
    try:
        ids = [srv.submit(p, e) for p, e, _ in small]
        big_p, big_e, _ = W.lumpy2d(seed=99, side=301, dx=0.05, nphip=200, dtau=1.5, eos=1)
        big = srv.submit(big_p, big_e)
        outs = [srv.poll(i) for i in ids]
        with pytest.raises(F.FsmError) as ex:
            srv.poll(big)
        assert ex.value.status == 12  # FSM_ERR_TOO_LARGE
        st = srv.stats()
    finally:
        srv.stop()
    assert all(o is not None for o in outs)
    assert st["completed"] == len(small) and st["failed"] == 1
    assert st["waves"] >= 2


@pytest.mark.gpu
def test_server_output_mask(ctx):
    p, e, _ = W.lumpy2d(seed=21, side=71, dx=0.09, nphip=64, dtau=0.6, eos=2, radius=2.0)
    srv = F.Server(outputs=["e", "u"])
    try:
        got = srv.poll(srv.submit(p, e))
        rid = srv.submit(p, e)
        view = srv.poll_view(rid)
        viewed = {k: np.array(v) for k, v in view.items() if k != "info"}
        srv.release(rid)
    finally:
        srv.stop()
    for k in ("e", "u"):
        np.testing.assert_array_equal(viewed[k], got[k])
    assert set(k for k in got if k != "info") == {"e", "u"}
    plain = ctx.run_event(p, e)
    np.testing.assert_array_equal(got["e"], plain["e"])
    np.testing.assert_array_equal(got["u"], plain["u"])
