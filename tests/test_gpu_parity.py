"""GPU parity tests: the sm_100a path through the C ABI against the reference's
float results (golden fixtures made from the reference sources), the oracle's
float restatement and its FP64 run.  Tolerances are defined in fsm_testutil."""
import numpy as np
import pytest

import fsm_b200 as F
import oracle_py as O
import workloads as W
from fsm_testutil import (compare, compare_parity, fsm_params, golden_names, load_golden,
                          oracle_params)

pytestmark = pytest.mark.gpu


def _oracle(p_fsm, e, nB=None, fp64=False):
    po = O.Params(**p_fsm.as_dict())
    return O.run(po, e, nB=nB, fp64=fp64)


@pytest.mark.parametrize("name", golden_names())
def test_gpu_matches_reference_fixture(ctx, name):
    d, e, nB, ref, meta = load_golden(name)
    p = fsm_params(d)
    got = ctx.run_event(p, e, nB)
    assert got["info"]["dim_phip"] == int(meta[0])
    assert got["info"]["tau"] == pytest.approx(float(meta[2]))
    # the FP64 precision oracle (the reference's sample set, FP64 values)
    ref64 = O.run(oracle_params(d), e, nB=nB, fp64=2)
    errs, rescued, cells, residual = compare_parity(got, ref, ref64, meta[2], baryon=bool(d["BARYON"]))
    errs64 = compare(got, ref64, meta[2], baryon=bool(d["BARYON"]))
    print(name, "vs reference float:", errs, "rescued (within tolerance of FP64 where the "
          "reference is noisy):", rescued, "of", cells, "residual:", residual, "vs FP64:", errs64)


def test_gpu_gaussian_full_grid(ctx):
    """The plain 2D configuration at full size (101^2, DIM_PHIP=51)."""
    p, e, _ = W.gaussian2d()
    got = ctx.run_event(p, e)
    ref = _oracle(p, e)
    ref64 = _oracle(p, e, fp64=2)
    compare_parity(got, ref, ref64, ref["tau"])
    compare(got, ref64, ref["tau"])


def test_gpu_lumpy_full_grid(ctx):
    """The lumpy 2D configuration at full size (261^2, DIM_PHIP=200, WB EoS)."""
    p, e, _ = W.lumpy2d(seed=1)
    got = ctx.run_event(p, e)
    ref = _oracle(p, e)
    ref64 = _oracle(p, e, fp64=2)
    errs = compare_parity(got, ref, ref64, ref["tau"])
    errs64 = compare(got, ref64, ref["tau"])
    print("lumpy2d vs float", errs, "vs FP64", errs64)


@pytest.mark.parametrize("nx,ny", [(41, 833), (829, 37)])
def test_gpu_long_lines(ctx, nx, ny):
    """Grids with a line longer than the strip kernels stage: the long-line
    spline kernels (both orientations) against the oracle."""
    p, e, _ = W.lumpy2d(seed=7, side=41, dx=0.08, nphip=64, dtau=0.6, eos=1, radius=1.2)
    p.DIM_X, p.DIM_Y = nx, ny
    F.lib().fsm_params_derive(p)
    rng = np.random.default_rng(8)
    x, y = W.axis(nx, p.DX), W.axis(ny, p.DY)
    e = W.hotspots(rng, x, y, radius=1.2).astype(np.float32).ravel()
    got = ctx.run_event(p, e)
    ref = _oracle(p, e)
    ref64 = _oracle(p, e, fp64=2)
    compare_parity(got, ref, ref64, ref["tau"])
    compare(got, ref64, ref["tau"])


def test_gpu_many_phi_nodes(ctx):
    """DIM_PHIP far above one staged run (2000 phi_p: 32 runs of the table)."""
    p, e, _ = W.lumpy2d(seed=21, side=61, dx=0.08, nphip=2000, dtau=0.7, eos=1, radius=1.5)
    got = ctx.run_event(p, e)
    assert got["info"]["dim_phip"] == 2000
    ref = _oracle(p, e)
    ref64 = _oracle(p, e, fp64=2)
    compare_parity(got, ref, ref64, ref["tau"])
    errs = compare(got, ref64, ref["tau"])
    print(f"2000 phi_p vs FP64: {errs}")


def test_gpu_2d_baryon(ctx):
    """Boost-invariant event with baryon charge: J^mu from the charge pass
    (spline of the first rapidity slice, per-slice bilinear fallback)."""
    p, e, nB = W.lumpy2d_baryon(seed=13, side=81, dx=0.08, nphip=48, dtau=0.7, nrap=5)
    got = ctx.run_event(p, e, nB)
    ref = _oracle(p, e, nB)
    ref64 = _oracle(p, e, nB, fp64=2)
    errs = compare_parity(got, ref, ref64, ref["tau"], baryon=True)
    errs64 = compare(got, ref64, ref["tau"], baryon=True)
    print("baryon2d vs float", errs, "vs FP64", errs64)


def _report(name, got, ref, ref64, tau, baryon=False, strict=True):
    errs, rescued, cells, residual = compare_parity(got, ref, ref64, tau, baryon=baryon)
    # the strict FP64 contract; for the extreme 2D shapes on T and Pi, and e
    # norm-wise (relative to T^{tau tau}: in their nearly light-like fringe
    # cells e is ~T^{tau tau}/20, and u and pi there fall under the bounded
    # residual of compare_parity)
    if strict:
        errs64 = compare(got, ref64, tau, baryon=baryon)
    else:
        errs64 = compare(got, ref64, tau, what=("T", "e", "Pi"), baryon=baryon, e_normwise=True)
    print(f"{name}: vs reference float {errs}; rescued {rescued} of {cells}; residual {residual}; "
          f"vs FP64 {errs64}")
    return errs64


def test_gpu_3d_baryon_full_size(ctx):
    """The 3D configuration with baryon charge at full size: 131 x 131 x 51
    cells, 21 tan-map rapidities, DIM_PHIP 100, DTAU 0.8 (875,211 cells, 1.84 G
    reference-equivalent samples), against the oracle's float run and its FP64
    precision run."""
    p, e, nB = W.baryon3d()
    assert (p.DIM_X, p.DIM_Y, p.DIM_ETA, p.DIM_RAP, p.DIM_PHIP) == (131, 131, 51, 21, 100)
    got = ctx.run_event(p, e, nB)
    ref = _oracle(p, e, nB)
    ref64 = _oracle(p, e, nB, fp64=2)
    assert got["info"]["dim_phip"] == ref["dim_phip"] == 100
    _report("baryon3d 131^2x51", got, ref, ref64, ref["tau"], baryon=True)


def _extreme_events():
    """The corners of the batched configuration's parameter ranges: the
    largest grid at the finest spacing and longest DTAU (the arc-length rule
    raises DIM_PHIP 64 -> 189; the widest staged windows), the smallest event,
    a mid-size one, and the largest sample count (301^2, DIM_PHIP 200)."""
    return [W.lumpy2d(seed=5, side=301, dx=0.05, nphip=64, dtau=1.5, eos=2, radius=6.0),
            W.lumpy2d(seed=6, side=101, dx=0.1, nphip=64, dtau=0.3, eos=1, radius=3.0),
            W.lumpy2d(seed=7, side=201, dx=0.075, nphip=100, dtau=0.9, eos=2, radius=5.0),
            W.lumpy2d(seed=8, side=301, dx=0.05, nphip=200, dtau=1.5, eos=1, radius=6.0),
            W.lumpy2d(seed=9, side=151, dx=0.1, nphip=64, dtau=1.5, eos=1, radius=4.0)]


def test_gpu_batch_extreme_shapes(ctx):
    """One batch holding the extreme shapes of the 512-event configuration:
    every event against the oracle's float and FP64 runs, and bit for bit
    against its own single-event result."""
    evs = _extreme_events()
    b = F.Batch(ctx, [p for p, _, _ in evs])
    assert b.info(0)["dim_phip"] == 189
    outs = b.run_host([(e, nB) for _, e, nB in evs])
    b.close()
    for (p, e, _), got in zip(evs, outs):
        ref = _oracle(p, e)
        ref64 = _oracle(p, e, fp64=2)
        got["info"] = {"tau": ref["tau"]}
        _report(f"{p.DIM_X}^2 dx {p.DX:.3f} dtau {p.DTAU:.2f} phi {ref['dim_phip']}", got, ref, ref64,
                ref["tau"], strict=False)
        single = ctx.run_event(p, e)
        for k in ("T", "e", "P", "Pi", "u", "pi"):
            assert np.array_equal(got[k], single[k]), k


def test_gpu_3d_baryon_reduced(ctx):
    """3D + baryon path on a reduced grid the oracle runs in seconds."""
    p, e, nB = W.baryon3d(seed=5, side=41, neta=21, nrap=21, nphip=40)
    got = ctx.run_event(p, e, nB)
    ref = _oracle(p, e, nB)
    ref64 = _oracle(p, e, nB, fp64=2)
    compare_parity(got, ref, ref64, ref["tau"], baryon=True)
    compare(got, ref64, ref["tau"], baryon=True)


def test_batch_equals_single_events(ctx):
    """Every event of a mixed 2D/3D batch equals its single-event result bit for bit."""
    evs = []
    for name in golden_names():
        d, e, nB, _, _ = load_golden(name)
        evs.append((fsm_params(d), e, nB))  # E_DEP_FS events included
    b = F.Batch(ctx, [p for p, _, _ in evs])
    outs = b.run_host([(e, nB) for _, e, nB in evs])
    for (p, e, nB), o in zip(evs, outs):
        s = ctx.run_event(p, e, nB)
        for k in o:
            d = np.abs(o[k] - s[k])
            assert np.array_equal(o[k], s[k]), (k, p.DIM_X, p.DIM_Y, p.DIM_ETA, int(np.count_nonzero(d)),
                                                float(d.max()))
    # a second launch (graph replay) gives the same results
    outs2 = b.run_host([(e, nB) for _, e, nB in evs])
    for o, o2 in zip(outs, outs2):
        for k in o:
            assert np.array_equal(o[k], o2[k])
    b.close()


def test_batches_on_recycled_allocations(ctx):
    """A context keeps the allocations of a destroyed batch for its next one:
    a batch built on that memory (after another batch wrote its own data into
    it) gives the same results as one built on fresh memory."""
    a = W.lumpy2d(seed=40, side=101, dx=0.08, nphip=64, dtau=0.7, eos=1, radius=3.0)
    b = W.lumpy2d(seed=41, side=81, dx=0.07, nphip=100, dtau=1.1, eos=2, radius=2.5)
    c = F.Context(0)
    try:
        fresh = F.Batch(c, [b[0], a[0]])
        want = fresh.run_host([(b[1], None), (a[1], None)])
        big = F.Batch(c, [a[0], a[0], b[0]])
        big.run_host([(a[1], None), (a[1], None), (b[1], None)])
        fresh.close()
        big.close()  # the larger allocations go to the context
        again = F.Batch(c, [b[0], a[0]])
        got = again.run_host([(b[1], None), (a[1], None)])
        again.close()
        for w, g in zip(want, got):
            for k in w:
                assert np.array_equal(w[k], g[k]), k
    finally:
        c.close()


def test_energy_bookkeeping_on_device(ctx):
    """The reference's total energies before and after streaming and the part
    inside E_FREEZE (src/FreestreamMilne.cpp:349-354, 531-545), summed on the
    device per event in the reference's cell order: equal bit for bit to
    sequential float32 sums of the same fields with the reference's volume
    factors (2D and 3D events, an E_DEP_FS event among them)."""
    evs = []
    for name in golden_names():
        d, e, nB, _, _ = load_golden(name)
        evs.append((fsm_params(d), e, nB))
    b = F.Batch(ctx, [p for p, _, _ in evs])
    outs = b.run_host([(e, nB) for _, e, nB in evs])
    got = b.energy()
    f32 = np.float32
    hbarc = f32(0.197326938)
    for i, ((p, e, _), o, g) in enumerate(zip(evs, outs, got)):
        info = b.info(i)
        tau = f32(info["tau"])
        e_fm4 = (np.asarray(e, f32) * f32(1.0) / hbarc + f32(1e-7)).astype(f32)
        t00 = np.asarray(o["T"], f32)[0]
        inside = np.where(np.asarray(o["e"], f32) * hbarc > f32(p.E_FREEZE), t00, f32(0))
        seq = lambda a: np.cumsum(a.astype(f32), dtype=f32)[-1]
        dx, dy, de = f32(p.DX), f32(p.DY), f32(p.DETA)
        if p.DIM_ETA > 1:
            vb = f32(f32(f32(f32(p.TAU0) * dx) * dy) * de)
            va = f32(f32(f32(tau * dx) * dy) * de)
        else:
            vb = f32(dx * dy)
            va = f32(f32(tau * dx) * dy)
        want = dict(before=f32(seq(e_fm4) * vb), after=f32(seq(t00) * va), inside=f32(seq(inside) * va))
        for k, v in want.items():
            assert f32(g[k]) == v, (i, k, g[k], v)
        assert f32(g["fraction"]) == f32(want["inside"] / want["after"])
    b.close()


def test_grouped_batch_downloads(ctx):
    """A batch with grouped outputs gives the same results as a per-event one,
    and download_groups copies back exactly the groups asked for."""
    evs = []
    for name in golden_names():
        d, e, nB, _, _ = load_golden(name)
        evs.append((fsm_params(d), e, nB))
    inputs = [(e, nB) for _, e, nB in evs]
    plain = F.Batch(ctx, [p for p, _, _ in evs])
    want = plain.run_host(inputs)
    plain.close()
    b = F.Batch(ctx, [p for p, _, _ in evs], grouped=True)
    got = b.run_host(inputs)
    for w, g in zip(want, got):
        assert sorted(w) == sorted(g)
        for k in w:
            assert np.array_equal(w[k], g[k]), k
    import torch
    groups = ["e", "u", "pi", "nB"]
    nbytes = b.groups_bytes(groups)
    expect = 0
    for p, _, _ in evs:
        dim = p.DIM_X * p.DIM_Y * p.DIM_ETA
        expect += 4 * dim * (1 + 4 + 10 + (1 if p.BARYON else 0))
    assert nbytes == expect
    host = torch.full((nbytes // 4,), np.nan, dtype=torch.float32).pin_memory()
    b.upload(torch.from_numpy(b.pack_inputs(inputs)).pin_memory().data_ptr())
    b.launch()
    b.download_groups(groups, host.data_ptr())
    b.check_errors()
    packed = host.numpy()
    assert not np.isnan(packed).any()
    for ev, w in enumerate(want):
        part = b.unpack_groups(packed, groups, ev)
        assert sorted(part) == sorted(k for k in groups if k in w)
        for k in part:
            assert np.array_equal(part[k], w[k]), (ev, k)
    assert b.offsets(0)[1] == 2**64 - 1  # no per-event output block in a grouped slab
    with pytest.raises(F.FsmError):
        b.group_offset(groups, "T", 0)  # T was not downloaded
    b.close()


@pytest.mark.parametrize("grouped", [False, True])
def test_packed_downloads(ctx, grouped):
    """Packed downloads (device gather + one copy) give the fields of the
    regular download; the components left out for 2D events are zero there."""
    evs = []
    for name in golden_names():
        d, e, nB, _, _ = load_golden(name)
        evs.append((fsm_params(d), e, nB))
    inputs = [(e, nB) for _, e, nB in evs]
    b = F.Batch(ctx, [p for p, _, _ in evs], grouped=grouped)
    want = b.run_host(inputs)
    import torch
    for groups in (["e", "P", "Pi", "u", "pi"], list(F.OUT_GROUPS)):
        for skip in (False, True):
            nbytes = b.packed_bytes(groups, skip)
            host = torch.full((nbytes // 4,), np.nan, dtype=torch.float32).pin_memory()
            b.download_packed(groups, host.data_ptr(), skip)
            b.check_errors()
            packed = host.numpy()
            assert not np.isnan(packed).any()
            for ev, w in enumerate(want):
                got = b.unpack_packed(packed, groups, ev, skip)
                assert sorted(got) == sorted(k for k in groups if k in w)
                for k in got:
                    assert np.array_equal(got[k], w[k]), (grouped, skip, ev, k)
    # the all-offsets call agrees with the one-component query
    offs = b.packed_offsets(list(F.OUT_GROUPS), True)
    for ev in range(b.n):
        for g, k in enumerate(F.OUT_GROUPS):
            for m in range(F.OUT_COMPS[k]):
                one = b.packed_offset(list(F.OUT_GROUPS), k, m, ev, True)
                assert (one if one is not None else -1) == offs[ev, g, m], (ev, k, m)
    full = b.packed_bytes(["u", "pi"])
    less = b.packed_bytes(["u", "pi"], True)
    n2d = sum(p.DIM_X * p.DIM_Y for p, _, _ in evs if p.DIM_ETA == 1)
    assert full - less == 4 * 4 * n2d  # u^eta, pi^{tau eta}, pi^{x eta}, pi^{y eta}
    b.close()


def test_device_entry_point(ctx):
    import torch
    p, e, _ = W.lumpy2d(seed=9, side=101, dx=0.08, nphip=64, dtau=0.7)
    dim = e.size
    d_e = torch.from_numpy(e).cuda()
    outs = {k: torch.zeros((F.OUT_COMPS[k] * dim,), dtype=torch.float32, device="cuda")
            for k in ("T", "e", "P", "Pi", "u", "pi")}
    stream = torch.cuda.current_stream().cuda_stream
    ctx.run_event_device(p, d_e.data_ptr(), None, {k: v.data_ptr() for k, v in outs.items()},
                         stream=stream)
    torch.cuda.synchronize()
    host = ctx.run_event(p, e)
    for k, v in outs.items():
        assert np.array_equal(v.cpu().numpy().reshape(host[k].shape), host[k]), k


def test_energy_dependent_tau(ctx):
    d, e, nB, ref, meta = load_golden("edepfs2d_45")
    got = ctx.run_event(fsm_params(d), e)
    assert got["info"]["dtau"] == pytest.approx(float(meta[1]), rel=0, abs=0)
    compare_parity(got, ref, O.run(oracle_params(d), e, fp64=2), meta[2])


def test_energy_dependent_tau_in_batches(ctx):
    """E_DEP_FS events inside a batch built before its inputs exist: each
    launch takes the profiles' sums on the device and plans with the resulting
    DTAU, so the batch reproduces the reference's DTAU and outputs (parity with
    the golden fixture), equals the one-event path bit for bit, and re-plans
    when a new profile changes DTAU."""
    d, e, nB, ref, meta = load_golden("edepfs2d_45")
    p = fsm_params(d)
    other = W.lumpy2d(seed=3, side=61, dx=0.08, nphip=48, dtau=0.6, eos=2, radius=2.0)
    b = F.Batch(ctx, [p, other[0], p])
    e2 = (e * np.float32(1.7)).astype(np.float32)  # a second profile: another DTAU
    outs = b.run_host([(e, None), (other[1], None), (e2, None)])
    assert b.info(0)["dtau"] == float(meta[1])
    assert b.info(2)["dtau"] != b.info(0)["dtau"]
    compare_parity(outs[0], ref, O.run(oracle_params(d), e, fp64=2), meta[2])
    for got, (pp, ee) in zip(outs, [(p, e), (other[0], other[1]), (p, e2)]):
        single = ctx.run_event(pp, ee)
        for k in ("T", "e", "P", "Pi", "u", "pi"):
            assert np.array_equal(got[k], single[k]), k
    # a launch with the profiles swapped re-plans and still matches
    outs2 = b.run_host([(e2, None), (other[1], None), (e, None)])
    for k in ("T", "e", "u", "pi"):
        assert np.array_equal(outs2[0][k], outs[2][k]) and np.array_equal(outs2[2][k], outs[0][k])
    b.close()


def test_energy_dependent_tau_device_entry(ctx):
    """E_DEP_FS with a device-resident profile: the device sums reproduce the
    reference's float running sums, so DTAU and every output match the host
    entry point's (and the reference's DTAU) exactly."""
    import torch
    d, e, nB, ref, meta = load_golden("edepfs2d_45")
    p = fsm_params(d)
    host = ctx.run_event(p, e)
    dim = e.size
    d_e = torch.from_numpy(np.ascontiguousarray(e)).cuda()
    outs = {k: torch.zeros((F.OUT_COMPS[k] * dim,), dtype=torch.float32, device="cuda")
            for k in ("T", "e", "P", "Pi", "u", "pi")}
    info = ctx.run_event_device(p, d_e.data_ptr(), None, {k: v.data_ptr() for k, v in outs.items()},
                                stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert info["dtau"] == float(meta[1]) == host["info"]["dtau"]
    for k, v in outs.items():
        assert np.array_equal(v.cpu().numpy().reshape(host[k].shape), host[k]), k


@pytest.mark.parametrize("case", ["lumpy2d", "baryon3d"])
def test_gpu_diagnostics(ctx, case):
    """Hydro-validity and vorticity fields on the GPU against the oracle's
    restatement (itself bit-exact with the reference's functions) on the same
    matched fields."""
    if case == "lumpy2d":
        p, e, nB = W.lumpy2d(seed=2, side=91, dx=0.08, nphip=64, dtau=0.8, eos=2, radius=3.0)
    else:
        p, e, nB = W.baryon3d(seed=5, side=31, neta=15, nrap=11, nphip=24)
    got = ctx.run_event(p, e, nB)
    dg = ctx.diagnostics(p, got)
    po = O.Params(**p.as_dict())
    po.DIM = p.DIM_X * p.DIM_Y * p.DIM_ETA
    ref = O.diagnostics(po, got["info"]["tau"], got["e"], got["P"], got["Pi"], got["u"], got["pi"])
    off = 0
    for k, c in F.DIAG_COMPS.items():
        a = np.asarray(dg[k], np.float32).reshape(c, -1)
        b = ref[off:off + c]
        off += c
        if k in ("beta", "omega"):  # powf of the temperature may differ by an ulp
            scale = np.abs(b).max() + 1e-30
            assert np.max(np.abs(a - b)) <= 1e-5 * scale, k
        else:
            np.testing.assert_array_equal(a, b, err_msg=k)


def test_autotune_keeps_results():
    """The autotuner only changes launch shapes: results with the tuned window
    equal those with the default, bit for bit."""
    evs = [W.lumpy2d(seed=30 + k, side=81 + 20 * k, dx=0.07, nphip=64, dtau=0.5 + 0.4 * k,
                     eos=1 + k % 2, radius=2.5) for k in range(3)]
    base = F.Context(0)
    ref = [base.run_event(p, e) for p, e, _ in evs]
    base.close()
    c = F.Context(0)
    t = c.autotune([p for p, _, _ in evs], [(e, nb) for _, e, nb in evs])
    assert 20 * 1024 <= t["window_bytes"] <= 48 * 1024 and t["ms"] > 0
    for k in (20 * 1024, 48 * 1024):  # 20 KB: the planner raises it where runs would be too many
        c.set_tuning(k)
        for (p, e, _), r in zip(evs, ref):
            got = c.run_event(p, e)
            for name in ("T", "e", "u", "pi"):
                np.testing.assert_array_equal(got[name], r[name], err_msg=f"{k} {name}")
    c.close()


def test_bucket_autotuner_choices_keep_results(tmp_path):
    """Every choice the per-bucket autotuner can make (windows of 24-40 KB,
    the 16-phi_p chunk, narrow tail tiles or 32 x 32 tiles only) gives the
    untuned results bit for bit; the 32-phi_p chunk a caller may set (a
    different summation order, not chosen by the tuner) passes the parity
    checks against the reference's float output and T and Pi against FP64.
    The tuned table survives a save / load round trip."""
    evs = [W.lumpy2d(seed=50, side=101, dx=0.1, nphip=64, dtau=0.4, eos=1, radius=3.0),   # 0, 0
           W.lumpy2d(seed=51, side=151, dx=0.08, nphip=100, dtau=1.0, eos=2, radius=4.0),  # 1, 1
           W.lumpy2d(seed=52, side=201, dx=0.05, nphip=64, dtau=1.0, eos=1, radius=4.0)]   # 2, 2
    base = F.Context(0)
    ref = [base.run_event(p, e) for p, e, _ in evs]
    base.close()
    c = F.Context(0)
    try:
        table = c.autotune_buckets([p for p, _, _ in evs], [(e, nb) for _, e, nb in evs])
        tuned = [k for k, t in enumerate(table) if t["window_bytes"]]
        assert sorted(tuned) == [0, 5, 10], tuned
        for t in table:
            if t["window_bytes"]:
                assert 24 * 1024 <= t["window_bytes"] <= 40 * 1024
                assert t["phi_chunk"] == 16 and t["ms"] > 0 and t["events"] == 1
                assert t["tile_shapes"] in (F.TILES_TAIL, F.TILES_SQUARE)
        path = tmp_path / "tuning.txt"
        c.save_tuning(path)
        c2 = F.Context(0)
        c2.load_tuning(path)
        for window in (24 * 1024, 28 * 1024, 32 * 1024, 36 * 1024, 40 * 1024):
            for chunk, tiles in ((16, F.TILES_TAIL), (16, F.TILES_SQUARE), (32, F.TILES_TAIL)):
                if chunk == 32 and window != 40 * 1024:
                    continue
                c2.set_tuning_buckets([{"window_bytes": window, "phi_chunk": chunk,
                                        "tile_shapes": tiles}] * 16)
                for (p, e, _), r in zip(evs, ref):
                    got = c2.run_event(p, e)
                    if chunk == 16:
                        for name in ("T", "e", "u", "pi"):
                            np.testing.assert_array_equal(got[name], r[name],
                                                          err_msg=f"{window} {tiles} {name}")
                    else:
                        o = _oracle(p, e)
                        o64 = _oracle(p, e, fp64=2)
                        compare_parity(got, o, o64, o["tau"])
                        compare(got, o64, o["tau"], what=("T", "Pi"))
        c2.close()
    finally:
        c.close()


@pytest.mark.parametrize("case", ["ic1_2d", "ic1_3d_baryon", "ic1_2d_edepfs"])
def test_initial_conditions_in_fm4(ctx, case):
    """The reference's own initial conditions (here the smooth elliptical
    Gaussian, IC_ENERGY = 1) are in fm^-4 and used as they are: through
    fsm_run_event_fm4 against the oracle fed the same profile (its fm^-4 mode
    is bit-exact with the reference's sources), float and FP64 runs; with
    E_DEP_FS the free-streaming time comes from the raw profile as well."""
    if case == "ic1_2d":
        p = F.default_params(DIM_X=61, DIM_Y=55, DX=0.4, DY=0.4, DIM_PHIP=48, DTAU=1.5, TAU0=0.5,
                             IC_ENERGY=1, EOS_TYPE=2)
    elif case == "ic1_3d_baryon":
        p = F.default_params(DIM_X=31, DIM_Y=29, DIM_ETA=11, DX=0.4, DY=0.4, DETA=0.4, DIM_RAP=9,
                             DIM_PHIP=24, DTAU=1.0, TAU0=0.5, IC_ENERGY=1, BARYON=1, IC_BARYON=1)
    else:
        p = F.default_params(DIM_X=61, DIM_Y=55, DX=0.4, DY=0.4, DIM_PHIP=48, DTAU=1.5, TAU0=0.5,
                             IC_ENERGY=1, E_DEP_FS=1, TAU_R=0.8, E_R=4.0, ALPHA=0.25)
    e = F.initial_profile(p, "energy")
    nB = F.initial_profile(p, "baryon") if p.BARYON else None
    got = ctx.run_event(p, e, nB, fm4=True)
    po = O.Params(**p.as_dict())
    ref = O.run(po, e, nB=nB, fm4=True)
    ref64 = O.run(po, e, nB=nB, fm4=True, fp64=2)
    assert got["info"]["dim_phip"] == ref["dim_phip"]
    assert got["info"]["dtau"] == pytest.approx(ref["dtau"], rel=0, abs=0)
    compare_parity(got, ref, ref64, ref["tau"], baryon=bool(p.BARYON))
    compare(got, ref64, ref["tau"], baryon=bool(p.BARYON))


def test_invalid_inputs_are_rejected(ctx):
    p = F.default_params(DIM_X=3)
    with pytest.raises(F.FsmError):
        ctx.run_event(p, np.zeros(3 * 101, np.float32))
    p = F.default_params(DIM_ETA=5, DIM_RAP=1, DETA=0.2)
    with pytest.raises(F.FsmError) as ei:
        ctx.run_event(p, np.zeros(101 * 101 * 5, np.float32))
    assert ei.value.status == 4


def test_narrow_tail_tiles_keep_results():
    """A batch large enough for the narrow tail tiles (64 x 16, 128 x 8,
    256 x 4, 16 x 64, 8 x 128, 4 x 256 over partial last strips) gives, bit for
    bit, the results of 32 x 32 tiles only; every remainder shape is covered."""
    evs = [W.lumpy2d(seed=60, side=301, dx=0.05, nphip=64, dtau=1.2, eos=1, radius=5.0),   # 13: 64x16, 16x64
           W.lumpy2d(seed=61, side=261, dx=0.06, nphip=100, dtau=0.8, eos=2, radius=5.0),  # 5: 128x8, 8x128
           W.lumpy2d(seed=62, side=301, dx=0.1, nphip=64, dtau=0.5, eos=2, radius=6.0),
           W.lumpy2d(seed=63, side=201, dx=0.075, nphip=64, dtau=1.0, eos=1, radius=5.0),  # 9: 64x16, 16x64
           W.lumpy2d(seed=64, side=261, dx=0.05, nphip=64, dtau=0.4, eos=1, radius=4.0),
           W.lumpy2d(seed=65, side=260, dx=0.06, nphip=64, dtau=0.9, eos=2, radius=5.0)]   # 4: 256x4, 4x256
    outs = {}
    for tiles in (F.TILES_TAIL, F.TILES_SQUARE):
        c = F.Context(0)
        try:
            c.set_tuning_buckets([{"window_bytes": 32768, "phi_chunk": 16, "tile_shapes": tiles}] * 16)
            b = F.Batch(c, [p for p, _, _ in evs])
            outs[tiles] = b.run_host([(e, None) for _, e, _ in evs])
            b.close()
        finally:
            c.close()
    for o, q in zip(outs[F.TILES_TAIL], outs[F.TILES_SQUARE]):
        for k in ("T", "e", "P", "Pi", "u", "pi"):
            assert np.array_equal(o[k], q[k]), k


def test_host_path_pinned_and_pageable_buffers(ctx):
    """The one-event host path copies pageable caller buffers through pinned
    chunks (several chunks for a 3D event's outputs) and pinned ones
    directly: both give the device entry point's results bit for bit."""
    import torch
    p, e, nb = W.baryon3d(seed=11, side=101, neta=21, nrap=11, nphip=32)
    pageable = ctx.run_event(p, e, nb)
    dim = p.DIM_X * p.DIM_Y * p.DIM_ETA
    assert 10 * dim * 4 > 8 << 20  # T alone spans several 8 MiB chunks
    pinned = {k: torch.zeros((F.OUT_COMPS[k], dim) if F.OUT_COMPS[k] > 1 else (dim,),
                             dtype=torch.float32).pin_memory().numpy() for k in F.OUT_COMPS}
    e_pin = torch.from_numpy(np.ascontiguousarray(e, dtype=np.float32)).pin_memory().numpy()
    nb_pin = torch.from_numpy(np.ascontiguousarray(nb, dtype=np.float32)).pin_memory().numpy()
    got = ctx.run_event(p, e_pin, nb_pin, into=pinned)
    d_e = torch.from_numpy(np.ascontiguousarray(e, dtype=np.float32)).cuda()
    d_nb = torch.from_numpy(np.ascontiguousarray(nb, dtype=np.float32)).cuda()
    dev = {k: torch.zeros(F.OUT_COMPS[k] * dim, dtype=torch.float32, device="cuda") for k in F.OUT_COMPS}
    ctx.run_event_device(p, d_e.data_ptr(), d_nb.data_ptr(), {k: v.data_ptr() for k, v in dev.items()})
    torch.cuda.synchronize()
    for k in F.OUT_COMPS:
        ref = dev[k].cpu().numpy().reshape(pageable[k].shape)
        assert np.array_equal(pageable[k], ref), k
        assert np.array_equal(got[k], ref), k


def test_cached_3d_plans_give_identical_results():
    """A context caches 3D plans by their parameters: an event planned afresh
    and the same event run again from the cached plan (after another shape
    replaced the context's one-event batch) agree bit for bit."""
    p, e, nB = W.baryon3d(seed=5, side=31, neta=15, nrap=9, nphip=24)
    q, e2, nB2 = W.baryon3d(seed=6, side=25, neta=13, nrap=11, nphip=20)
    c = F.Context(0)
    try:
        first = c.run_event(p, e, nB)
        c.run_event(q, e2, nB2)
        again = c.run_event(p, e, nB)
        for k, v in first.items():
            if isinstance(v, np.ndarray):
                assert np.array_equal(v, again[k]), k
    finally:
        c.close()
