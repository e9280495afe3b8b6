"""CPU tests of the host side: the C-ABI library loads and exports every entry
point include/fsm.h declares, parameter handling mirrors the reference, the
library refuses to compute without a GPU, and the Landau-matching algorithm
(compiled for the CPU from the same header the kernel uses) agrees with the
oracle's reference-faithful solver."""
import ctypes
import pathlib
import re

import numpy as np
import pytest

import fsm_b200 as F
import oracle_py as O

ROOT = pathlib.Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "fsm.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fsm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = F.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/fsm.h but not exported"
        assert n in F.SIGNATURES, f"{n} missing from the ctypes binding"


def test_param_struct_layout_matches_reference_order():
    assert [f for f, _ in F.PARAM_FIELDS] == [f for f, _ in O.PARAM_FIELDS]
    assert ctypes.sizeof(F.Params) == ctypes.sizeof(O.Params) == 28 * 4


def test_params_default_match_reference():
    p = F.default_params()
    for k, v in O.DEFAULTS.items():
        if k in ("DIM", "TAU"):
            continue
        assert getattr(p, k) == pytest.approx(v), k
    assert p.DIM == 101 * 101 and p.TAU == pytest.approx(0.6)


def test_python_params_match_library():
    """The library-free parameter block (used by the workload generators, so
    that the CPU reference timing never loads libfsm.so) has the library's
    defaults and derives DIM and TAU bit for bit like fsm_params_derive."""
    import fsm_params as FP
    assert F.Params is FP.Params
    a, b = F.default_params(), FP.default_params()
    assert bytes(a) == bytes(b)
    rng = np.random.default_rng(0)
    for _ in range(200):
        kw = dict(DIM_X=int(rng.integers(4, 400)), DIM_Y=int(rng.integers(4, 400)),
                  DIM_ETA=int(rng.integers(1, 60)), TAU0=float(rng.uniform(0.01, 2.0)),
                  DTAU=float(rng.uniform(0.0, 3.0)))
        a, b = F.default_params(**kw), FP.default_params(**kw)
        assert bytes(a) == bytes(b)


def test_params_positional_file(tmp_path):
    # keys are ignored: only the position of each value matters (src/FileIO.cpp:166-245)
    vals = ["2", "1", "5", "3", "0.7", "2.5", "0.9", "1.1", "31", "29", "7", "5", "33", "0.12",
            "0.13", "0.2", "0.25", "0.75", "0.3", "2", "1.9", "0", "0", "3.0", "0.8", "0.5"]
    text = "".join(f"KEY{i}\t{v}\n" for i, v in enumerate(vals))
    f = tmp_path / "freestream_input"
    f.write_text(text)
    p = F.read_params_file(f)
    assert (p.OUTPUTFORMAT, p.BARYON, p.IC_ENERGY, p.IC_BARYON) == (2, 1, 5, 3)
    assert (p.DIM_X, p.DIM_Y, p.DIM_ETA, p.DIM_RAP, p.DIM_PHIP) == (31, 29, 7, 5, 33)
    assert p.DX == pytest.approx(0.12) and p.DTAU == pytest.approx(0.75)
    assert p.EOS_TYPE == 2 and p.VISCOUS_MATCHING == 0 and p.ALPHA == pytest.approx(0.5)
    assert p.DIM == 31 * 29 * 7 and p.TAU == pytest.approx(0.3 + 0.75)


def test_params_missing_file_reports_file_error(tmp_path):
    p = F.default_params()
    st = F.lib().fsm_params_read_file(str(tmp_path / "nope").encode(), ctypes.byref(p))
    assert st == 8  # FSM_ERR_FILE, defaults untouched
    assert p.DIM_X == 101


def test_status_strings():
    for code in F.STATUS:
        assert F.lib().fsm_status_str(code)


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = F.lib().fsm_ctx_create(ctypes.byref(h), None)
    assert st == 6  # FSM_ERR_NO_DEVICE: the library never computes on the CPU


def test_batch_download_entry_points_reject_null_batches():
    L = F.lib()
    assert L.fsm_batch_create_ex(None, 1, None, 0, None) == 1  # FSM_ERR_INVALID_ARG
    assert L.fsm_batch_download_groups(None, 1, None, None) == 1
    assert L.fsm_batch_download_packed(None, 1, F.PACK_SKIP_ETA, None, None) == 1
    assert L.fsm_batch_packed_offset(None, 1, 0, 0, 0, 0, None) == 1
    assert L.fsm_batch_packed_offsets(None, 1, 0, None, 0) == 1
    assert L.fsm_batch_group_offset(None, 1, 0, 0, None) == 1
    assert L.fsm_batch_groups_bytes(None, 1) == 0 and L.fsm_batch_packed_bytes(None, 1, 0) == 0


def test_parallel_planning_matches_serial():
    """The planner's tables are identical whether the worker pool plans the
    eta slices of a 3D event in parallel or one thread plans them."""
    import workloads as W
    L = ctypes.CDLL(str(ROOT / "freestream-milne_b200" / "_build" / "libfsm_hosttest.so"))
    L.fsm_hosttest_plan_digest.argtypes = [ctypes.POINTER(F.Params), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_ulonglong)]
    cases = [W.baryon3d(seed=1, side=41, neta=51, nrap=41)[0],
             W.baryon3d(seed=2, side=31, neta=25, nrap=21, nphip=40)[0],
             W.lumpy2d(seed=3, side=61, nphip=300)[0]]
    for p in cases:
        d = []
        for serial in (1, 0, 0):
            h = ctypes.c_ulonglong()
            assert L.fsm_hosttest_plan_digest(ctypes.byref(p), serial, ctypes.byref(h)) == 0
            d.append(h.value)
        assert d[0] == d[1] == d[2], (p.DIM_ETA, p.DIM_RAP, d)


SHAPE_TX = {0: 32, 1: 64, 2: 128, 3: 16, 4: 8, 5: 4, 6: 256}
SHAPE_TY = {0: 32, 1: 16, 2: 8, 3: 64, 4: 128, 5: 256, 6: 4}


def test_tiles_cover_every_cell_once():
    """The 2D tiling -- 32 x 32 tiles plus the narrow shapes over partial last
    strips -- covers every cell of the grid exactly once, plans runs for every
    shape it uses, keeps each run's staged window inside the kernel's largest,
    and needs no more tiles (each 1024 cells of work) than 32 x 32 tiles alone."""
    import numpy as np
    import workloads as W
    L = ctypes.CDLL(str(ROOT / "freestream-milne_b200" / "_build" / "libfsm_hosttest.so"))
    L.fsm_hosttest_tiles.argtypes = [ctypes.POINTER(F.Params), ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    cap = 4096
    buf = np.zeros(5 * cap, np.int32)
    nch = np.zeros(7, np.int32)
    box = ctypes.c_int()
    sides = [(5, 7), (9, 40), (31, 33), (32, 32), (41, 41), (45, 41), (101, 101),
             (151, 151), (201, 261), (301, 301), (100, 900), (263, 17), (8, 300), (131, 131),
             (36, 260), (260, 36), (68, 100)]
    for nx, ny in sides:
        p, _, _ = W.lumpy2d(seed=3, side=41, dx=0.08, nphip=64, dtau=0.9, eos=1, radius=1.0)
        p.DIM_X, p.DIM_Y = nx, ny
        W.derive(p)
        slots = {}
        for tail in (1, 0):
            n = L.fsm_hosttest_tiles(ctypes.byref(p), tail, 32768, buf.ctypes.data, cap,
                                     nch.ctypes.data, ctypes.byref(box))
            assert 0 < n <= cap, (nx, ny, n)
            cover = np.zeros((nx, ny), np.int32)
            t = buf[:5 * n].reshape(n, 5)
            for x0, y0, sh, x1, y1 in t:
                tx, ty = SHAPE_TX[int(sh)], SHAPE_TY[int(sh)]
                assert x0 < x1 <= nx and y0 < y1 <= ny, (nx, ny, x0, y0, sh, x1, y1)
                cover[x0:min(x0 + tx, x1), y0:min(y0 + ty, y1)] += 1  # the cells the tile stores
                assert nch[sh] > 0, (nx, ny, sh)
            assert (cover == 1).all(), (nx, ny, tail, int(cover.min()), int(cover.max()))
            if not tail:
                assert set(t[:, 2].tolist()) == {0}
            assert box.value * 16 <= 96 * 1024
            slots[tail] = n * 1024
        assert slots[1] <= slots[0], (nx, ny, slots)


def _host_landau():
    L = ctypes.CDLL(str(ROOT / "freestream-milne_b200" / "_build" / "libfsm_hosttest.so"))
    L.fsm_hosttest_landau_cell.argtypes = ([ctypes.c_void_p] * 2 + [ctypes.c_int] * 4 +
                                           [ctypes.c_float, ctypes.c_void_p])
    return L


def _boosted_fluid(rng, is3d, tau):
    e = 10 ** rng.uniform(-3, 2)
    P = e * rng.uniform(0, 1, 3) * (1 if rng.random() < 0.8 else 0.01)
    rap = rng.normal(0, 1.5 if rng.random() < 0.5 else 3.0, 3)
    if not is3d:
        rap[2] = 0
    v = np.tanh(rap) / np.sqrt(3)
    gam = 1 / np.sqrt(1 - np.sum(v ** 2))
    L = np.eye(4)
    L[0, 0] = gam
    L[0, 1:] = gam * v
    L[1:, 0] = gam * v
    L[1:, 1:] += (gam - 1) * np.outer(v, v) / max(np.sum(v ** 2), 1e-300)
    Tr = np.diag([e, P[0], P[1], P[2] if is3d else 0.0])
    if not is3d:
        L[3, :] = 0
        L[:, 3] = 0
        L[3, 3] = 1
    Tm = L @ Tr @ L.T
    S = np.diag([1, 1, 1, 1 / tau])
    Tm = S @ Tm @ S
    if not is3d:
        Tm[3, :] = 0
        Tm[:, 3] = 0
    iu = [(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]
    return np.array([Tm[a, b] for a, b in iu], np.float32)


def test_landau_algorithm_matches_oracle_on_boosted_fluids():
    """The kernel's Rayleigh-quotient iteration (adjugate steps for the 3 x 3
    boost-invariant problem, partial pivoting in 3D) vs the oracle's Francis-QR
    solver with the reference's selection rules."""
    L = _host_landau()
    rng = np.random.default_rng(5)
    tau = 1.3
    worst_e = worst_u = 0.0
    for k in range(6000):
        is3d = k % 2
        T10 = _boosted_fluid(rng, is3d, tau)
        ok1, e1, u1 = O.landau_cell(T10, tau)
        out = np.zeros(24, np.float32)
        J = np.zeros(4, np.float32)
        ok2 = L.fsm_hosttest_landau_cell(T10.ctypes.data, J.ctypes.data, is3d, 0, 1, 1,
                                         ctypes.c_float(tau), out.ctypes.data)
        assert ok1 == ok2, (T10, is3d)
        if ok1:
            worst_e = max(worst_e, abs(out[0] - e1) / e1)
            worst_u = max(worst_u, float(np.max(np.abs(out[3:7] - u1)) / u1[0]))
    assert worst_e < 1e-6 and worst_u < 1e-6


def test_landau_fallback_for_empty_and_null_cells():
    L = _host_landau()
    out = np.zeros(24, np.float32)
    J = np.zeros(4, np.float32)
    for T10 in (np.zeros(10, np.float32),
                # null dust along x: no timelike eigenvector
                np.array([1, 1, 0, 0, 1, 0, 0, 0, 0, 0], np.float32)):
        ok = L.fsm_hosttest_landau_cell(T10.ctypes.data, J.ctypes.data, 0, 0, 1, 1,
                                        ctypes.c_float(1.0), out.ctypes.data)
        ok_o, e_o, u_o = O.landau_cell(T10, 1.0)
        assert ok == ok_o == 0
        assert out[0] == np.float32(1e-3) and tuple(out[3:7]) == (1, 0, 0, 0)


def test_windowed_spline_slopes_match_oracle_spline():
    """The prep kernels' segment-windowed elimination (fsm_spline.cuh) gives the
    natural-spline node slopes of the whole line (oracle, src/FreeStream.cpp:
    121-154) to far below float rounding, on lines of every length class
    (segment starts exactly at the last node, lines shorter than the window)."""
    L = ctypes.CDLL(str(ROOT / "freestream-milne_b200" / "_build" / "libfsm_hosttest.so"))
    L.fsm_hosttest_line_slopes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_void_p]
    L.fsm_hosttest_line_slopes.restype = None
    rng = np.random.default_rng(11)
    for n in (4, 5, 9, 17, 33, 41, 57, 101, 151, 201, 261, 281, 301):
        d = np.float32(rng.uniform(0.05, 0.1))
        lo = np.float32(-((n - 1) / 2.0) * d)
        x = (np.arange(n, dtype=np.float32) * d + lo).astype(np.float64)
        y = (rng.exponential(5.0, 8)[:, None] *
             np.exp(-(x[None, :] - rng.uniform(-5, 5, 8)[:, None]) ** 2 / 0.32)).sum(0)
        y = (y / 0.197326938 + 1e-7).astype(np.float32)
        got = np.zeros(n, dtype=np.float32)
        L.fsm_hosttest_line_slopes(y.ctypes.data, n, d, lo, got.ctypes.data)
        want = O.spline_derivs(x, y.astype(np.float64)) * np.float64(d)
        scale = np.abs(y).max()
        assert np.max(np.abs(got - want)) <= 1e-6 * scale, n


def test_text_writer_matches_reference_format(tmp_path):
    """fsm_write_field reproduces the reference's own output files byte for byte
    (the golden run of FREESTREAMMILNE::run_freestream_milne wrote them through
    src/FileIO.cpp:11-131), using the reference's float fields."""
    d = np.load(ROOT / "tests" / "golden" / "full_entry_31x29.npz", allow_pickle=True)
    (tmp_path / "freestream_input").write_text(str(d["freestream_input"]))
    p = F.read_params_file(str(tmp_path / "freestream_input"))
    F.lib().fsm_params_derive(p)
    for name in ("e_dat", "ux_dat", "pixy_dat", "e_projection_dat"):
        want = str(d["file_" + name]).encode()
        # values back from the reference's own file, so only the formatting is tested
        proj = "projection" in name
        if proj:
            vals = np.array([[float(t) for t in row.split()] for row in want.decode().splitlines()],
                            dtype=np.float32)  # rows = y, columns = x
            grid = np.zeros((p.DIM_X, p.DIM_Y), np.float32)
            grid[:, :] = vals.T
            var = grid.ravel()
        else:
            var = np.array([float(r.split()[3]) for r in want.decode().splitlines()], np.float32)
        out = tmp_path / (name + ".txt")
        F.write_field(out, var, p, projection=proj, nthreads=3)
        assert out.read_bytes() == want, name


@pytest.mark.parametrize("case", ["lumpy2d", "baryon3d"])
def test_all_output_files_match_reference_writers(tmp_path, case):
    """fsm_write_outputs writes the reference's whole post-matching file set
    (src/FreestreamMilne.cpp:561-673) byte for byte like the reference's own
    writers (src/FileIO.cpp:11-131, compiled from the reference sources) on the
    same float fields -- the Landau-matched outputs and diagnostics of an
    oracle run -- with the files formatted concurrently."""
    if not O.ref_available():
        pytest.skip("reference build not present")
    import workloads as W
    if case == "lumpy2d":
        p, e, nB = W.lumpy2d(seed=4, side=31, dx=0.1, nphip=24, dtau=0.6, eos=2, radius=1.2)
        p.DIM_Y = 29
        W.derive(p)
        e = e.reshape(31, 31)[:, :29].ravel().copy()
    else:
        p, e, nB = W.baryon3d(seed=3, side=21, neta=9, nrap=7, nphip=16)
    po = O.Params(**p.as_dict())
    res = O.run(po, e, nB=nB)
    f32 = {k: np.asarray(res[k], np.float32) for k in ("e", "P", "Pi", "u", "pi", "nB", "V") if k in res}
    n = p.DIM_X * p.DIM_Y * p.DIM_ETA
    d17 = np.asarray(O.diagnostics(po, res["tau"], f32["e"], f32["P"], f32["Pi"], f32["u"], f32["pi"]),
                     np.float32).reshape(17, n)
    diag, off = {}, 0
    for k, c in F.DIAG_COMPS.items():
        diag[k] = d17[off:off + c]
        off += c
    p.TAU = res["tau"]
    mine = tmp_path / "mine"
    mine.mkdir()
    F.write_outputs(mine, p, f32, diag, nthreads=4)
    theirs = tmp_path / "ref"
    (theirs / "output").mkdir(parents=True)
    O.ref_write_outputs(theirs, O.Params(**p.as_dict()), f32, d17)
    a = sorted(x.name for x in mine.iterdir())
    b = sorted(x.name for x in (theirs / "output").iterdir())
    assert a == b and len(a) == (52 if p.BARYON else 47), (len(a), set(a) ^ set(b))
    for name in a:
        assert (mine / name).read_bytes() == (theirs / "output" / name).read_bytes(), name


def _ic_files(run, p, rng):
    """Writes the reference's input files for the readers into run/initial_profiles."""
    d = run / "initial_profiles"
    d.mkdir(parents=True)
    NX, NY, NE = p.DIM_X, p.DIM_Y, p.DIM_ETA
    vals = rng.gamma(1.0, 5.0, NX * NY * NE).astype(np.float32)
    xmin = np.float32(-1.0 * (np.float32(NX - 1) / 2.0) * np.float32(p.DX))
    ymin = np.float32(-1.0 * (np.float32(NY - 1) / 2.0) * np.float32(p.DY))
    emin = np.float32(-1.0 * (np.float32(NE - 1) / 2.0) * np.float32(p.DETA))
    lines = []
    for ix in range(NX):
        for iy in range(NY):
            for ie in range(NE):
                v = vals[(ix * NY + iy) * NE + ie]
                lines.append(f"{ix * p.DX + xmin:.6g} {iy * p.DY + ymin:.6g} {ie * p.DETA + emin:.6g} {v:.7g}")
    (d / "e.dat").write_text("\n".join(lines) + "\n")
    return d, vals


@pytest.mark.parametrize("case", ["2d", "3d"])
def test_initial_conditions_match_reference(tmp_path, case):
    """The reference's initial conditions (analytic, Monte-Carlo with the C
    library's rand(), and every file reader) bit for bit against its own
    functions compiled from its sources, on the same inputs and rand() seed."""
    if not O.ref_available():
        pytest.skip("reference build not present")
    libc = ctypes.CDLL(None)
    ne = 1 if case == "2d" else 9
    p = F.default_params(DIM_X=23, DIM_Y=19, DIM_ETA=ne, DX=0.13, DY=0.11, DETA=0.3,
                         ETA_FLAT=0.6, ETA_WIDTH=0.45)
    po = O.Params(**p.as_dict())
    rng = np.random.default_rng(3)
    d, vals = _ic_files(tmp_path, p, rng)
    n = p.DIM_X * p.DIM_Y * p.DIM_ETA

    def ours(ic, kind="energy"):
        q = F.Params(**p.as_dict())
        if kind == "energy":
            q.IC_ENERGY = ic
        else:
            q.IC_BARYON = ic
        return F.initial_profile(q, kind, d)

    for ic, which in ((1, 1), (3, 3), (2, 2), (6, 6)):
        libc.srand(777)
        a = ours(ic)
        libc.srand(777)
        b = O.ref_initial(tmp_path, po, which)
        assert np.array_equal(a, b), ic
    for ic, which in ((1, 11), (2, 12)):
        libc.srand(99)
        a = ours(ic, "baryon")
        libc.srand(99)
        b = O.ref_initial(tmp_path, po, which)
        assert np.array_equal(a, b), ("baryon", ic)
    # CPU-VH ("d d d value" lines in eta, y, x order)
    lines = [f"0 0 0 {v:.7g}" for v in vals]
    (d / "e.dat").write_text("\n".join(lines) + "\n")
    assert np.array_equal(ours(4), O.ref_initial(tmp_path, po, 4))
    # block formats: superMC (ed.dat, x-major), TRENTO (12 header lines,
    # y-major), TRENTO 3D (one value per cell)
    t = vals[:p.DIM_X * p.DIM_Y]
    (d / "ed.dat").write_text(" ".join(f"{v:.7g}" for v in t) + "\n")
    assert np.array_equal(F.read_profile(d / "ed.dat", p, "supermc_block"), O.ref_initial(tmp_path, po, 21))
    (d / "e.dat").write_text("# header\n" * 12 + " ".join(f"{v:.7g}" for v in t) + "\n")
    assert np.array_equal(F.read_profile(d / "e.dat", p, "trento_block"), O.ref_initial(tmp_path, po, 22))
    (d / "e.dat").write_text(" ".join(f"{v:.7g}" for v in vals) + "\n")
    assert np.array_equal(F.read_profile(d / "e.dat", p, "trento3d_block"), O.ref_initial(tmp_path, po, 23))
    assert n == vals.size
    # missing files and unknown initial conditions are errors, not exits
    q = F.Params(**p.as_dict())
    q.IC_ENERGY = 3
    with pytest.raises(F.FsmError) as ei:
        F.initial_profile(q, "energy", tmp_path / "nowhere")
    assert ei.value.status == 8
    q.IC_ENERGY = 5
    with pytest.raises(F.FsmError) as ei:
        F.initial_profile(q, "energy", d)
    assert ei.value.status == 3


def test_combined_planes_cover_sampled_pairs_with_reference_weights():
    """Every sampled (eta slice, rapidity) pair of a 3D plan has its own
    combined plane, listed under the source eta pair it reads, with the
    weights (1 - eta_frac) rf(efl) and eta_frac rf(efl + 1) of the reference's
    eta interpolation and rapidity factors (src/FreeStream.cpp:264-266, 345,
    381-382); pairs that cannot sample the grid have none."""
    import workloads as W
    L = ctypes.CDLL(str(ROOT / "freestream-milne_b200" / "_build" / "libfsm_hosttest.so"))
    ip, fp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)
    L.fsm_hosttest_comb_planes.argtypes = [ctypes.POINTER(F.Params), ip, ip, fp, ctypes.c_int,
                                           fp, fp, fp, ip]
    for p in (W.baryon3d(seed=1, side=41, neta=51, nrap=41)[0],
              W.baryon3d(seed=2, side=31, neta=25, nrap=21, nphip=40)[0]):
        NE, NR = p.DIM_ETA, p.DIM_RAP
        plane_of = np.zeros(NE * NR, np.int32)
        cw_start = np.zeros(NE, np.int32)
        cap = NE * NR
        cw = np.zeros((cap, 5), np.float32)
        pair3 = np.zeros((NE * NR, 3), np.float32)
        rapf = np.zeros(NE * NR, np.float32)
        rapfB = np.zeros(NE * NR, np.float32)
        lohi = np.zeros(2, np.int32)
        c = lambda a, t: a.ctypes.data_as(t)
        n = L.fsm_hosttest_comb_planes(ctypes.byref(p), c(plane_of, ip), c(cw_start, ip), c(cw, fp), cap,
                                       c(pair3, fp), c(rapf, fp), c(rapfB, fp), c(lohi, ip))
        assert 0 < n <= cap
        efl, efrac, D = pair3[:, 0].astype(int), pair3[:, 1], pair3[:, 2]
        irap = np.tile(np.arange(NR), NE)
        bound = np.float32((p.DIM_X + p.DIM_Y) * max(p.DX, p.DY))
        sampled = ((irap >= lohi[0]) & (irap < lohi[1]) & (efl >= 1) & (efl < NE - 1) &
                   np.isfinite(D) & (np.abs(D) <= bound))
        assert np.array_equal(plane_of >= 0, sampled)
        assert sorted(plane_of[sampled].tolist()) == list(range(n))
        assert cw_start[-1] == n and np.all(np.diff(cw_start) >= 0)
        pair_of_plane = np.full(n, -1)
        pair_of_plane[plane_of[sampled]] = np.nonzero(sampled)[0]
        for e in range(NE - 1):
            for k in range(cw_start[e], cw_start[e + 1]):
                pr = pair_of_plane[int(cw[k, 0])]
                assert efl[pr] == e
                r = irap[pr]
                om = np.float32(1.0) - efrac[pr]
                assert cw[k, 1] == np.float32(om * rapf[e * NR + r])
                assert cw[k, 2] == np.float32(efrac[pr] * rapf[(e + 1) * NR + r])
                assert cw[k, 3] == np.float32(om * rapfB[e * NR + r])
                assert cw[k, 4] == np.float32(efrac[pr] * rapfB[(e + 1) * NR + r])
        # the combined value is the reference's eta interpolation of the
        # rapidity-weighted slices to float rounding
        rng = np.random.default_rng(0)
        e0, e1 = rng.uniform(0, 50, n).astype(np.float32), rng.uniform(0, 50, n).astype(np.float32)
        k = np.argsort(cw[:n, 0])
        pr = pair_of_plane[np.arange(n)]
        got = cw[k, 1] * e0 + cw[k, 2] * e1
        f, r0 = efrac[pr].astype(np.float64), efl[pr]
        ref = ((1 - f) * e0 * rapf[r0 * NR + irap[pr]] + f * e1 * rapf[(r0 + 1) * NR + irap[pr]])
        assert np.allclose(got, ref, rtol=1e-6, atol=1e-30 + 1e-6 * np.abs(ref).max())
