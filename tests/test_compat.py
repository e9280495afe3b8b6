"""The drop-in FREESTREAMMILNE class (freestream-milne_b200/compat/FreestreamMilne.cpp):
it compiles as the single translation unit callers include, behaves like the
reference's class around the compute (freestream_input, output/*.dat, the 17
vectors), and its numbers are the library's GPU path."""
import os
import pathlib
import subprocess

import numpy as np
import pytest

import fsm_b200 as F
from fsm_testutil import fsm_params

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden" / "full_entry_31x29.npz"


def _build(tmp_path):
    exe = tmp_path / "compat_driver"
    lib = ROOT / "freestream-milne_b200" / "lib"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror",
                    f"-I{ROOT / 'freestream-milne_b200' / 'compat'}", f"-I{ROOT / 'include'}",
                    "-o", str(exe), str(ROOT / "tests" / "compat_driver.cpp"), f"-L{lib}", "-lfsm",
                    f"-Wl,-rpath,{lib}"], check=True)
    return exe


def _setup_run_dir(tmp_path):
    d = np.load(GOLD, allow_pickle=True)
    run = tmp_path / "run"
    (run / "output").mkdir(parents=True)
    (run / "freestream_input").write_text(str(d["freestream_input"]))
    e = np.asarray(d["e_gev"], dtype=np.float32)
    e.tofile(run / "e.bin")
    return d, run, e


def test_compat_class_compiles_and_has_no_cpu_fallback(tmp_path):
    exe = _build(tmp_path)
    _, run, _ = _setup_run_dir(tmp_path)
    if F.device_count() > 0:
        pytest.skip("a GPU is present; the GPU test covers the run")
    r = subprocess.run([str(exe), "e.bin", "out.bin"], cwd=run, capture_output=True, text=True)
    assert r.returncode != 0                      # no device: an error, not a CPU result
    assert "freestream-milne:" in r.stdout
    assert (run / "output" / "initial_e.dat").exists()  # written before the compute, as the reference


@pytest.mark.gpu
def test_compat_class_matches_library_and_reference_files(tmp_path, ctx):
    exe = _build(tmp_path)
    d, run, e = _setup_run_dir(tmp_path)
    r = subprocess.run([str(exe), "e.bin", "out.bin"], cwd=run, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = np.fromfile(run / "out.bin", dtype=np.float64)
    tau, vec = raw[0], raw[1:].reshape(17, -1)
    p = F.read_params_file(str(run / "freestream_input"))
    F.lib().fsm_params_derive(p)
    got = ctx.run_event(p, e)
    assert tau == pytest.approx(got["info"]["tau"])
    hbarc = np.float32(0.197326938)
    n = p.DIM
    # the class's vectors are exactly the library's float outputs in GeV/fm^3
    np.testing.assert_array_equal(vec[0], got["e"].astype(np.float64) * hbarc)
    np.testing.assert_array_equal(vec[1], got["P"].astype(np.float64) * hbarc)
    for m in range(4):
        np.testing.assert_array_equal(vec[2 + m], got["u"].reshape(4, n)[m].astype(np.float64))
    for m in range(10):
        np.testing.assert_array_equal(vec[6 + m], got["pi"].reshape(10, n)[m].astype(np.float64) * hbarc)
    np.testing.assert_array_equal(vec[16], got["Pi"].astype(np.float64) * hbarc)
    # the reference's vectors: same cells within the parity tolerance on e
    ref = np.asarray(d["vectors"], dtype=np.float64).reshape(17, -1)
    mask = ref[0] > 1e-6 * ref[0].max()
    assert np.max(np.abs(vec[0] - ref[0])[mask] / ref[0][mask]) < 1e-4
    # output files: same layout as the reference's, values within tolerance
    for name, comp in (("e_dat", 0), ("ux_dat", 3), ("pixy_dat", 11)):
        mine = (run / "output" / (name[:-4] + ".dat")).read_text().splitlines()
        theirs = str(d["file_" + name]).splitlines()
        assert len(mine) == len(theirs)
        a = np.array([[float(t) for t in l.split()] for l in mine])
        b = np.array([[float(t) for t in l.split()] for l in theirs])
        np.testing.assert_array_equal(a[:, :3], b[:, :3])
        scale = np.abs(b[:, 3]).max()
        assert np.max(np.abs(a[:, 3] - b[:, 3])) <= 1e-3 * scale, name
