import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG = ROOT / "freestream-milne_b200"
for p in (ROOT / "tests", ROOT / "oracle", PKG):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def _make(dirpath, *targets):
    r = subprocess.run(["make", "-s", "-C", str(dirpath), *targets], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"make in {dirpath} failed:\n{r.stdout}\n{r.stderr}")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")
    # incremental builds of the oracle (test infrastructure) and the library
    sys.path.insert(0, str(ROOT))
    from __graft_entry__ import oracle_make_args
    _make(ROOT / "oracle", *oracle_make_args())
    _make(PKG, "all", "hosttest")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    if not _has_gpu():
        pytest.skip("no CUDA device")
    import fsm_b200 as F
    c = F.Context(0)
    yield c
    c.close()
