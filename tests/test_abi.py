"""The C-ABI library loads and exports every symbol declared in include/*.h
(no compute calls: this runs without a GPU)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
LIB = REPO / "diff-fvr_b200" / "fvr" / "libfvr_b200.so"


def _declared():
    names = set()
    for h in (REPO / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(fvr_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        subprocess.run(["make", "-C", str(REPO / "diff-fvr_b200" / "csrc"), "-j8"], check=True)
    return ctypes.CDLL(str(LIB))


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_the_header():
    import fvr._lib as L

    assert sorted(L.SIGNATURES) == _declared()


def test_integration_guide_maps_every_entry_point():
    """INTEGRATION.md's entry-point table names every declared symbol, so a
    maintainer binding the library finds each one next to the reference
    interface it replaces."""
    text = (REPO / "INTEGRATION.md").read_text()
    missing = [n for n in _declared() if f"`{n}`" not in text]
    assert not missing, f"not mapped in INTEGRATION.md: {missing}"


def test_status_strings_and_queries(lib):
    import fvr._lib as L

    L.load()
    assert L.load().fvr_status_string(0).decode() == "ok"
    assert "workspace" in L.load().fvr_status_string(4).decode()
    assert L.load().fvr_fft_supported(192) == 1
    assert L.load().fvr_fft_supported(17) == 1
    assert L.load().fvr_fft_supported(131) == 0
    assert L.query("fvr_stencil_bytes", 3, 3, 3, 0) == 4 * 4 * 4 * 64
    assert L.query("fvr_stencil_bytes", 3, 3, 3, 1) == 4 * 4 * 4 * 32


def test_product_path_fails_loudly_without_a_gpu():
    """CPU inputs are moved to the CUDA device; with none present the call
    raises FvrError instead of computing on the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")

    import fvr._lib as L
    from fvr.slice_ops import fourier_slice_3d

    vol = torch.zeros(1, 2, 4, 4, 4)
    u = torch.zeros(1, 3)
    f = torch.zeros(4)
    with pytest.raises(L.FvrError):
        fourier_slice_3d(vol, u, u, f, f, (1.5, 1.5, 1.5))


def test_native_autograd_binding_loads():
    """The native autograd binding (csrc/fvr_autograd.cpp) builds against the
    installed PyTorch, imports, and refuses a prepared launch with null
    pointers before anything runs (no GPU needed)."""
    import sys

    import torch

    sys.path.insert(0, str(REPO / "diff-fvr_b200" / "csrc"))
    import build_autograd

    build_autograd.build()
    from fvr import _fvr_autograd as A
    from fvr import torch_engine

    assert torch_engine._NATIVE is A
    with pytest.raises(RuntimeError, match="null pointer"):
        A.SnccCall(fn=0, status=0, dtype=0, stencil=0, scales=0, D=1, H=1, W=1, C=1, views=[0], ftargs=[0], hp=0,
                   lin=0, R=1, kappa=0.0, variant=0, ws=0, ws_bytes=0, device=0, keep=[torch.zeros(1)])
