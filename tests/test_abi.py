"""The C-ABI library loads on a CPU-only host and exports every symbol include/*.h declares."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(liar_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("liar_gpu_create", "liar_gpu_destroy", "liar_gpu_last_error", "liar_gpu_mesh_build",
                     "liar_gpu_trace", "liar_gpu_trace_device"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from liar_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_python_binding_covers_header():
    from liar_b200 import _native
    missing = sorted(declared_functions() - set(_native.SIGNATURES))
    assert not missing, f"no ctypes signature for {missing}"


def test_abi_version_without_gpu():
    from liar_b200 import _native
    lib = _native.load()
    assert lib.liar_gpu_abi_version() == 1


def test_create_fails_cleanly_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    from liar_b200 import _native
    lib = _native.load()
    h = ctypes.c_void_p()
    rc = lib.liar_gpu_create(ctypes.byref(h), 0)
    assert rc == -3  # LIAR_ERR_NO_DEVICE, no exception, no crash
    assert not h.value
