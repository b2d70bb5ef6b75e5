"""The C ABI library loads and exports every function include/*.h declares (CPU only: no
compute call is made; creating an engine without a GPU must fail cleanly with a message)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_functions() -> list[str]:
    names: list[str] = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w\s\*]*?\b(sp_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from pyspectral_b200 import _lib, build

    build.build()
    return _lib.load()


def test_header_declares_entry_points():
    names = _declared_functions()
    assert {"sp_create", "sp_step", "sp_bind", "sp_diagnostics", "sp_destroy"} <= set(names)


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from pyspectral_b200 import _lib

    assert set(_declared_functions()) <= set(_lib.SIGNATURES)


def test_abi_version(lib):
    assert lib.sp_abi_version() == 1


def test_library_targets_sm100a_only():
    from pyspectral_b200 import build

    cmd = " ".join(build.command())
    assert "arch=compute_100a,code=sm_100a" in cmd
    assert "sm_90" not in cmd and "sm_80" not in cmd


def test_create_without_gpu_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    st = ctypes.c_int(0)
    h = lib.sp_create(16, 2, 0, 1, 0, ctypes.byref(st))
    assert not h
    assert st.value == -2
    assert lib.sp_create_error()


def test_create_rejects_bad_arguments(lib):
    st = ctypes.c_int(0)
    assert not lib.sp_create(7, 2, 0, 1, 0, ctypes.byref(st)) and st.value == -1
    assert not lib.sp_create(16, 4, 0, 1, 0, ctypes.byref(st)) and st.value == -1
    assert not lib.sp_create(16, 2, 1, 1, 0, ctypes.byref(st)) and st.value == -5
    assert b"basdevant" in lib.sp_create_error()
    assert not lib.sp_create(16, 2, 0, 1, 9, ctypes.byref(st)) and st.value == -1
    # null handles are rejected, not dereferenced
    assert lib.sp_step(None, 0.1, None) == -1
    assert lib.sp_set_graph(None, 1) == -1
    assert lib.sp_last_error(None) == b"null handle"


def test_streaming_switch_and_probe_arguments(lib):
    """Host-side behaviour of the fused engine's pass switch and of the failure-path probe:
    the switch round-trips without a device; the probe rejects its poll counts before any
    CUDA call."""
    prev = lib.sp_column_streaming()
    assert prev == 1  # the streamed column pass is the default
    try:
        assert lib.sp_set_column_streaming(0) == 0 and lib.sp_column_streaming() == 0
        assert lib.sp_set_column_streaming(1) == 0 and lib.sp_column_streaming() == 1
    finally:
        lib.sp_set_column_streaming(prev)
    assert lib.sp_wait_probe(0, None) == -1
    assert lib.sp_wait_probe((1 << 20) + 1, None) == -1
    assert b"polls" in lib.sp_create_error()
    assert lib.sp_take_device_error(None) == -1
