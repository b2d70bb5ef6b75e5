"""The allocation-free spectrum entry point against the regular one.

``sp_spectrum_noalloc`` serves callers that may not allocate device memory (their own pool
allocator owns the GPU, or they cannot afford cudaMalloc's implicit synchronisation): it needs
no engine handle and keeps its shell accumulators in a fixed file-scope device array.  These
tests call it through the C ABI on a state the engine holds and compare with ``sp_spectrum``
(the engine's regular entry point), twice in a row, because the shared array keeps the previous
call's sums and each call must clear them.  The file name sorts last so a failure here never
hides the other tests' results; it also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, state, n, dim, fp64, nshell, stream):
    out = np.full(nshell, np.nan)
    st = lib.sp_spectrum_noalloc(ctypes.c_void_p(state.data_ptr()), n, dim, int(fp64),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nshell,
                                 stream)
    return st, out


@pytest.mark.parametrize("dim,n,dtype", [(2, 96, "float64"), (2, 256, "float32"),
                                         (3, 24, "float64"), (3, 32, "float32")])
def test_noalloc_spectrum_matches_regular_twice(dim, n, dtype):
    from pyspectral_b200 import Config, initial
    from pyspectral_b200.registry import get

    s = get("b200").make(Config(n=n, dim=dim, dtype=dtype, nu=1e-3))
    ic = (initial.random_phase_2d(n, k0=6, seed=11) if dim == 2
          else initial.to_spectral(initial.random_3d(n, k0=3, seed=11), 3))
    s.set_state(ic)
    s.advance(2, 1e-3)
    lib = s.lib
    k, regular = s.diag.spectrum(s.state_native())
    nshell = len(regular)
    for _ in range(2):  # the second call must not see the first call's sums
        st, got = _noalloc(lib, s.state_native(), n, dim, dtype == "float64", nshell,
                           s._stream())
        assert st == 0, lib.sp_create_error()
        np.testing.assert_allclose(got, regular, rtol=1e-12, atol=1e-300)
    assert got.sum() == pytest.approx(s.diag.energy(s.state_native()), rel=1e-12)


def test_noalloc_spectrum_large_grid_accumulates_in_the_array_itself():
    """Above 6144 shells the histogram no longer fits the kernel's shared memory and every
    block adds straight into the file-scope array: 8704^2 fp32 (6156 shells), twice in a row,
    so the clearing of that path is checked too."""
    from pyspectral_b200 import Config, initial
    from pyspectral_b200.registry import get

    n = 8704
    s = get("b200").make(Config(n=n, dim=2, dtype="float32", nu=1e-5))
    s.set_state(initial.random_phase_2d(n, k0=40, seed=5))
    k, regular = s.diag.spectrum(s.state_native())
    nshell = len(regular)
    assert nshell > 6144
    for _ in range(2):
        st, got = _noalloc(s.lib, s.state_native(), n, 2, False, nshell, s._stream())
        assert st == 0, s.lib.sp_create_error()
        np.testing.assert_allclose(got, regular, rtol=1e-12, atol=1e-300)


def test_noalloc_spectrum_rejects_sizes_beyond_its_array():
    import torch

    from pyspectral_b200 import _lib

    lib = _lib.load()
    dummy = torch.zeros(16, dtype=torch.complex128, device="cuda")
    n = 32768  # 2D: 23171 shells > SP_NOALLOC_MAX_SHELLS; rejected before any device work
    nshell = int(np.floor(np.sqrt(2) * (n // 2) + 0.5)) + 1
    st, out = _noalloc(lib, dummy, n, 2, True, nshell, None)
    assert st == -1
    assert b"SP_NOALLOC_MAX_SHELLS" in lib.sp_create_error()
    assert np.isnan(out).all()
    st, _ = _noalloc(lib, dummy, 64, 2, True, 7, None)  # wrong shell count for n = 64
    assert st == -1 and b"nshell" in lib.sp_create_error()
