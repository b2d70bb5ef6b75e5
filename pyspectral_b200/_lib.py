"""ctypes binding of libspectral_b200.so (declarations in include/spectral_b200.h).

The library is loaded from this package directory only.  A missing library or a missing CUDA
device raises :class:`BackendUnavailable` — there is no other implementation to fall back to.
"""

from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Any

from pyspectral_b200.base import BackendUnavailable

LIB_PATH = Path(__file__).resolve().parent / "libspectral_b200.so"

# status codes (enum sp_status)
SP_OK = 0
STATUS_NAMES = {0: "SP_OK", -1: "SP_ERR_ARG", -2: "SP_ERR_CUDA", -3: "SP_ERR_CUFFT",
                -4: "SP_ERR_STATE", -5: "SP_ERR_UNSUPPORTED"}
# enum sp_form / sp_fft_mode
FORM_CODES = {"basdevant": 0, "rotational": 1}
FFT_CUFFT, FFT_CUFFT_LEAN, FFT_FUSED = 0, 1, 2
# enum sp_size_index
SZ_MODES, SZ_NCOMP, SZ_NWORK, SZ_NINV, SZ_NFWD = 0, 1, 2, 3, 4
SZ_STATE_BYTES, SZ_WORK_BYTES, SZ_AUX_BYTES, SZ_FFTWS_BYTES, SZ_NSHELL, SZ_COUNT = 5, 6, 7, 8, 9, 10

_vp, _i, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
_i64, _u64, _f = ctypes.c_int64, ctypes.c_uint64, ctypes.c_float
_dp = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); the exported C ABI
SIGNATURES: dict[str, tuple[Any, list[Any]]] = {
    "sp_abi_version": (_i, []),
    "sp_create": (_vp, [_i, _i, _i, _i, _i, ctypes.POINTER(_i)]),
    "sp_destroy": (None, [_vp]),
    "sp_query_sizes": (_i, [_vp, ctypes.POINTER(ctypes.c_int64), _i]),
    "sp_bind": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "sp_set_physics": (_i, [_vp, _d, _d, _d, _d, _d]),
    "sp_set_forcing_amplitude": (_i, [_vp, _d]),
    "sp_prepare": (_i, [_vp, _vp]),
    "sp_step": (_i, [_vp, _d, _vp]),
    "sp_sync_state": (_i, [_vp, _vp]),
    "sp_set_graph": (_i, [_vp, _i]),
    "sp_set_column_streaming": (_i, [_i]),
    "sp_column_streaming": (_i, []),
    "sp_take_device_error": (_i, [ctypes.POINTER(ctypes.c_uint)]),
    "sp_wait_probe": (_i, [ctypes.c_uint, _vp]),
    "sp_diagnostics": (_i, [_vp, _vp, _d, _d, _dp, _vp]),
    "sp_max_velocity": (_i, [_vp, _vp, _dp, _dp, _vp]),
    "sp_spectrum": (_i, [_vp, _vp, _dp, _i, _vp]),
    "sp_run_phase": (_i, [_vp, _i, _i, _vp]),
    "sp_kernel_launches": (ctypes.c_int64, [_vp]),
    "sp_last_error": (ctypes.c_char_p, [_vp]),
    "sp_create_error": (ctypes.c_char_p, []),
    "sp_spectrum_noalloc": (_i, [_vp, _i, _i, _i, _dp, _i, _vp]),
    "sp_batch_create": (_vp, [_i, _i, _i, ctypes.POINTER(_i)]),
    "sp_batch_destroy": (None, [_vp]),
    "sp_batch_query_sizes": (_i, [_vp, ctypes.POINTER(ctypes.c_int64), _i]),
    "sp_batch_bind": (_i, [_vp, _vp, _vp, _vp]),
    "sp_batch_set_physics": (_i, [_vp, _dp, _d, _d, _d, _d]),
    "sp_batch_set_step": (_i, [_vp, _dp, _dp, _vp]),
    "sp_batch_prepare": (_i, [_vp, _vp]),
    "sp_batch_step": (_i, [_vp, _vp]),
    "sp_batch_sync_state": (_i, [_vp, _vp]),
    "sp_batch_diagnostics": (_i, [_vp, _d, _d, _dp, _vp]),
    "sp_batch_max_velocity": (_i, [_vp, _dp, _vp]),
    "sp_batch_kernel_launches": (ctypes.c_int64, [_vp]),
    "sp_batch_last_error": (ctypes.c_char_p, [_vp]),
    "sp_batch_tile_supported": (_i, [_i, _i]),
    "sp_batch_set_tile": (_i, [_vp, _i]),
    "sp_batch_tile": (_i, [_vp]),
    "sp_group_create": (_vp, [ctypes.POINTER(_vp), _i, ctypes.POINTER(_i)]),
    "sp_group_destroy": (None, [_vp]),
    "sp_group_step": (_i, [_vp, _vp]),
    "sp_group_last_error": (ctypes.c_char_p, [_vp]),
    "sp_group_worklist_bytes": (_i, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "sp_group_bind": (_i, [_vp, _vp]),
    "sp_group_set_worklist": (_i, [_vp, _i]),
    "sp_group_worklist": (_i, [_vp]),
    "sp_group_kernel_launches": (ctypes.c_int64, [_vp]),
    "sp_mma_tile_check": (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _vp]),
    "sp_nonlinear": (_i, [_vp, _vp, _vp, _vp]),
    "sp_filter_spectrum": (_i, [_vp, _i, _vp, _i, _i, _i, _i, _vp]),
    "sp_closure_param_count": (_i, []),
    "sp_closure_create": (_vp, [_i, _i, ctypes.POINTER(_i)]),
    "sp_closure_destroy": (None, [_vp]),
    "sp_closure_last_error": (ctypes.c_char_p, [_vp]),
    "sp_closure_kernel_launches": (_i64, [_vp]),
    "sp_closure_set_params": (_i, [_vp, _vp]),
    "sp_closure_get_params": (_i, [_vp, _vp]),
    "sp_closure_get_grad": (_i, [_vp, _vp]),
    "sp_closure_set_scales": (_i, [_vp, _vp, _f, _i]),
    "sp_closure_get_scales": (_i, [_vp, _vp]),
    "sp_closure_set_adam": (_i, [_vp, _d, _d, _d, _d, _d, _i, _i]),
    "sp_closure_set_shell_gain": (_i, [_vp, _vp, _i]),
    "sp_closure_shell_count": (_i, [_vp]),
    "sp_closure_set_update": (_i, [_vp, _i]),
    "sp_closure_bank_load": (_i, [_vp, _vp, _i]),
    "sp_closure_add_snapshot": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "sp_closure_bank_read": (_i, [_vp, _i, _vp]),
    "sp_closure_bank_count": (_i, [_vp]),
    "sp_closure_bank_reset": (_i, [_vp]),
    "sp_closure_grad": (_i, [_vp, _i64, _i, _u64, _vp]),
    "sp_closure_train": (_i, [_vp, _i, _i, _u64, _vp]),
    "sp_closure_step_count": (_i64, [_vp]),
    "sp_closure_train_begin": (_i, [_vp, _i, _u64, _vp]),
    "sp_closure_train_finish": (_i, [_vp, _vp]),
    "sp_closure_grad_buffer": (_vp, [_vp]),
    "sp_closure_losses": (_i, [_vp, _i64, _i, _vp]),
    "sp_closure_infer": (_i, [_vp, _vp, _i64, _i, _vp, _i, _vp]),
    "sp_closure_infer_async": (_i, [_vp, _vp, _i64, _i, _vp, _i, _vp]),
    "sp_attach_closure": (_i, [_vp, _vp]),
    "sp_run_to": (_i, [_vp, _d, _d, _d, _i, _d, _d, _i64, _dp, ctypes.POINTER(_i64), _dp, _vp]),
    "sp_slab_create": (_vp, [_i, _i, _i, _i, _i, ctypes.POINTER(_i)]),
    "sp_slab_destroy": (None, [_vp]),
    "sp_slab_last_error": (ctypes.c_char_p, [_vp]),
    "sp_slab_kernel_launches": (_i64, [_vp]),
    "sp_slab_query_sizes": (_i, [_vp, ctypes.POINTER(ctypes.c_int64), _i]),
    "sp_slab_exchange_block_bytes": (_i64, [_vp, _i]),
    "sp_slab_bind": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "sp_slab_set_physics": (_i, [_vp, _d, _d, _d, _d, _d]),
    "sp_slab_set_forcing_amplitude": (_i, [_vp, _d]),
    "sp_slab_set_dt": (_i, [_vp, _d, _vp]),
    "sp_slab_prepare": (_i, [_vp, _vp]),
    "sp_slab_stage_part": (_i, [_vp, _i, _i, _vp]),
    "sp_slab_max_velocity": (_i, [_vp, _vp, _vp]),
    "sp_slab_energy": (_i, [_vp, _vp, _vp, _vp]),
    "sp_closure_check": (_i, [_vp, _vp]),
}

_LIB: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Load (once) and declare the library; BackendUnavailable if it is not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise BackendUnavailable(
            f"{LIB_PATH.name} is not built (run `python -m pyspectral_b200.build`)")
    try:
        lib = ctypes.CDLL(str(LIB_PATH))
    except OSError as e:
        raise BackendUnavailable(f"cannot load {LIB_PATH.name}: {e}") from e
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class EngineError(RuntimeError):
    """A call into the engine returned a non-zero status."""


def check(lib: ctypes.CDLL, handle: int | None, status: int, what: str) -> None:
    """Raise EngineError with the engine's message when ``status`` is not SP_OK."""
    if status == SP_OK:
        return
    msg = lib.sp_last_error(handle) if handle else lib.sp_create_error()
    text = msg.decode() if msg else ""
    raise EngineError(f"{what} failed: {STATUS_NAMES.get(status, status)}: {text}")


def dptr(arr: Any) -> ctypes.c_void_p:
    """Device pointer of a torch tensor (or None)."""
    return ctypes.c_void_p(arr.data_ptr()) if arr is not None else ctypes.c_void_p(0)


def check_device_errors(lib: ctypes.CDLL) -> None:
    """Raise EngineError when a kernel of this library flagged a device-side error (bounded
    wait that gave up) since the last check; clears the flags.  Synchronous."""
    bits = ctypes.c_uint(0)
    st = lib.sp_take_device_error(ctypes.byref(bits))
    if st != 0:
        raise EngineError(f"sp_take_device_error failed: {STATUS_NAMES.get(st, st)}")
    if bits.value:
        raise EngineError(f"device error bits {bits.value:#x}: a streamed column pass timed out "
                          "waiting for its TMA data; the state is invalid, and bulk copies into "
                          "the timed-out block's shared memory may still have been in flight "
                          "when it exited: recreate the solver (a new process is the safe "
                          "choice)")
