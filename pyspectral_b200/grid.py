"""Spectral-grid conventions shared with the reference (src/pyspectral/grid.py:1-67).

Physical arrays are ``(n,)*dim`` with axes (x, y[, z]); spectral arrays are the real-to-complex
transform over the last axis, shape ``(n,)*(dim-1) + (n//2+1,)``, unnormalised like
``numpy.fft.rfftn``.  Box side 2 pi, so wavenumbers are integers.  These helpers build host-side
arrays (set-up, checks, initial conditions); the device kernels recompute k from the index.
"""

from __future__ import annotations

import numpy as np


def spectral_shape(n: int, dim: int) -> tuple[int, ...]:
    """Shape of one scalar field in r2c spectral space."""
    return (n,) * (dim - 1) + (n // 2 + 1,)


def wavenumbers(n: int, dim: int) -> tuple[np.ndarray, ...]:
    """Broadcastable float64 wavenumber vectors: full axes 0..n/2-1,-n/2..-1; last axis 0..n/2."""
    full = np.concatenate([np.arange(0, n // 2), np.arange(-(n // 2), 0)]).astype(np.float64)
    half = np.arange(n // 2 + 1, dtype=np.float64)
    axes = [full] * (dim - 1) + [half]
    out = []
    for a, v in enumerate(axes):
        shape = [1] * dim
        shape[a] = v.size
        out.append(v.reshape(shape))
    return tuple(out)


def k_squared(n: int, dim: int) -> np.ndarray:
    """|k|^2 on the spectral grid."""
    k2 = np.zeros(spectral_shape(n, dim))
    for k in wavenumbers(n, dim):
        k2 = k2 + k * k
    return k2


def dealias_mask(n: int, dim: int, kind: str = "2/3") -> np.ndarray:
    """Retained modes: ``"2/3"`` keeps 3|k_i| < n on every axis; ``"phase-shift"`` keeps the
    sphere |k|^2 < 2 (n/3)^2."""
    if kind == "2/3":
        keep = np.ones(spectral_shape(n, dim), dtype=bool)
        for k in wavenumbers(n, dim):
            keep = keep & (3.0 * np.abs(k) < n)
        return keep
    if kind == "phase-shift":
        return k_squared(n, dim) < 2.0 * (n / 3.0) ** 2
    raise ValueError(kind)


def hermitian_weights(n: int, dim: int) -> np.ndarray:
    """1 on the first and last (Nyquist) planes of the half axis, 2 elsewhere."""
    w = np.full(n // 2 + 1, 2.0)
    w[0] = w[-1] = 1.0
    return np.broadcast_to(w.reshape((1,) * (dim - 1) + (-1,)), spectral_shape(n, dim))


def physical_grid(n: int, dim: int) -> tuple[np.ndarray, ...]:
    """Coordinates x_j = 2 pi j / n as broadcastable vectors."""
    x = 2.0 * np.pi * np.arange(n) / n
    out = []
    for a in range(dim):
        shape = [1] * dim
        shape[a] = n
        out.append(x.reshape(shape))
    return tuple(out)


def n_shells(n: int, dim: int) -> int:
    """Number of spectrum shells, floor(sqrt(dim) n/2 + 0.5) + 1 (diagnostics.py:39)."""
    return int(np.floor(np.sqrt(dim) * (n // 2) + 0.5)) + 1
