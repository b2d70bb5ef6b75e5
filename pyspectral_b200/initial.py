"""Initial conditions (host NumPy, float64), generated once before a run.

The physical-space generators reproduce the reference's fields (src/pyspectral/initial.py:10-87)
for the same arguments and seeds; :func:`random_phase_2d` is the fixed-amplitude, uniform-phase
vorticity field of the decaying-turbulence workload (E(k) ~ k^4 exp(-2 (k/k0)^2)), built
directly in spectral space so an 8192^2 state needs no host FFT.
"""

from __future__ import annotations

import numpy as np

from pyspectral_b200.grid import (dealias_mask, hermitian_weights, physical_grid,
                                  spectral_shape, wavenumbers)


def taylor_green_2d(n: int) -> np.ndarray:
    """omega = 2 sin x sin y; decays exactly as exp(-2 nu t) under Navier-Stokes."""
    x, y = physical_grid(n, 2)
    return 2.0 * np.sin(x) * np.sin(y)


def smooth_2d(n: int) -> np.ndarray:
    """Smooth, zero-mean, non-band-limited 2D vorticity."""
    x, y = physical_grid(n, 2)
    w = np.exp(0.8 * np.cos(x) + 0.6 * np.sin(2.0 * y + 0.4 * np.cos(x)))
    w = w + 0.5 * np.sin(x + y) * np.cos(y)
    return w - w.mean()


def _noise_spectrum(n: int, dim: int, k0: float, seed: int, ncomp: int) -> np.ndarray:
    """Gaussian white noise shaped to a shell spectrum ~ k^4 exp(-2 (k/k0)^2), dealiased."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((ncomp,) + (n,) * dim)
    spec = np.fft.rfftn(white, axes=tuple(range(-dim, 0)))
    kk = np.sqrt(sum(k * k for k in wavenumbers(n, dim)))
    area = kk ** (dim - 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        shape = np.sqrt(kk**4 * np.exp(-2.0 * (kk / k0) ** 2) / np.where(kk > 0, area, 1.0))
    shape[kk == 0] = 0.0
    return spec * shape * dealias_mask(n, dim)


def random_2d(n: int, k0: float = 8.0, seed: int = 0, energy: float = 0.5) -> np.ndarray:
    """Random vorticity (Gaussian amplitudes) with kinetic energy ``energy``."""
    spec = _noise_spectrum(n, 2, k0, seed, 1)[0]
    k2 = sum(k * k for k in wavenumbers(n, 2))
    w = hermitian_weights(n, 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        e = 0.5 * np.sum(np.where(k2 > 0, w * np.abs(spec) ** 2 / k2, 0.0)) / float(n) ** 4
    return np.fft.irfftn(spec, s=(n, n), axes=(0, 1)) * np.sqrt(energy / e)


def taylor_green_3d(n: int) -> np.ndarray:
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0; shape (3, n, n, n)."""
    x, y, z = physical_grid(n, 3)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    return np.stack(np.broadcast_arrays(u, v, np.zeros_like(u * v)))


def random_3d(n: int, k0: float = 4.0, seed: int = 0, energy: float = 0.5) -> np.ndarray:
    """Random solenoidal velocity with kinetic energy ``energy``."""
    spec = _noise_spectrum(n, 3, k0, seed, 3)
    ks = wavenumbers(n, 3)
    k2 = sum(k * k for k in ks)
    inv = np.where(k2 > 0, 1.0 / np.where(k2 > 0, k2, 1.0), 0.0)
    div = sum(k * c for k, c in zip(ks, spec, strict=True))
    spec = np.stack([c - k * div * inv for k, c in zip(ks, spec, strict=True)])
    u = np.fft.irfftn(spec, s=(n, n, n), axes=(1, 2, 3))
    e = 0.5 * np.mean(np.sum(u * u, axis=0))
    return u * np.sqrt(energy / e)


def to_spectral(field: np.ndarray, dim: int, dealias: str = "2/3") -> np.ndarray:
    """Physical field -> dealiased r2c spectral state (complex128)."""
    n = field.shape[-1]
    return np.fft.rfftn(field, axes=tuple(range(-dim, 0))) * dealias_mask(n, dim, dealias)


def random_phase_2d(n: int, k0: float = 12.0, seed: int = 0, energy: float = 0.5) -> np.ndarray:
    """Spectral vorticity with fixed amplitudes and uniform random phases (complex128).

    Mode amplitudes |omega_k| ~ k^(5/2) exp(-(k/k0)^2), so the shell energy spectrum
    E(k) = sum_shell |omega_k|^2 / (2 k^2) ~ k^4 exp(-2 (k/k0)^2); phases are uniform in
    [0, 2 pi) from ``numpy.random.default_rng(seed)``.  The ky = 0 column is made Hermitian
    (omega(-kx, 0) = conj(omega(kx, 0))) so the physical field is real; the field is
    2/3-dealiased and scaled to kinetic energy ``energy``.
    """
    shape = spectral_shape(n, 2)
    rng = np.random.default_rng(seed)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=shape)
    kx, ky = wavenumbers(n, 2)
    k2 = kx * kx + ky * ky
    kk = np.sqrt(k2)
    amp = kk**2.5 * np.exp(-((kk / k0) ** 2))
    spec = amp * np.exp(1j * phase)
    # Hermitian ky = 0 column: rows n-i mirror rows i (0 < i < n/2); kx = 0 and kx = -n/2 real
    col = spec[:, 0]
    half = n // 2
    col[n - half + 1:] = np.conj(col[1:half][::-1])
    col[0] = col[0].real
    col[half] = col[half].real
    spec[:, -1] = spec[:, -1].real
    spec = spec * dealias_mask(n, 2)
    w = hermitian_weights(n, 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        e = 0.5 * np.sum(np.where(k2 > 0, w * np.abs(spec) ** 2 / k2, 0.0)) / float(n) ** 4
    return spec * np.sqrt(energy / e)
