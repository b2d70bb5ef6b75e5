"""ORACLE — test infrastructure only; never imported by the product package.

CPU restatement of the learned closure and of the spectral helpers it is built on:

* ``filter_spectrum``: pad_spectrum (src/pyspectral/validation.py:24-35) — zero-pad or
  truncate an r2c spectrum, keeping |k| < min(n, n_to)/2 on every axis, rescaled by
  (n_to/n)^dim — followed, optionally, by the target grid's 2/3 mask.  Pinned by fixtures the
  reference itself produced (the pad_* arrays of tests/golden/reference_vectors.npz, script
  tests/golden/make_golden.py).
* ``snapshot_fields``: the four physical fields of a bank entry (filtered vorticity, its x and y
  derivatives, the subgrid term) from coarse spectra, with numpy's normalised inverse FFT.
* the network (75 -> 64 -> 64 -> 64 -> 1, GELU tanh form), its mean-squared-error gradient and
  Adam, with the device's bf16 rounding points: GEMM operands (inputs, hidden activations,
  layer weights and the back-propagated pre-activation gradients) are rounded to bf16 (nearest,
  ties to even); products are accumulated in float64 here (fp32 on the tensor cores); bias
  folding, GELU, the output layer and the optimiser are fp32.  The closure has no reference
  implementation; this restatement is pinned by finite differences of its own loss
  (tests/test_closure_host.py) and checks the device kernels in tests/test_gpu_closure.py.
* ``pick_tile``: the counter hash that draws training tiles (splitmix64 finaliser).
"""

from __future__ import annotations

import math
from typing import Any

import numpy as np

from oracle.numpy_oracle import dealias_mask, spectral_shape, wavenumbers

K, H, IN, TILE = 80, 64, 75, 128
WSZ = H * K
NPARAM = 3 * WSZ + K
BIAS_IN, BIAS_H = 75, 64
C0, C1 = np.float32(0.7978845608028654), np.float32(0.044715)
F32 = np.float32


# ------------------------------------------------------------------------ spectral helpers
def filter_spectrum(a: np.ndarray, n_to: int, dim: int = 2, dealias: bool = True) -> np.ndarray:
    """pad_spectrum (validation.py:24-35), then the 2/3 mask of grid n_to if ``dealias``."""
    n = a.shape[-2]
    m = min(n, n_to) // 2
    full = np.fft.fftfreq(n_to, 1.0 / n_to).astype(np.int64)
    keep_full = np.abs(full) < m
    dst_full = np.nonzero(keep_full)[0]
    src_full = full[keep_full] % n
    dst_half = src_half = np.arange(m)
    dst_idx = [dst_full] * (dim - 1) + [dst_half]
    src_idx = [src_full] * (dim - 1) + [src_half]
    out = np.zeros(a.shape[: a.ndim - dim] + spectral_shape(n_to, dim), dtype=a.dtype)
    out[(...,) + np.ix_(*dst_idx)] = a[(...,) + np.ix_(*src_idx)] * (n_to / n) ** dim
    if dealias:
        out = out * dealias_mask(n_to, dim)
    return out


def snapshot_fields(wbar: np.ndarray, fine_nl: np.ndarray, coarse_nl: np.ndarray) -> np.ndarray:
    """(4, n, n): omega, d omega/dx, d omega/dy and S = fine_nl - coarse_nl, physical."""
    n = wbar.shape[0]
    mask = dealias_mask(n, 2)
    kx, ky = wavenumbers(n, 2)
    w = wbar * mask
    s = (fine_nl - coarse_nl) * mask
    spec = [w, 1j * kx * w, 1j * ky * w, s]
    return np.stack([np.fft.irfft2(a, s=(n, n)) for a in spec])


# ------------------------------------------------------------------------ numerics
def bf16(x: Any) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even); returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(z: np.ndarray) -> np.ndarray:
    """GELU in the dtype of z (float32 as on the device, float64 for exact checks)."""
    c0, c1 = z.dtype.type(C0), z.dtype.type(C1)
    t = np.tanh(c0 * z * (1 + c1 * z * z))
    return (0.5 * z * (1 + t)).astype(z.dtype)


def gelu_d(z: np.ndarray) -> np.ndarray:
    c0, c1 = z.dtype.type(C0), z.dtype.type(C1)
    z2 = z * z
    t = np.tanh(c0 * z * (1 + c1 * z2))
    return (0.5 * (1 + t) + 0.5 * z * (1 - t * t) * c0 * (1 + 3 * c1 * z2)).astype(z.dtype)


def _mm(a: np.ndarray, b: np.ndarray, ft: Any = F32) -> np.ndarray:
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(ft)


def mix64(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def pick_tile(seed: int, step: int, i: np.ndarray, count: int, n: int) -> tuple[np.ndarray, ...]:
    """(snapshot, row, segment) of training tiles i of ``step``."""
    i = np.asarray(i, dtype=np.uint64)
    key = (np.uint64(step) << np.uint64(32)) | (i & np.uint64(0xFFFFFFFF))
    with np.errstate(over="ignore"):
        h = mix64(np.uint64(seed) + mix64(key))
    lo = h & np.uint64(0xFFFFFFFF)
    snap = (h >> np.uint64(32)) % np.uint64(count)
    row = lo % np.uint64(n)
    seg = (lo // np.uint64(n)) % np.uint64(n // TILE)
    return snap.astype(np.int64), row.astype(np.int64), seg.astype(np.int64)


# ------------------------------------------------------------------------ network
def tile_features(fields: np.ndarray, inscale: np.ndarray, row: int, y0: int) -> np.ndarray:
    """(128, 80) inputs of the points (row, y0 .. y0+127): 75 stencil values, 1, zeros."""
    n = fields.shape[-1]
    rows = (row + np.arange(-2, 3)) % n
    cols = (y0 + np.arange(-2, TILE + 2)) % n
    st = fields[:3][:, rows][:, :, cols].astype(F32) * np.asarray(inscale, F32)[:, None, None]
    X = np.zeros((TILE, K), F32)
    p = np.arange(TILE)
    for f in range(3):
        for dx in range(5):
            for dy in range(5):
                X[:, f * 25 + dx * 5 + dy] = st[f, dx, p + dy]
    X[:, BIAS_IN] = 1.0
    return X


def _extend(h: np.ndarray) -> np.ndarray:
    out = np.zeros((h.shape[0], K), h.dtype)
    out[:, :H] = h
    out[:, BIAS_H] = 1.0
    return out


def forward(params: np.ndarray, X: np.ndarray, exact: bool = False) -> dict[str, Any]:
    """Tile forward pass.  exact=True drops the bf16 rounding and runs in float64 (the smooth
    function whose derivative the backward pass restates)."""
    ft = np.float64 if exact else F32
    rnd = (lambda a: np.asarray(a, np.float64)) if exact else bf16
    W = rnd(params[: 3 * WSZ]).reshape(3, H, K)
    w4 = params[3 * WSZ:].astype(ft)
    xb = rnd(X)
    z1 = _mm(xb, W[0].T, ft)
    h1e = _extend(rnd(gelu(z1)))
    z2 = _mm(h1e, W[1].T, ft)
    h2e = _extend(rnd(gelu(z2)))
    z3 = _mm(h2e, W[2].T, ft)
    h3 = gelu(z3)
    y = (w4[BIAS_H] + h3.astype(np.float64) @ w4[:H].astype(np.float64)).astype(ft)
    return {"W": W, "w4": w4, "x": xb, "z1": z1, "h1e": h1e, "z2": z2, "h2e": h2e, "z3": z3,
            "h3": h3, "y": y, "rnd": rnd, "ft": ft}


def backward(c: dict[str, Any], target: np.ndarray, inv_batch: float) -> tuple[np.ndarray, float]:
    """Gradient of mean((y - target)^2) (inv_batch = 1 / batch points) and the tile's sum of
    squared residuals."""
    ft, rnd = c["ft"], c["rnd"]
    r = (c["y"] - target.astype(ft)).astype(ft)
    dy = (2 * r * ft(inv_batch)).astype(ft)
    W, w4 = c["W"], c["w4"]
    g = np.zeros(NPARAM, np.float64)
    dz3 = rnd(dy[:, None] * w4[None, :H] * gelu_d(c["z3"]))
    g[3 * WSZ: 3 * WSZ + H] = c["h3"].astype(np.float64).T @ dy.astype(np.float64)
    g[3 * WSZ + BIAS_H] = float(dy.astype(np.float64).sum())
    g[2 * WSZ: 3 * WSZ] = (dz3.astype(np.float64).T @ c["h2e"].astype(np.float64)).ravel()
    dh2 = _mm(dz3, W[2], ft)[:, :H]
    dz2 = rnd(dh2 * gelu_d(c["z2"]))
    g[WSZ: 2 * WSZ] = (dz2.astype(np.float64).T @ c["h1e"].astype(np.float64)).ravel()
    dh1 = _mm(dz2, W[1], ft)[:, :H]
    dz1 = rnd(dh1 * gelu_d(c["z1"]))
    g[0:WSZ] = (dz1.astype(np.float64).T @ c["x"].astype(np.float64)).ravel()
    return g, float((r.astype(np.float64) ** 2).sum())


def batch_grad(params: np.ndarray, bank: np.ndarray, inscale: np.ndarray, outscale: float,
               seed: int, step: int, ntiles: int) -> tuple[np.ndarray, float]:
    """Gradient and mean loss of one training step (bank: (count, 4, n, n))."""
    count, n = bank.shape[0], bank.shape[-1]
    snap, row, seg = pick_tile(seed, step, np.arange(ntiles), count, n)
    inv_batch = 1.0 / (ntiles * TILE)
    g = np.zeros(NPARAM)
    loss = 0.0
    for s, r, q in zip(snap, row, seg):
        y0 = int(q) * TILE
        X = tile_features(bank[s], inscale, int(r), y0)
        target = bank[s, 3, r, y0: y0 + TILE].astype(F32) * F32(1.0 / outscale)
        gt, lt = backward(forward(params, X), target, inv_batch)
        g += gt
        loss += lt
    return g, loss * inv_batch


def learning_rate(t: int, lr: float, lr_min: float, total: int, warmup: int) -> float:
    if warmup > 0 and t <= warmup:
        return lr * t / warmup
    span = total - warmup if total > warmup else 1
    x = min((t - warmup) / span, 1.0)
    return lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * x))


def adam(params: np.ndarray, m: np.ndarray, v: np.ndarray, g: np.ndarray, t: int, lr: float,
         lr_min: float = 0.0, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8,
         total: int = 1, warmup: int = 0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """One Adam update (step t, 1-based) in float64; returns (params, m, v)."""
    a = learning_rate(t, lr, lr_min, total, warmup)
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return params - a * mh / (np.sqrt(vh) + eps), m, v


def infer_field(params: np.ndarray, fields: np.ndarray, inscale: np.ndarray, outscale: float,
                clip: bool = False) -> np.ndarray:
    """Closure term S at every point of an n x n field (fields: omega, omega_x, omega_y)."""
    n = fields.shape[-1]
    out = np.zeros((n, n), F32)
    for row in range(n):
        for seg in range(n // TILE):
            y0 = seg * TILE
            y = forward(params, tile_features(fields, inscale, row, y0))["y"]
            s = (F32(outscale) * y).astype(F32)
            if clip:
                s = np.where(s * fields[0, row, y0: y0 + TILE] > 0, F32(0), s)
            out[row, y0: y0 + TILE] = s
    return out
