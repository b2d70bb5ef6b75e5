"""Array shim for code written against pyspectral's ``ops`` protocol
(``TorchOps``, src/pyspectral/ops.py:85-123): device arrays here are torch CUDA tensors.

Only the host-side members (conversion, scalar reads, synchronisation) are provided: the
transforms and reductions that pyspectral's generic ``Diagnostics`` builds from ``irfftn`` and
``bincount`` run here as the engine's own kernels (:mod:`pyspectral_b200.diagnostics`), so no
library FFT is reachable through this shim.
"""

from __future__ import annotations

from typing import Any

import numpy as np


class TorchOps:
    """torch implementation of the shim."""

    name = "torch"

    def __init__(self, device: str = "cuda") -> None:
        import torch

        self.torch = torch
        self.device = device

    def asarray(self, a: np.ndarray, dtype: Any = None) -> Any:
        t = self.torch.as_tensor(np.ascontiguousarray(a), device=self.device)
        return t if dtype is None else t.to(dtype)

    def to_numpy(self, a: Any) -> np.ndarray:
        if isinstance(a, np.ndarray):
            return a
        return a.detach().cpu().numpy()

    def to_int(self, a: Any) -> Any:
        return a.to(self.torch.int64)

    def sqrt(self, a: Any) -> Any:
        return self.torch.sqrt(a)

    def amax_abs(self, a: Any) -> float:
        return float(a.abs().max())

    def scalar(self, a: Any) -> float:
        return float(a)

    def synchronize(self) -> None:
        self.torch.cuda.synchronize()
