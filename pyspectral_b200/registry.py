"""Variant registry, same shape as the reference's (src/pyspectral/backends/__init__.py:17-117).

Each entry names a solver class of this package; classes load lazily, so a missing library or
GPU only marks the entries unavailable.  ``pyspectral_b200.pyspectral_plugin`` adds the same
entries to pyspectral's own registry.
"""

from __future__ import annotations

import importlib
from dataclasses import dataclass, field
from typing import Any

from pyspectral_b200.base import BackendUnavailable, SpectralSolver
from pyspectral_b200.config import Config


@dataclass(frozen=True)
class Variant:
    """One ``backend/variant`` entry."""

    backend: str
    variant: str
    module: str
    cls: str
    gpu: bool
    description: str
    kwargs: dict[str, Any] = field(default_factory=dict)
    default: bool = False

    @property
    def name(self) -> str:
        return f"{self.backend}/{self.variant}"

    def load(self) -> type[SpectralSolver]:
        mod = importlib.import_module(f"pyspectral_b200.{self.module}")
        return getattr(mod, self.cls)

    def available(self) -> tuple[bool, str]:
        try:
            return self.load().available()
        except Exception as e:  # noqa: BLE001
            return False, f"{type(e).__name__}: {e}"

    def make(self, cfg: Config) -> SpectralSolver:
        cls = self.load()
        ok, why = cls.available()
        if not ok:
            raise BackendUnavailable(f"{self.name}: {why}")
        return cls(cfg, **self.kwargs)


REGISTRY: list[Variant] = [
    Variant("b200", "fused-inplace", "solver", "B200EagerSolver", True,
            "sm_100a fused pointwise kernels + in-place batched cuFFT, plain launches"),
    Variant("b200", "fused-inplace-lean", "solver", "B200LeanSolver", True,
            "as above, single-field cuFFT plans (cuFFT workspace of one field), graph step"),
    Variant("b200", "fused-inplace-graph", "solver", "B200Solver", True,
            "as above, batched plans, whole step replayed from one CUDA graph with "
            "device-resident dt/forcing", default=True),
    Variant("b200", "fused-fft-graph", "solver", "B200FusedSolver", True,
            "hand-written sm_100a FFTs fused with every pointwise phase over the dealiased "
            "modes (2D: row + column pass per RK stage; 3D: y, z, y and x passes), no cuFFT, "
            "one CUDA graph per step"),
]


def names() -> list[str]:
    return [v.name for v in REGISTRY]


def get(name: str) -> Variant:
    """``backend/variant`` or a bare backend name (its default entry)."""
    for v in REGISTRY:
        if v.name == name:
            return v
    matches = [v for v in REGISTRY if v.backend == name]
    if matches:
        return next((v for v in matches if v.default), matches[-1])
    raise KeyError(f"unknown backend {name!r}; choose from {names()}")


def make_solver(name: str, cfg: Config) -> SpectralSolver:
    return get(name).make(cfg)


def available() -> list[tuple[Variant, bool, str]]:
    return [(v, *v.available()) for v in REGISTRY]
