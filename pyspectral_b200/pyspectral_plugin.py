"""Registration of the B200 engine as variants of pyspectral's own backend registry.

pyspectral lists its solvers in ``pyspectral.backends.REGISTRY`` (src/pyspectral/backends/
__init__.py:67-91); a ``Variant`` imports its class from ``pyspectral.backends.<module>``
(:35-38).  :func:`register` appends entries whose ``load()`` returns a class that is at the same
time a :class:`pyspectral_b200.solver.B200Solver` and a subclass of pyspectral's
``SpectralSolver`` (src/pyspectral/backends/base.py:19), so ``make_solver("b200", cfg)``,
``pyspectral run --backend b200`` and the reference's own tests pick it up unchanged.

Requires pyspectral to be importable; this module is not imported by the rest of the package.
"""

from __future__ import annotations

from typing import Any

_CLASSES: dict[str, type] = {}


def _plugin_class(base_name: str) -> type:
    """B200 solver class ``base_name`` re-based on pyspectral's SpectralSolver."""
    if base_name in _CLASSES:
        return _CLASSES[base_name]
    from pyspectral.backends.base import BackendUnavailable as RefUnavailable
    from pyspectral.backends.base import SpectralSolver as RefSolver

    from pyspectral_b200 import solver as mod
    from pyspectral_b200.base import BackendUnavailable

    impl = getattr(mod, base_name)

    def __init__(self: Any, cfg: Any) -> None:  # noqa: N807
        # pyspectral callers catch pyspectral's own BackendUnavailable
        try:
            impl.__init__(self, cfg)
        except BackendUnavailable as e:
            raise RefUnavailable(str(e)) from e

    cls = type(f"Pyspectral{base_name}", (impl, RefSolver),
               {"__module__": __name__, "__init__": __init__})
    _CLASSES[base_name] = cls
    return cls


def register(registry: list | None = None) -> list[Any]:
    """Append the b200 variants to pyspectral's REGISTRY (idempotent); returns them."""
    from dataclasses import dataclass

    from pyspectral.backends import REGISTRY, Variant

    reg = REGISTRY if registry is None else registry

    @dataclass(frozen=True)
    class B200Variant(Variant):
        """Variant whose class lives in pyspectral_b200 instead of pyspectral.backends."""

        def load(self) -> type:
            return _plugin_class(self.cls)

    entries = [
        B200Variant("b200", "fused-inplace", "pyspectral_b200.solver", "B200EagerSolver",
                    "#17becf", True, "B200 sm_100a fused kernels + in-place batched cuFFT"),
        B200Variant("b200", "fused-inplace-lean", "pyspectral_b200.solver", "B200LeanSolver",
                    "#17becf", True, "B200, single-field cuFFT plans, graph step"),
        B200Variant("b200", "fused-inplace-graph", "pyspectral_b200.solver", "B200Solver",
                    "#17becf", True, "B200, whole step in one CUDA graph, device-resident dt",
                    default=True),
        B200Variant("b200", "fused-fft-graph", "pyspectral_b200.solver", "B200FusedSolver",
                    "#17becf", True, "B200 2D, hand-written FFTs fused with the pointwise "
                    "phases, no cuFFT"),
    ]
    have = {v.name for v in reg}
    added = [e for e in entries if e.name not in have]
    reg.extend(added)
    return added
