"""Run configuration: the parameters of one periodic-box IF-RK4 run.

Same fields, defaults, validation and FFT-count tables as the reference's ``Config``
(src/pyspectral/config.py:12-92), so a configuration built for pyspectral means the same thing
here.  The linear operator integrated by the integrating factor is

    L(k) = -(nu k^2 + alpha [k^2 <= drag_k2]) + force_amp [force_klo <= |k| <= force_khi]
"""

from __future__ import annotations

from dataclasses import dataclass, replace

FORMS_2D = ("basdevant", "advective")
FORMS_3D = ("basdevant", "rotational")
DEALIAS = ("2/3", "phase-shift")

# (dim, form) -> (inverse FFTs, forward FFTs) per right-hand-side evaluation
_SPLIT = {
    (2, "basdevant"): (2, 2),   # u, v -> v^2 - u^2, uv
    (2, "advective"): (4, 1),   # u, v, w_x, w_y -> u.grad w
    (3, "basdevant"): (3, 5),   # u -> traceless u_i u_j
    (3, "rotational"): (6, 3),  # u, omega -> u x omega
}


@dataclass(frozen=True)
class Config:
    """Physical and numerical parameters of a run on the ``[0, 2 pi)^dim`` box."""

    n: int
    dim: int = 2
    nu: float = 1e-3
    alpha: float = 0.0
    alpha_kmax: float = 0.0
    force_amp: float = 0.0
    force_klo: float = 0.0
    force_khi: float = 0.0
    dtype: str = "float32"
    form: str = "auto"
    dealias: str = "2/3"

    def __post_init__(self) -> None:
        if self.dim not in (2, 3):
            raise ValueError("dim must be 2 or 3")
        if self.n < 8 or self.n % 2:
            raise ValueError("n must be even and >= 8")
        if self.dtype not in ("float32", "float64"):
            raise ValueError("dtype must be float32 or float64")
        allowed = FORMS_2D if self.dim == 2 else FORMS_3D
        if self.form != "auto" and self.form not in allowed:
            raise ValueError(f"form must be one of {allowed} for dim={self.dim}")
        if self.dealias not in DEALIAS:
            raise ValueError(f"dealias must be one of {DEALIAS}")

    def resolved_form(self, default: str | None = None) -> str:
        """Concrete nonlinear form: ``auto`` becomes ``default`` (or basdevant)."""
        return self.form if self.form != "auto" else (default or "basdevant")

    @property
    def drag_k2(self) -> float:
        """Upper k^2 of the drag band; effectively infinite for uniform drag."""
        return self.alpha_kmax * self.alpha_kmax if self.alpha_kmax > 0 else 1e30

    @property
    def is_fp64(self) -> bool:
        return self.dtype == "float64"

    def with_(self, **kw: object) -> Config:
        """Copy with some fields replaced."""
        return replace(self, **kw)  # type: ignore[arg-type]


def fft_split(dim: int, form: str) -> tuple[int, int]:
    """(inverse, forward) real FFTs per right-hand-side evaluation."""
    return _SPLIT[(dim, form)]


def ffts_per_stage(dim: int, form: str) -> int:
    """Real FFTs per right-hand-side evaluation (4 stages per step)."""
    a, b = _SPLIT[(dim, form)]
    return a + b
