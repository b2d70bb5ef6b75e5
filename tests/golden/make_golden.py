"""Generate tests/golden/reference_vectors.npz by running the reference implementation.

Run where pyspectral's sources are available, with PYSPECTRAL_SRC naming its src/ directory:

    PYSPECTRAL_SRC=/path/to/pyspectral/src python tests/golden/make_golden.py

Every array is produced by pyspectral itself (NumpySolver, Diagnostics, initial, validation):
the cross-backend parity protocol of tests/test_backends.py:24-47 (forcing and dt changes), the
exact Taylor-Green decay of tests/test_backends.py:50-59, explicit RK4, the advective form,
fp32 oracle runs, diagnostics values and initial conditions.  The GPU box never needs the
reference: the tests read these vectors only.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

SRC = os.environ.get("PYSPECTRAL_SRC")
if not SRC:
    sys.exit("set PYSPECTRAL_SRC to pyspectral's src/ directory")
sys.path.insert(0, SRC)

from pyspectral import initial  # noqa: E402
from pyspectral.backends.numpy_ref import NumpySolver  # noqa: E402
from pyspectral.config import Config  # noqa: E402
from pyspectral.diagnostics import Diagnostics  # noqa: E402
from pyspectral.validation import pad_spectrum  # noqa: E402

OUT = Path(__file__).with_name("reference_vectors.npz")


def parity_case(dim: int, form: str, alpha_kmax: float, dtype: str = "float64"):
    """tests/test_backends.py:24-47 protocol on the oracle."""
    n = 32 if dim == 2 else 16
    cfg = Config(n=n, dim=dim, nu=0.01, alpha=0.5, alpha_kmax=alpha_kmax, force_amp=0.3,
                 force_klo=1, force_khi=2.5, dtype=dtype, form=form)
    ic = (initial.to_spectral(initial.random_2d(n, k0=4), 2) if dim == 2
          else initial.to_spectral(initial.random_3d(n, k0=2), 3))
    s = NumpySolver(cfg)
    s.set_state(ic)
    s.advance(5, 0.01)
    s.set_forcing_amplitude(0.1)
    s.advance(3, 0.007)
    return ic, s.get_state()


def main() -> None:
    out: dict[str, np.ndarray] = {}
    for dim, form in [(2, "basdevant"), (3, "basdevant"), (3, "rotational")]:
        for akm in (0.0, 2.0):
            ic, fin = parity_case(dim, form, akm)
            key = f"parity_{dim}d_{form}_akm{int(akm)}"
            out[key + "_ic"] = ic
            out[key + "_final"] = fin
            if akm == 2.0:
                _, f32 = parity_case(dim, form, akm, "float32")
                out[key + "_final_fp32"] = f32
    # advective 2D form (same protocol, form only available on the oracle)
    ic, fin = parity_case(2, "advective", 2.0)
    out["parity_2d_advective_akm2_final"] = fin
    # exact 2D Taylor-Green decay (tests/test_backends.py:50-59)
    n, nu = 32, 0.05
    s = NumpySolver(Config(n=n, dim=2, nu=nu, dtype="float64"))
    w0 = initial.to_spectral(initial.taylor_green_2d(n), 2)
    s.set_state(w0)
    s.advance(20, 0.05)
    out["tgv2d_ic"] = w0
    out["tgv2d_final"] = s.get_state()
    # explicit RK4 on a nonlinear 2D flow
    w0 = initial.to_spectral(initial.smooth_2d(32), 2)
    s = NumpySolver(Config(n=32, dim=2, nu=0.01, dtype="float64"), integrator="rk4")
    s.set_state(w0)
    s.advance(5, 0.01)
    out["rk4_2d_ic"] = w0
    out["rk4_2d_final"] = s.get_state()
    # diagnostics
    u3 = initial.to_spectral(initial.random_3d(16, k0=2), 3)
    w2 = initial.to_spectral(initial.random_2d(32, k0=4), 2)
    for key, st, dim, nn in (("diag3d", u3, 3, 16), ("diag2d", w2, 2, 32)):
        d = Diagnostics(nn, dim)
        out[key + "_state"] = st
        out[key + "_values"] = np.array([d.energy(st), d.enstrophy(st), d.palinstrophy(st),
                                         d.band_energy(st, 1.0, 2.5), d.max_velocity_sum(st)])
        out[key + "_spectrum"] = d.spectrum(st)[1]
    # initial conditions
    out["ic_random_2d_n32_k4_s0"] = initial.random_2d(32, k0=4)
    out["ic_random_3d_n16_k2_s0"] = initial.random_3d(16, k0=2)
    out["ic_smooth_2d_n32"] = initial.smooth_2d(32)
    out["ic_tgv3d_n16_spec"] = initial.to_spectral(initial.taylor_green_3d(16), 3)
    # spectral filter used by the closure pipeline (validation.py:25-35)
    out["pad_tgv2d_16_to_32"] = pad_spectrum(initial.to_spectral(initial.taylor_green_2d(16), 2),
                                             32, 2)
    rng = np.random.default_rng(7)
    for n, n_to, dim in ((32, 16, 2), (16, 24, 2), (24, 24, 2), (16, 8, 3), (8, 12, 3)):
        shp = (n,) * (dim - 1) + (n // 2 + 1,)
        a = rng.normal(size=shp) + 1j * rng.normal(size=shp)
        key = f"pad_rand{dim}d_{n}_to_{n_to}"
        out[key + "_in"] = a
        out[key] = pad_spectrum(a, n_to, dim)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1024:.0f} KiB, {len(out)} arrays)")


if __name__ == "__main__":
    main()
