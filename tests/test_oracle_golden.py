"""The oracle pinned against vectors produced by the reference itself (tests/golden).

CPU only.  If these pass, the NumPy restatement in oracle/ computes what pyspectral's
NumpySolver / Diagnostics / initial compute, to round-off.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle.numpy_oracle import OracleDiagnostics, OracleSolver

GOLDEN = np.load(Path(__file__).parent / "golden" / "reference_vectors.npz")


def rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.abs(a - b).max() / np.abs(b).max())


def _parity_run(dim: int, form: str, akm: float, dtype: str = "float64") -> np.ndarray:
    n = 32 if dim == 2 else 16
    key = f"parity_{dim}d_{'basdevant' if form == 'advective' else form}_akm{int(akm)}"
    s = OracleSolver(n, dim, nu=0.01, alpha=0.5, alpha_kmax=akm, force_amp=0.3, force_klo=1,
                     force_khi=2.5, dtype=dtype, form=form)
    s.set_state(GOLDEN[key + "_ic"])
    s.advance(5, 0.01)
    s.set_forcing_amplitude(0.1)
    s.advance(3, 0.007)
    return s.get_state()


@pytest.mark.parametrize("dim,form", [(2, "basdevant"), (3, "basdevant"), (3, "rotational")])
@pytest.mark.parametrize("akm", [0.0, 2.0])
def test_oracle_matches_reference_fp64(dim, form, akm):
    key = f"parity_{dim}d_{form}_akm{int(akm)}"
    assert rel(_parity_run(dim, form, akm), GOLDEN[key + "_final"]) < 1e-13


@pytest.mark.parametrize("dim,form", [(2, "basdevant"), (3, "basdevant"), (3, "rotational")])
def test_oracle_matches_reference_fp32(dim, form):
    key = f"parity_{dim}d_{form}_akm2"
    assert rel(_parity_run(dim, form, 2.0, "float32"), GOLDEN[key + "_final_fp32"]) < 1e-6


def test_oracle_advective_form():
    assert rel(_parity_run(2, "advective", 2.0), GOLDEN["parity_2d_advective_akm2_final"]) < 1e-13


def test_oracle_tgv2d():
    s = OracleSolver(32, 2, nu=0.05)
    s.set_state(GOLDEN["tgv2d_ic"])
    s.advance(20, 0.05)
    assert rel(s.get_state(), GOLDEN["tgv2d_final"]) < 1e-14


def test_oracle_rk4():
    s = OracleSolver(32, 2, nu=0.01, integrator="rk4")
    s.set_state(GOLDEN["rk4_2d_ic"])
    s.advance(5, 0.01)
    assert rel(s.get_state(), GOLDEN["rk4_2d_final"]) < 1e-14


@pytest.mark.parametrize("key,dim,n", [("diag3d", 3, 16), ("diag2d", 2, 32)])
def test_oracle_diagnostics(key, dim, n):
    d = OracleDiagnostics(n, dim)
    st = GOLDEN[key + "_state"]
    vals = [d.energy(st), d.enstrophy(st), d.palinstrophy(st), d.band_energy(st, 1.0, 2.5),
            d.max_velocity_sum(st)]
    np.testing.assert_allclose(vals, GOLDEN[key + "_values"], rtol=1e-13)
    np.testing.assert_allclose(d.spectrum(st)[1], GOLDEN[key + "_spectrum"], rtol=1e-12,
                               atol=1e-18)
