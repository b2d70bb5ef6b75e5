"""Host logic of the validation runs: the oracle's CFL run loop pinned to the reference's own
driver (src/pyspectral/simulate.py:40-96 with NumpySolver), and the dissipation comparison."""

from __future__ import annotations

import importlib.util
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.numpy_oracle import OracleSolver, run_cfl
from pyspectral_b200 import initial
from pyspectral_b200.validation import TGV_NU, compare_dissipation

# pyspectral's source tree (its src/ directory), when the reference itself is available
_SRC = os.environ.get("PYSPECTRAL_SRC", "")


def _reference_importable() -> bool:
    if importlib.util.find_spec("pyspectral") is None and _SRC and Path(_SRC).exists():
        sys.path.append(_SRC)
    return importlib.util.find_spec("pyspectral") is not None


@pytest.mark.skipif(not _reference_importable(), reason="pyspectral not importable (set PYSPECTRAL_SRC to its src/ directory)")
@pytest.mark.parametrize("form", ["rotational", "basdevant"])
def test_oracle_run_loop_matches_the_reference_driver(form):
    from pyspectral.backends.numpy_ref import NumpySolver
    from pyspectral.config import Config as RefConfig
    from pyspectral.simulate import run as ref_run

    n, t_end, diag_dt = 12, 0.35, 0.1
    ic = initial.to_spectral(initial.taylor_green_3d(n), 3)
    ref = NumpySolver(RefConfig(n=n, dim=3, nu=TGV_NU, form=form, dtype="float64"))
    ref.set_state(ic)
    r = ref_run(ref, t_end, cfl=0.5, dt_max=0.05, cfl_every=10, diag_dt=diag_dt)
    s = OracleSolver(n, 3, nu=TGV_NU, form=form)
    s.set_state(ic)
    o = run_cfl(s, t_end, cfl=0.5, dt_max=0.05, cfl_every=10, diag_dt=diag_dt)
    assert o["steps"] == r.steps
    assert np.allclose(o["t"], r.t, rtol=0, atol=1e-14)
    assert np.allclose(o["energy"], r.energy, rtol=1e-12, atol=0)
    assert np.allclose(o["enstrophy"], r.enstrophy, rtol=1e-12, atol=0)
    assert np.abs(s.get_state() - ref.get_state()).max() <= 1e-12 * np.abs(ref.get_state()).max()


def test_compare_dissipation_peak_and_error():
    tr = np.linspace(0.0, 10.0, 101)
    er = np.exp(-((tr - 9.0) ** 2))  # peak 1 at t = 9
    t = np.linspace(0.0, 12.0, 121)  # the reference samples and beyond: interpolation exact
    eps = 1.02 * np.exp(-((t - 9.0) ** 2))
    c = compare_dissipation(t, eps, {"t": tr, "dissipation": er})
    assert c["ref_peak_value"] == pytest.approx(1.0)
    assert c["ref_peak_time"] == pytest.approx(9.0)
    assert c["peak_rel_err"] == pytest.approx(0.02, rel=1e-6)
    # the error is taken over the reference's span only (t <= 10 here)
    assert c["max_abs_err_over_peak"] == pytest.approx(0.02, rel=1e-3)
