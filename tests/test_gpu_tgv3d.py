"""3D Taylor-Green vortex at Re = 1600 to t = 10 against the fp64 oracle's run at 128^3, and the
IF-RK4 temporal order on the device.

The reference validates this flow by its dissipation eps(t) = 2 nu Z(t)
(src/pyspectral/validation.py:152-200).  tests/golden/tgv3d_re1600_n128_fp64.json is the
oracle's run (tests/golden/make_tgv3d_oracle.py: rotational form, CFL 0.5, dt_max 0.05, dt
refreshed every 10 steps, records every 0.1); the device runs the same schedule through
``simulate.run`` on both 3D engines (cuFFT, and the fused passes of this library).  fp64: every
record's energy and enstrophy within 1e-9 relative, and the
same number of steps; the Basdevant form reaches the same flow (the two forms differ by a
gradient that the projection removes).  fp32: the dissipation history within 1e-3 of the peak.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from pyspectral_b200.validation import TGV_NU, compare_dissipation, tgv3d

pytestmark = pytest.mark.gpu

FIX = json.loads((Path(__file__).parent / "golden" / "tgv3d_re1600_n128_fp64.json").read_text())
REF = {"t": FIX["t"], "dissipation": [2.0 * TGV_NU * z for z in FIX["enstrophy"]]}


ENGINES = ["b200/fused-inplace-graph", "b200/fused-fft-graph"]  # cuFFT, hand-written passes


@pytest.mark.parametrize("variant", ENGINES)
@pytest.mark.parametrize("form", ["rotational", "basdevant"])
def test_tgv3d_128_fp64_matches_the_oracle_to_t10(form, variant):
    r = tgv3d(variant, FIX["n"], FIX["t_end"], cfl=FIX["cfl"],
              dtype="float64", diag_dt=FIX["diag_dt"], form=form)
    assert r["steps"] == FIX["steps"]
    assert np.allclose(r["t"], FIX["t"], rtol=0, atol=1e-12)
    for key in ("energy", "enstrophy"):
        a, b = np.array(r[key]), np.array(FIX[key])
        assert np.abs(a / b - 1).max() < 1e-9, key


@pytest.mark.parametrize("variant", ENGINES)
def test_tgv3d_128_fp32_dissipation_follows_the_oracle(variant):
    r = tgv3d(variant, FIX["n"], FIX["t_end"], cfl=FIX["cfl"],
              dtype="float32", diag_dt=FIX["diag_dt"], form="rotational")
    c = compare_dissipation(np.array(r["t"]), np.array(r["dissipation_2nuZ"]), REF)
    assert c["max_abs_err_over_peak"] < 1e-3
    assert abs(c["peak_rel_err"]) < 1e-3


@pytest.mark.parametrize("variant", ["b200/fused-inplace-graph", "b200/fused-fft-graph"])
def test_ifrk4_self_convergence_is_fourth_order_on_the_device(variant):
    """validation.py:86-100 on the device engines (fp64, 64^2 nonlinear flow): order ~ 4."""
    from pyspectral_b200.validation import temporal_convergence

    r = temporal_convergence(variant)
    assert 3.8 < r["order"] < 4.3, r
    assert r["err"][-1] < 1e-8


def test_spectral_convergence_in_n_matches_the_oracle():
    """validation.py:103-119 on the device (fp64): the error against the 192^2 run falls
    exponentially with n, and every grid's error equals the oracle's (its states agree to
    round-off)."""
    from oracle.numpy_oracle import OracleSolver
    from pyspectral_b200 import initial
    from pyspectral_b200.validation import pad_spectrum, spatial_convergence

    r = spatial_convergence("b200/fused-inplace-graph")

    def solve(n):
        s = OracleSolver(n, 2, nu=r["nu"])
        s.set_state(initial.to_spectral(initial.smooth_2d(n), 2))
        s.advance(int(round(r["t_end"] / r["dt"])), r["dt"])
        return s.get_state()

    n_ref = r["n_ref"]
    w_ref = np.fft.irfftn(solve(n_ref), s=(n_ref, n_ref), axes=(0, 1))
    for n, e in zip(r["n"], r["err"]):
        w = np.fft.irfftn(pad_spectrum(solve(n), n_ref), s=(n_ref, n_ref), axes=(0, 1))
        want = float(np.abs(w - w_ref).max() / np.abs(w_ref).max())
        assert abs(e - want) <= 1e-3 * want + 1e-12, (n, e, want)
    err = dict(zip(r["n"], r["err"]))
    assert err[64] < 1e-9 < err[32] < err[16]
