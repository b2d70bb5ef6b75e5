"""Checkpoint / resume in the reference's format (src/pyspectral/validation.py:204-221).

An ``.npz`` with ``state`` (complex64 for fp32 runs, complex128 otherwise), ``t``, ``amp``
(forcing growth rate) and ``hist`` (the run history as JSON), plus any extra arrays — so a run
chunked with ``run(..., wall_limit=...)`` can stop, be saved and resume, and a checkpoint
written by pyspectral loads here and vice versa.
"""

from __future__ import annotations

import json
from pathlib import Path
from typing import Any

import numpy as np

from pyspectral_b200.simulate import RunResult


def save_checkpoint(path: str | Path, solver: Any, result: RunResult | None = None,
                    **extra: Any) -> Path:
    """Write the solver's state, time, forcing amplitude and run history."""
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    st = solver.get_state()
    if solver.cfg.dtype == "float32":
        st = st.astype(np.complex64)
    hist = json.dumps((result or RunResult()).as_dict())
    with open(p, "wb") as f:
        np.savez(f, state=st, t=solver.t, amp=solver.force_amp, hist=hist, **extra)
    return p


def load_checkpoint(path: str | Path, solver: Any) -> tuple[RunResult, Any]:
    """Restore state, time and forcing amplitude into ``solver``; returns the run history and
    the opened archive (for extra arrays)."""
    z = np.load(Path(path), allow_pickle=False)
    solver.set_state(z["state"])
    solver.t = float(z["t"])
    solver.set_forcing_amplitude(float(z["amp"]))
    h = json.loads(str(z["hist"]))
    res = RunResult(t=h["t"], energy=h["energy"], enstrophy=h["enstrophy"], dt=h["dt"],
                    steps=h["steps"], wall=h["wall_s"])
    return res, z
