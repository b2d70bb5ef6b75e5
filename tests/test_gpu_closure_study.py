"""The learned-closure study end to end on its reduced configuration: batched-engine data,
tcgen05 training, a-posteriori test against the DNS, and the DNS fallback."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_small_study_runs_end_to_end():
    from pyspectral_b200 import closure_les as cl

    sc = cl.StudyConfig.small()
    res = cl.run_study(sc)
    net = res.pop("net")
    assert res["data"]["snapshots"] == sc.snapshots
    assert net.bank_count == sc.snapshots + min(4, sc.test_seeds)
    tr = res["train"]
    assert np.isfinite(tr["loss_last"]) and tr["loss_last"] < tr["loss_first"]
    ev = res["evaluation"]
    assert ev["records_per_run"] >= 3
    assert ev["closure"]["finite"] and ev["no_closure"]["finite"]
    assert len(ev["dns_spectrum"]) == sc.k_check + 1
    assert ev["accepted"] == (ev["closure"]["e_err_max"] <= sc.err_bound)
    assert ev["dns_wall_s"] > 0 and ev["les_wall_s"] > 0
    assert -1.0 <= res["a_priori_corr"] <= 1.0

    # the fallback picks the DNS for a rejected closure and the coarse run otherwise
    st = cl.fine_states(sc, [7])[0]
    s_dns, path = cl.run_coarse_or_fine(net, False, sc, st, 0.1)
    assert path == "dns" and s_dns.n == sc.n_fine
    s_les, path = cl.run_coarse_or_fine(net, True, sc, st, 0.1)
    assert path == "closure" and s_les.n == sc.n_coarse
    assert np.all(np.isfinite(s_les.get_state()))
