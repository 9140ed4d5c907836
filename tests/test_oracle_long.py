"""The restatement (oracle/psg_oracle.c) over all 10,000 ticks of the 32^3
uniform field against the reference's own run of the same rays
(tests/golden/long32.npz). CPU only: this pins the oracle that the GPU
tests compare with at the configured length, with the bars of
tests/test_gpu_long.py (x_HII within 1e-3 after the last tick, 2e-3 at the
intermediate checkpoints, 99.9th percentile 1e-3; lasthit exact; deposit
counters within 1e-3 in sum)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "long32.npz")), reason="long32.npz not generated")
def test_restatement_10000_ticks_vs_reference(phys):
    from oracle import Oracle
    from psphray_b200 import fields
    g = load_golden("long32.npz")
    w = fields.make_workload("iliev32")
    orc = Oracle(w.field, phys)
    orc.build_tree(8)
    cps = [int(c) for c in g["checkpoints"]]
    for t in range(1, cps[-1] + 1):
        orc.tick(w.schedule.rays_for_tick(t), t, w.tick_time)
        if t in cps:
            d = np.abs(orc.lambdaH - g[f"c{t}_lambdaH"].astype(np.float64))
            assert np.array_equal(orc.lasthit, g[f"c{t}_lasthit"].astype(np.int64)), t
            assert d.max() <= (1e-3 if t == cps[-1] else 2e-3), (t, d.max())
            assert np.quantile(d, 0.999) <= 1e-3, t
            dh = np.abs(orc.hits.astype(np.int64) - g[f"c{t}_hits"])
            assert dh.sum() <= 1e-3 * g[f"c{t}_hits"].sum(), t
