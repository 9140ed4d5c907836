"""The explicit solver (psg_flags.euler: step_evolve_euler(), solve.c:225-316)
against the reference's own code built without USE_LSODA
(tests/golden/euler16.npz, made by tests/golden/make_golden_euler.py):
Step records through psg_step_evolve, and 20 ticks of the 16^3 uniform
field with the photons an early-terminated step leaves for the next one
(loop.c:745)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["iso", "noniso"])
def test_step_evolve_euler_vs_reference(gpu_ctx, units, kind):
    from psphray_b200 import api
    g = load_golden("euler16.npz")
    phys = api.Physics(units, isothermal=(kind == "iso"), euler=True)
    gpu_ctx.set_physics(phys)
    n = len(g[f"{kind}_in_lambdaH"])
    steps = np.zeros(n, api.STEP_DTYPE)
    for k in ("lambdaH", "ie", "yGdepHI", "heat", "time", "nH", "T", "yeMET"):
        steps[k] = g[f"{kind}_in_{k}"]
    out = gpu_ctx.step_evolve(steps)
    # up to 10000 explicit steps each: the right-hand side's rate rows
    # (FP32 values and slopes, 6e-8 relative) against the reference's double table
    assert np.max(np.abs(out["lambdaH"] - g[f"{kind}_out_lambdaH"])) < 1e-6
    assert np.max(np.abs(out["ie"] - g[f"{kind}_out_ie"]) / g[f"{kind}_out_ie"]) < 1e-6
    assert np.array_equal(out["refined"], g[f"{kind}_out_refined"])
    assert np.array_equal(out["step_remain"], g[f"{kind}_out_step_remain"])


def test_ticks_euler_vs_reference(gpu_ctx, units):
    from psphray_b200 import api
    from psphray_b200 import fields
    g = load_golden("euler16.npz")
    f = fields.make_workload("iliev32", n_side=16, nray=16).field
    phys = api.Physics(units, isothermal=True, euler=True)
    gpu_ctx.set_physics(phys)
    gpu_ctx.load(f)
    gpu_ctx.build_tree(8)
    R, tt = int(g["nray"]), float(g["tick_time"])
    rays = g["tick_rays"]
    t = 1
    for batch in (4, 1, 8, 7):
        gpu_ctx.run_ticks(rays[(t - 1) * R:(t - 1 + batch) * R], R, batch, t, tt)
        t += batch
        st = gpu_ctx.state()
        assert np.array_equal(st["lasthit"], g["st_lasthit"][t - 2])
        assert np.array_equal(st["hits"], g["st_hits"][t - 2])
        # the reference sums absorbed photons in float; the explicit steps
        # integrate the difference
        assert np.max(np.abs(st["lambdaH"] - g["st_lambdaH"][t - 2])) < 2e-5
