"""psg_step_evolve_noalloc (a fixed in-library device buffer instead of the
context's growable scratch) against psg_step_evolve, both through the C ABI,
on two calls in a row; against the oracle's solver directly; that repeated
calls leave the device's free memory unchanged; and its size limit. Both
entry points run the same kernel, so their results must agree to the
tolerance of the step_evolve parity tests (they are in fact identical).

It is for hosts that cannot allocate device memory while a step is under
way (their pool allocator already holds the free memory, or they cannot
afford the synchronisation of cudaMalloc), so the property that matters is
that a call takes no memory at all."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_field, load_golden

pytestmark = pytest.mark.gpu

MAX_STEPS = 16384          # PSG_NOALLOC_MAX_STEPS in include/psg.h


def _steps(f, phys, tick_time, seed, n):
    from psphray_b200.api import STEP_DTYPE
    rng = np.random.default_rng(seed)
    s = np.zeros(n, STEP_DTYPE)
    s["lambdaH"] = 10 ** rng.uniform(-6, 0, n)
    s["ie"] = float(f.ie[0]) * 10 ** rng.uniform(-0.5, 0.5, n)
    s["yGdepHI"] = np.where(rng.random(n) < 0.7, 10 ** rng.uniform(-4, 0, n), 0.0)
    s["heat"] = s["yGdepHI"] * 1e-3 * float(f.ie[0])
    s["time"] = tick_time * rng.integers(1, 200, n)
    s["nH"] = float(f.rho[0]) * phys.unit("H_PER_MASS")
    s["T"] = 1e4
    return s


def _noalloc(ctx, steps):
    from psphray_b200 import api
    L = api.lib()
    fn = L.psg_step_evolve_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    fn.restype = C.c_int
    out = np.ascontiguousarray(steps.copy(), api.STEP_DTYPE)
    return fn(ctx.h, out.ctypes.data, len(out)), out


@pytest.mark.parametrize("iso", [True, False])
def test_noalloc_matches_step_evolve(gpu_ctx, phys, phys_noniso, iso):
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    p = phys if iso else phys_noniso
    gpu_ctx.set_physics(p)
    for call, (seed, n) in enumerate([(21, 3000), (22, MAX_STEPS)]):
        steps = _steps(f, p, float(g["tick_time"]), seed, n)
        exp = gpu_ctx.step_evolve(steps.copy())
        rc, out = _noalloc(gpu_ctx, steps)
        assert rc == 0, f"call {call}: rc {rc}"
        assert np.max(np.abs(out["lambdaH"] - exp["lambdaH"])) < 1e-12
        assert np.max(np.abs(out["ie"] - exp["ie"]) / exp["ie"]) < 1e-12
        assert np.all(out["step_remain"] == exp["step_remain"])


def test_noalloc_vs_oracle_and_no_memory_taken(gpu_ctx, phys):
    """Isothermal steps against the restatement's closed form (1e-12, the
    bar of psg_step_evolve's own oracle test); then ten calls up to the
    buffer's size, with the device's free bytes read before and after."""
    import torch
    from oracle import Oracle
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    gpu_ctx.set_physics(phys)
    orc = Oracle(f, phys)
    steps = _steps(f, phys, float(g["tick_time"]), 31, 512)
    steps["heat"] = 0.0
    rc, out = _noalloc(gpu_ctx, steps)
    assert rc == 0
    exp = np.array([orc.solve(s["lambdaH"], s["ie"], 0.0, s["yGdepHI"], 0.0, s["time"], s["nH"], 1e4)[0]
                    for s in steps])
    assert np.max(np.abs(out["lambdaH"] - exp)) < 1e-12
    big = _steps(f, phys, float(g["tick_time"]), 32, MAX_STEPS)
    rc, _ = _noalloc(gpu_ctx, big)                 # warm-up at the full size
    assert rc == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for i in range(10):
        rc, _ = _noalloc(gpu_ctx, big[: MAX_STEPS - 997 * i])
        assert rc == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_oversize(gpu_ctx, phys):
    from psphray_b200 import api
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    gpu_ctx.set_physics(phys)
    steps = _steps(f, phys, float(g["tick_time"]), 23, MAX_STEPS + 1)
    rc, out = _noalloc(gpu_ctx, steps)
    assert rc == -1                               # PSG_E_INVAL
    assert b"exceed" in api.lib().psg_last_error(gpu_ctx.h)
    assert np.array_equal(out, steps)             # nothing touched
