"""The CUDA path (libpsg.so through its C ABI) against the C restatement and
the golden fixtures. Bit-exact for the tree and hit lists; FP64 tolerances
stated per test for deposit and update."""
import numpy as np
import pytest

from conftest import golden_field, leaf_sets_from_gpu, leaf_sets_from_oracle, load_golden
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _gpu(ctx, field, phys, flag=None, ppc=8):
    ctx.set_physics(phys)
    ctx.load(field, flag=flag)
    ctx.build_tree(ppc)
    return ctx


def test_loaded_code_is_sm100a(gpu_ctx):
    """The runtime loaded SASS built for sm_100a (binaryVersion 100), not a
    JIT translation of PTX for another architecture."""
    import ctypes as C
    from psphray_b200 import api
    b, p = C.c_int(0), C.c_int(0)
    assert api.lib().psg_device_arch(gpu_ctx.h, C.byref(b), C.byref(p)) == 0
    assert b.value == 100 and p.value == 100, (b.value, p.value)


@pytest.mark.parametrize("name", ["uniform16.npz", "lognormal16.npz", "edges.npz"])
def test_tree_golden(gpu_ctx, phys, name):
    g = load_golden(name)
    f = golden_field(g)
    _gpu(gpu_ctx, f, phys, flag=g.get("flag"))
    leaf_of, keys, lbox, ebox = leaf_sets_from_gpu(gpu_ctx.tree(), f.n)
    assert np.array_equal(leaf_of, g["leaf_of"])
    assert np.array_equal(keys, g["leaf_keys"])
    assert np.array_equal(lbox, g["leaf_box"])
    assert np.array_equal(ebox, g["empty_box"])


@pytest.mark.parametrize("kind,n_side,ppc", [("iliev32", 32, 8), ("lognormal128", 32, 8),
                                             ("iliev32", 24, 1), ("lognormal128", 24, 3)])
def test_tree_vs_oracle(gpu_ctx, phys, kind, n_side, ppc):
    from psphray_b200 import fields
    f = fields.make_workload(kind, n_side=n_side, nray=8, seed=11).field
    _gpu(gpu_ctx, f, phys, ppc=ppc)
    orc = Oracle(f, phys)
    orc.build_tree(ppc)
    ot = orc.tree_cells()
    gt = gpu_ctx.tree()
    assert gt["ncells"] == len(ot["head"])
    for a, b in zip(leaf_sets_from_gpu(gt, f.n), leaf_sets_from_oracle(ot, f.n)):
        assert np.array_equal(a, b)


def _check_hits(off, hits, g_off, g_ipar, g_d, g_b):
    assert np.array_equal(off, g_off)
    assert np.array_equal(hits["ipar"], g_ipar)
    assert np.array_equal(hits["d"], g_d)
    assert np.array_equal(hits["b"], g_b)


def test_trace_golden_uniform(gpu_ctx, phys):
    g = load_golden("uniform16.npz")
    _gpu(gpu_ctx, golden_field(g), phys)
    R = int(g["nray"])
    for t in (1, 2, 3):
        off, hits = gpu_ctx.trace(g["rays"][(t - 1) * R:t * R])
        _check_hits(off, hits, g[f"t{t}_off"], g[f"t{t}_ipar"], g[f"t{t}_d"], g[f"t{t}_b"])


@pytest.mark.parametrize("name", ["lognormal16.npz", "edges.npz"])
def test_trace_golden(gpu_ctx, phys, name):
    g = load_golden(name)
    _gpu(gpu_ctx, golden_field(g), phys, flag=g.get("flag"))
    off, hits = gpu_ctx.trace(g["rays"])
    _check_hits(off, hits, g["off"], g["ipar"], g["d"], g["b"])


def test_rt_trace_shim(gpu_ctx, phys):
    """psg_rt_trace(), rt_trace()'s signature: one ray, same list."""
    g = load_golden("edges.npz")
    _gpu(gpu_ctx, golden_field(g), phys, flag=g["flag"])
    for i in (0, 7, 14, len(g["rays"]) - 1):
        r = g["rays"][i]
        x = gpu_ctx.rt_trace(r["s"], r["dir"], np.float32(r["length"]))
        sl = slice(g["off"][i], g["off"][i + 1])
        assert np.array_equal(x["ipar"], g["ipar"][sl])
        assert np.array_equal(x["d"], g["d"][sl])


@pytest.mark.parametrize("kind,n_side,nray", [("iliev32", 32, 256), ("lognormal128", 32, 256)])
def test_trace_vs_oracle(gpu_ctx, phys, kind, n_side, nray):
    from psphray_b200 import fields
    w = fields.make_workload(kind, n_side=n_side, nray=nray, seed=5)
    _gpu(gpu_ctx, w.field, phys)
    orc = Oracle(w.field, phys)
    orc.build_tree(8)
    rays = w.schedule.rays_for_ticks(1, 3)
    off, hits = gpu_ctx.trace(rays)
    o_off, o = orc.trace_all(rays)
    assert off[-1] > 0
    _check_hits(off, hits, o_off, o["ipar"], o["d"], o["b"])


def test_ticks_vs_oracle(gpu_ctx, phys):
    """40 ticks in batches of 8 and 1: lasthit and per-particle hit counters
    exact; lambdaH within 1e-9 of the sequential FP64 restatement (the GPU
    sums optical depth with a warp scan and transmits with exp(-sum))."""
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    _gpu(gpu_ctx, f, phys)
    orc = Oracle(f, phys)
    orc.build_tree(8)
    R = int(g["nray"])
    tt = float(g["tick_time"])
    t = 1
    for batch in (8, 8, 1, 8, 7, 8):
        rays = g["rays"][(t - 1) * R:(t - 1 + batch) * R]
        st = gpu_ctx.run_ticks(rays, R, batch, t, tt)
        exp_hits = 0
        for k in range(batch):
            s = orc.tick(rays[k * R:(k + 1) * R], t + k, tt)
            exp_hits += s["hits"]
        assert st["hits"] == exp_hits
        t += batch
        gs = gpu_ctx.state()
        assert np.array_equal(gs["lasthit"], orc.lasthit)
        assert np.array_equal(gs["hits"], orc.hits)
        assert np.max(np.abs(gs["lambdaH"] - orc.lambdaH)) < 1e-9
        assert np.max(np.abs(gs["ie"] - orc.ie) / orc.ie) < 1e-6
    assert t == 41


def test_ticks_vs_reference_golden(gpu_ctx, phys):
    """Against the reference's own LSODA run: x_HII within 1e-3 after 40
    ticks, lasthit exact."""
    g = load_golden("uniform16.npz")
    _gpu(gpu_ctx, golden_field(g), phys)
    R = int(g["nray"])
    gpu_ctx.run_ticks(g["rays"], R, 40, 1, float(g["tick_time"]))
    gs = gpu_ctx.state()
    assert np.array_equal(gs["lasthit"], g["st_lasthit"][-1])
    assert np.max(np.abs(gs["lambdaH"] - g["st_lambdaH"][-1])) < 1e-3


def test_step_evolve_vs_oracle(gpu_ctx, phys):
    from psphray_b200.api import STEP_DTYPE
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    gpu_ctx.set_physics(phys)
    orc = Oracle(f, phys)
    rng = np.random.default_rng(9)
    n = 512
    steps = np.zeros(n, STEP_DTYPE)
    steps["lambdaH"] = 10 ** rng.uniform(-8, 0, n)
    steps["ie"] = float(f.ie[0])
    steps["yGdepHI"] = np.where(rng.random(n) < 0.7, 10 ** rng.uniform(-5, 1, n), 0.0)
    steps["time"] = float(g["tick_time"]) * rng.integers(1, 5000, n)
    steps["nH"] = float(f.rho[0]) * phys.unit("H_PER_MASS")
    steps["T"] = 1e4
    out = gpu_ctx.step_evolve(steps.copy())
    exp = np.array([orc.solve(s["lambdaH"], s["ie"], 0.0, s["yGdepHI"], 0.0, s["time"], s["nH"], 1e4)[0]
                    for s in steps])
    assert np.max(np.abs(out["lambdaH"] - exp)) < 1e-12
    assert np.all(out["step_remain"] == 0.0)


def test_step_evolve_noniso_vs_oracle(gpu_ctx, phys_noniso):
    """Not isothermal: lambdaH and ie integrated together; GPU (rtol 1e-6;
    the reference's LSODA runs at 1e-4) against the restatement (rtol 1e-10)."""
    from psphray_b200.api import STEP_DTYPE
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    gpu_ctx.set_physics(phys_noniso)
    orc = Oracle(f, phys_noniso, isothermal=False)
    rng = np.random.default_rng(10)
    n = 128
    steps = np.zeros(n, STEP_DTYPE)
    steps["lambdaH"] = 10 ** rng.uniform(-6, 0, n)
    steps["ie"] = float(f.ie[0]) * 10 ** rng.uniform(-0.5, 0.5, n)
    steps["yGdepHI"] = np.where(rng.random(n) < 0.7, 10 ** rng.uniform(-4, 0, n), 0.0)
    steps["heat"] = steps["yGdepHI"] * 1e-3 * float(f.ie[0])
    steps["time"] = float(g["tick_time"]) * rng.integers(1, 200, n)
    steps["nH"] = float(f.rho[0]) * phys_noniso.unit("H_PER_MASS")
    steps["T"] = 1e4
    out = gpu_ctx.step_evolve(steps.copy())
    for s, o in zip(steps, out):
        lam, ie, rc = orc.solve(s["lambdaH"], s["ie"], 0.0, s["yGdepHI"], s["heat"], s["time"], s["nH"], s["T"])
        assert rc == 0
        assert abs(o["lambdaH"] - lam) < 1e-5
        # rate tables are linear in log T, so the right-hand side is only
        # continuous: the integrations agree to ~1e-5, not to rtol
        assert abs(o["ie"] - ie) / ie < 1e-4


def test_errors_are_reported_not_trapped(gpu_ctx, phys):
    """Call-order and device-status errors come back as codes."""
    from psphray_b200 import api
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    fresh = api.Context(0)
    with pytest.raises(api.PsgError) as e:
        fresh.run_ticks(g["rays"][:16], 16, 1, 1, 1.0)
    assert e.value.code == -1
    fresh.close()
    bad = golden_field(g)
    bad.rho = bad.rho.copy()
    bad.rho[:] = np.nan                      # nH = NaN: the solver flags a non-finite state
    _gpu(gpu_ctx, bad, phys)
    with pytest.raises(api.PsgError) as e:
        gpu_ctx.run_ticks(g["rays"][:16], 16, 1, 1, float(g["tick_time"]))
    assert e.value.code == -6
    # the context stays usable
    _gpu(gpu_ctx, f, phys)
    gpu_ctx.run_ticks(g["rays"][:16], 16, 1, 1, float(g["tick_time"]))


def test_capped_deposits_vs_oracle(gpu_ctx, phys):
    """Rays carrying 1e3x the photons saturate particles (the cap of
    loop.c:482-485) and end early on the 1e-10 cut: both settled exactly
    as the sequential restatement settles them."""
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    _gpu(gpu_ctx, f, phys)
    orc = Oracle(f, phys)
    orc.build_tree(8)
    R = int(g["nray"])
    rays = g["rays"][:4 * R].copy()
    rays["Nph"] *= 1e3
    st = gpu_ctx.run_ticks(rays, R, 4, 1, float(g["tick_time"]))
    sat = 0
    for k in range(4):
        sat += orc.tick(rays[k * R:(k + 1) * R], k + 1, float(g["tick_time"]))["saturated"]
    assert sat > 0 and st["saturated"] == sat
    gs = gpu_ctx.state()
    assert np.array_equal(gs["hits"], orc.hits)
    assert np.max(np.abs(gs["lambdaH"] - orc.lambdaH)) < 1e-9


@pytest.mark.parametrize("boost", [1e6, 1e9])
def test_capped_runs_vs_oracle(gpu_ctx, phys, boost):
    """Rays from the corner source of the 32^3 uniform field (in-box rays of
    ~480 hits: the whole-block and quarter-block deposit groups) carrying
    1e6x and 1e9x the photons: runs of capped hits mixed with uncapped ones,
    against the sequential restatement: saturation count, per-particle
    deposit counters exact, lambda to 1e-9. The ticks run as two batches:
    the first (just after the load) settles capped hits one at a time and
    caps most of its hits, so the second settles them with the affine-map
    scan -- both forms of the deposit against the same restatement."""
    from psphray_b200 import fields
    w = fields.make_workload("iliev32", nray=128, seed=5)
    f = w.field
    _gpu(gpu_ctx, f, phys)
    orc = Oracle(f, phys)
    orc.build_tree(8)
    R = 128
    rays = w.schedule.rays_for_ticks(1, 2)
    rays["Nph"] *= boost
    st = gpu_ctx.run_ticks(rays[:R], R, 1, 1, w.tick_time)
    st2 = gpu_ctx.run_ticks(rays[R:], R, 1, 2, w.tick_time)
    assert st["saturated"] > 1e-3 * st["hits"]
    st["saturated"] += st2["saturated"]
    sat = 0
    for k in range(2):
        sat += orc.tick(rays[k * R:(k + 1) * R], k + 1, w.tick_time)["saturated"]
    assert sat > 1000 and st["saturated"] == sat
    gs = gpu_ctx.state()
    assert np.array_equal(gs["hits"], orc.hits)
    assert np.array_equal(gs["lasthit"], orc.lasthit)
    assert np.max(np.abs(gs["lambdaH"] - orc.lambdaH)) < 1e-9


def test_ticks_noniso_vs_oracle(gpu_ctx, phys_noniso):
    """Not isothermal, 8-bin blackbody rays (photo-heating on): 6 ticks on
    the log-normal field through the work-queue integrator against the
    restatement's tight integration; counters exact, state to the
    integrator's tolerance."""
    from psphray_b200 import fields
    w = fields.make_workload("lognormal128", n_side=16, nray=64, seed=21)
    f = w.field
    _gpu(gpu_ctx, f, phys_noniso)
    orc = Oracle(f, phys_noniso, isothermal=False)
    orc.build_tree(8)
    rays = w.schedule.rays_for_ticks(1, 6)
    assert np.any(rays["freq"] > 13.7 * f.units.EV)
    gpu_ctx.run_ticks(rays[:3 * 64], 64, 3, 1, w.tick_time)
    gpu_ctx.run_ticks(rays[3 * 64:], 64, 3, 4, w.tick_time)
    for k in range(6):
        assert orc.tick(rays[k * 64:(k + 1) * 64], k + 1, w.tick_time)["rc"] == 0
    gs = gpu_ctx.state()
    assert np.array_equal(gs["lasthit"], orc.lasthit)
    assert np.array_equal(gs["hits"], orc.hits)
    assert np.max(np.abs(gs["lambdaH"] - orc.lambdaH)) < 1e-4
    assert np.max(np.abs(gs["ie"] - orc.ie) / orc.ie) < 1e-4
    assert np.max(np.abs(gs["ie"] - f.ie) / f.ie) > 1e-3     # the gas did heat or cool
