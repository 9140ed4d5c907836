"""Lists longer than the shared-memory sorts hold, on the device against the
restatement (oracle/psg_oracle.c) and the emission oracle (oracle/recomb.py):

  * rays with more than 8192 hits (PSG_SORT_MAX): the per-ray merge sort in
    global memory -- ~10,000 hits (three merge passes, the result in the
    scratch half) and ~27,000 (four passes) beside empty and ordinary
    lists; hit lists bit-exact, in the batch path too;
  * particles hit by more than 32768 rays of one tick (the slot run's
    shared buffer): the run merge-sorted in global memory; hit counters and
    lasthit exact, lambdaH within 1e-9 of the sequential restatement, two
    contexts bit-identical;
  * more recombination rays than one sort tile (2048): the device-wide
    merge passes (one and two) give the oracle's (species, emitter, draw)
    order, rays bit-exact (directions to a float rounding)."""
import numpy as np
import pytest

from oracle import Oracle

pytestmark = pytest.mark.gpu


def _wide_field(n_side, sml_box, seed):
    from psphray_b200 import fields
    f = fields.uniform_field(n_side, seed)
    f.sml[:] = np.float32(sml_box * f.boxsize)
    return f


def _long_rays(f):
    """48 rays: 16 along the box diagonal through the whole box (25-30 k
    hits), 16 shorter ones from the same corner (~10 k), 8 inside (up to
    28 k), 8 outside pointing away (none)."""
    from psphray_b200 import fields
    L = f.boxsize
    rng = np.random.default_rng(3)
    R = 48
    rays = np.zeros(R, fields.RAY_DTYPE)
    d = np.ones((R, 3)) + rng.normal(0, 0.15, (R, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    rays["dir"] = d
    rays["s"] = rng.random((R, 3)) * 0.05 * L
    rays["length"] = 2 * L
    rays["length"][16:32] = 0.08 * L
    rays["Nph"] = 1e50
    rays["freq"] = 13.6 * f.units.EV * 1.5
    rays["length"][32:] = 0.02 * L
    rays["s"][32:] = rng.random((16, 3)) * L
    rays["s"][40:] = 2.5 * L
    return rays


def test_rays_longer_than_the_class_sorts(gpu_ctx, phys):
    f = _wide_field(32, 0.6, 11)
    gpu_ctx.set_physics(phys)
    gpu_ctx.load(f)
    gpu_ctx.build_tree(8)
    orc = Oracle(f, phys)
    orc.build_tree(8)
    rays = _long_rays(f)
    off, hits = gpu_ctx.trace(rays)
    o_off, o = orc.trace_all(rays)
    n = np.diff(o_off)
    assert n[:16].min() > 16384 and 8192 < n[16:32].min() and n[16:32].max() <= 16384
    assert n[40:].max() == 0
    assert np.array_equal(off, o_off)
    assert np.array_equal(hits["ipar"], o["ipar"])
    assert np.array_equal(hits["d"], o["d"]) and np.array_equal(hits["b"], o["b"])


def test_long_rays_in_ticks(phys):
    """The same rays as two ticks of 24 through the batch path (captured
    graph with the long rays' kernel): state against the restatement."""
    from psphray_b200 import api, fields
    f = _wide_field(32, 0.6, 11)
    rays = _long_rays(f)
    w = fields.make_workload("iliev32", n_side=4, nray=48)
    rays["Nph"] = w.schedule.rays_for_tick(1)["Nph"]      # the corner source's photons per ray
    tt = w.tick_time
    ctx = api.Context(0)
    try:
        ctx.set_physics(phys)
        ctx.load(f)
        ctx.build_tree(8)
        orc = Oracle(f, phys)
        orc.build_tree(8)
        st = ctx.run_ticks(rays, 24, 2, 1, tt)
        h = 0
        for t in (1, 2):
            h += orc.tick(rays[(t - 1) * 24:t * 24], t, tt)["hits"]
        assert st["hits"] == h
        s = ctx.state()
        assert np.array_equal(s["hits"], orc.hits) and np.array_equal(s["lasthit"], orc.lasthit)
        assert np.max(np.abs(s["lambdaH"] - orc.lambdaH)) < 1e-9
    finally:
        ctx.close()


def test_particles_hit_by_more_rays_than_the_slot_buffer(phys):
    from psphray_b200 import api, fields
    w = fields.make_workload("iliev32", n_side=6, nray=40000, seed=9)
    f = w.field
    f.sml[:] = np.float32(f.boxsize)
    rays = w.schedule.rays_for_tick(1)
    orc = Oracle(f, phys)
    orc.build_tree(8)
    nhit = orc.tick(rays, 1, w.tick_time)["hits"]
    assert np.sum(orc.hits > 32768) > 10
    states = []
    for _ in range(2):
        ctx = api.Context(0)
        try:
            ctx.set_physics(phys)
            ctx.load(f)
            ctx.build_tree(8)
            st = ctx.run_ticks(rays, 40000, 1, 1, w.tick_time)
            states.append(ctx.state())
        finally:
            ctx.close()
    a, b = states
    for k in ("lambdaH", "ie", "hits", "lasthit"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["hits"], orc.hits) and np.array_equal(a["lasthit"], orc.lasthit)
    assert np.max(np.abs(a["lambdaH"] - orc.lambdaH)) < 1e-9
    assert st["hits"] == nhit


@pytest.mark.parametrize("nrec", [3000, 5000])
def test_many_recombination_rays_vs_oracle(units, nrec):
    """nrec draws from a marked half of the particles at tick 2: 3000 take
    one merge pass after the tiles (the result in the scratch half), 5000
    take two."""
    import recomb
    from psphray_b200 import api, fields
    w = fields.make_workload("iliev32", n_side=16, nray=16)
    f = w.field
    phys = api.Physics(units, isothermal=True, on_the_spot=False)
    c = {k: phys.unit(k) for k in ("HI_ENERGY", "BOLTZMANN", "H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf",
                                   "hemf")}
    lte = recomb.lte_table(c["HI_ENERGY"], c["BOLTZMANN"], lambda e: phys.xs_get("HI", e))
    rng = np.random.default_rng(nrec)
    ctx = api.Context(0)
    try:
        ctx.set_physics(phys)
        ctx.load(f)
        ctx.build_tree(8)
        ctx.set_recombination(nrec=nrec, threshold=0.1, disable_lte=False, seed=77)
        yg = (rng.random(f.n) * 1e-3).astype(np.float32)
        mark = np.where(rng.random(f.n) < 0.5, 1, -1).astype(np.int32)
        lam = (0.2 + 0.8 * rng.random(f.n))
        ctx.set_state(lambdaH=lam)
        ctx.set_rec_state(yg, mark)
        s0 = ctx.state()
        src = w.schedule.rays_for_tick(2)
        st = ctx.run_ticks(src, len(src), 1, 2, w.tick_time)
        rays, ipar = ctx.rec_rays()
        pos = np.asarray(f.pos, np.float32).reshape(-1, 3)
        o_rays, o_em, _ = recomb.emit(yg, s0["lambdaH"], mark, pos, np.asarray(f.mass, np.float32), s0["ie"], 2,
                                      nrec, 77, f.boxsize, c, lte=lte)
        assert st["rec_rays"] == nrec == len(o_rays)
        assert np.array_equal(ipar, o_em)
        assert np.array_equal(rays["s"], o_rays["s"]) and np.array_equal(rays["Nph"], o_rays["Nph"])
        assert np.array_equal(rays["freq"], o_rays["freq"]) and np.array_equal(rays["length"], o_rays["length"])
        assert np.max(np.abs(rays["dir"] - o_rays["dir"])) < 1e-6
    finally:
        ctx.close()
