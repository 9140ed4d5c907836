"""The batch machinery around the kernels: a batch after its traversal is
replayed from a captured CUDA graph (sizes fixed by the batch's shape,
counts read on the device); the same batch issued launch by launch (per-
launch timing on) must give the identical state; a batch waits for the
device twice; and the autotuner chooses launch shapes without changing the
run's state or its results."""
import numpy as np
import pytest

from conftest import golden_field, load_golden

pytestmark = pytest.mark.gpu


def _ctx(phys, field):
    from psphray_b200 import api
    ctx = api.Context(0)
    ctx.set_physics(phys)
    ctx.load(field)
    ctx.build_tree(8)
    return ctx


def _batches(ctx, w, nb, K, t0=1):
    R = w.schedule.nray
    out = []
    for b in range(nb):
        first = t0 + b * K
        rays = np.concatenate([w.schedule.rays_for_tick(first + i) for i in range(K)])
        out.append(ctx.run_ticks(rays, R, K, first, w.tick_time))
    return out


@pytest.mark.parametrize("iso", [True, False])
def test_graph_replay_equals_launch_by_launch(phys, phys_noniso, iso):
    """Six batches of 4 ticks (the second and later replay the captured
    graph) against the same batches issued one launch at a time."""
    from psphray_b200 import fields
    p = phys if iso else phys_noniso
    wa = fields.make_workload("iliev32", n_side=24, nray=96, seed=5)
    wb = fields.make_workload("iliev32", n_side=24, nray=96, seed=5)
    a, b = _ctx(p, wa.field), _ctx(p, wb.field)
    try:
        b.set_timing(True)
        sa = _batches(a, wa, 6, 4)
        sb = _batches(b, wb, 6, 4)
        ga, gb = a.state(), b.state()
    finally:
        a.close()
        b.close()
    for k in ("lambdaH", "ie", "hits", "lasthit"):
        assert np.array_equal(ga[k], gb[k]), k
    assert [s["hits"] for s in sa] == [s["hits"] for s in sb]
    assert [s["active"] for s in sa] == [s["active"] for s in sb]
    assert all(s["host_syncs"] == 2 for s in sa), [s["host_syncs"] for s in sa]
    assert (ga["lasthit"] > 0).sum() > 1000


def test_batch_after_hits_grow(phys):
    """Batches whose hit counts grow past the buffers' capacity: the buffers
    grow (a new graph is captured) and the ticks still match the oracle."""
    from oracle import Oracle
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    ctx = _ctx(phys, f)
    orc = Oracle(f, phys)
    orc.build_tree(8)
    rays = g["rays"]
    R = int(g["nray"])
    try:
        t = 1
        for K in (1, 2, 4, 8):          # more ticks per batch: more hits each time
            ctx.run_ticks(rays[(t - 1) * R:(t - 1 + K) * R], R, K, t, float(g["tick_time"]))
            for k in range(K):
                orc.tick(rays[(t - 1 + k) * R:(t + k) * R], t + k, float(g["tick_time"]))
            t += K
        s = ctx.state()
    finally:
        ctx.close()
    assert np.array_equal(s["lasthit"], orc.lasthit)
    assert np.array_equal(s["hits"], orc.hits)
    assert np.max(np.abs(s["lambdaH"] - orc.lambdaH)) < 1e-9


def test_autotune_keeps_state_and_results(phys_noniso):
    """psg_autotune on a batch of the 32^3 field, not isothermal: the
    particle state is unchanged by the call; a batch run with the chosen
    shapes matches the default shapes' batch (the deposit groups only
    reassociate the FP64 scan, which can move an adaptive step decision: the
    integrator's tolerance, 1e-6 in x_HI; counters exact); the choice is
    cached for new contexts on the device; leaf sizes other than the
    reference's 8 are refused."""
    import torch
    from psphray_b200 import api, fields
    w = fields.make_workload("iliev32", n_side=32, nray=256, seed=9)
    w2 = fields.make_workload("iliev32", n_side=32, nray=256, seed=9)
    K = 4
    rays = np.concatenate([w.schedule.rays_for_tick(1 + i) for i in range(K)])
    a, b = _ctx(phys_noniso, w.field), _ctx(phys_noniso, w2.field)
    try:
        with pytest.raises(api.PsgError):
            a.set_tune(leaf_size=16)
        before = a.state()
        d = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
        torch.cuda.synchronize()
        best, ms = a.autotune(d.data_ptr(), 256, K, 1, w.tick_time, reps=1)
        after = a.state()
        for k in ("lambdaH", "ie", "hits", "lasthit"):
            assert np.array_equal(before[k], after[k]), k
        assert ms > 0 and best["leaf_size"] == 8
        assert a.tune() == best
        b.set_tune(trace_warps=4, deposit_long=96, deposit_mid=384, update_minblocks=1)
        a.run_ticks(rays, 256, K, 1, w.tick_time)
        b.run_ticks(rays, 256, K, 1, w.tick_time)
        sa, sb = a.state(), b.state()
        c = api.Context(0)
        try:
            assert c.tune() == best
        finally:
            c.close()
    finally:
        a.close()
        b.close()
    assert np.array_equal(sa["lasthit"], sb["lasthit"]) and np.array_equal(sa["hits"], sb["hits"])
    assert np.max(np.abs(sa["lambdaH"] - sb["lambdaH"])) <= 1e-6
    assert np.max(np.abs(sa["ie"] - sb["ie"]) / sb["ie"]) <= 1e-4


@pytest.mark.parametrize("iso", [True, False])
def test_recombination_graph_equals_one_by_one(units, iso):
    """Not on the spot (nrec recombination rays per tick emitted on the
    device): from the second call on, a call's ticks replay one captured
    tick with no host read between them (two waits per call: the traversal
    of the call's source rays, traced together before the ticks, and the
    counters at the end); the same calls
    issued launch by launch, tick by tick (per-launch timing on), must give
    the identical state, counters and emitted rays."""
    from psphray_b200 import api, fields
    p = api.Physics(units, isothermal=iso, on_the_spot=False)
    wa = fields.make_workload("iliev32", n_side=20, nray=64, seed=3)
    wb = fields.make_workload("iliev32", n_side=20, nray=64, seed=3)
    a, b = _ctx(p, wa.field), _ctx(p, wb.field)
    try:
        for c in (a, b):
            c.set_recombination(nrec=40, seed=11)
        b.set_timing(True)
        sa = _batches(a, wa, 5, 4)
        sb = _batches(b, wb, 5, 4)
        ga, gb = a.state(), b.state()
        ra, rb = a.rec_state(), b.rec_state()
        rays_a, rays_b = a.rec_rays(), b.rec_rays()
    finally:
        a.close()
        b.close()
    for k in ("lambdaH", "ie", "hits", "lasthit"):
        assert np.array_equal(ga[k], gb[k]), k
    for x, y in zip(ra, rb):
        assert np.array_equal(x, y)
    assert np.array_equal(rays_a[0].view(np.uint8), rays_b[0].view(np.uint8))
    assert np.array_equal(rays_a[1], rays_b[1])
    for k in ("hits", "active", "rec_rays", "saturated"):
        assert [s[k] for s in sa] == [s[k] for s in sb], k
    assert [s["rec_photons"] for s in sa] == pytest.approx([s["rec_photons"] for s in sb], rel=1e-12)
    assert all(s["host_syncs"] == 2 for s in sa[1:]), [s["host_syncs"] for s in sa]
    assert sa[-1]["rec_rays"] == 4 * 40
