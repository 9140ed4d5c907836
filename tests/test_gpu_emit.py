"""Device ray emission (psg_set_sources / psg_emit_rays / psg_run_ticks_emit)
against the emission oracle: the same source per ray, photons, energies and
source state bit for bit; directions to the float rounding of cos/sin; and
the ticks run on emitted rays identical to the ticks run on the same rays
passed in from the host."""
import numpy as np
import pytest

from conftest import golden_field, load_golden
from emit import Emitter
from test_emit_oracle import SPECTRA, Src

pytestmark = pytest.mark.gpu


def _sources(box):
    rng = np.random.default_rng(4)
    src = [Src(tuple(rng.random(3) * box), float(10 ** rng.uniform(-1, 1)), specid=int(i % 2))
           for i in range(12)]
    src.append(Src((0.5 * box, 0.5 * box, 0.0), type=0, ticks=(0, 3, 6), ngamma_dots=(0.5, 2.0, 1.0),
                   radius=0.2 * box, dir=(0.0, 0.0, 1.0), specid=1))
    return src


def _compare(dev, ref):
    assert np.array_equal(dev["Nph"], ref["Nph"])
    assert np.array_equal(dev["freq"], ref["freq"])
    assert np.array_equal(dev["length"], ref["length"])
    assert np.array_equal(dev["s"], ref["s"])
    # cos/sin of the device and of the host libm may differ in the last bit
    # of the double; after rounding to float at most one float ulp
    assert np.max(np.abs(dev["dir"] - ref["dir"])) <= 1.2e-7


def test_emit_vs_oracle(gpu_ctx, phys):
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    gpu_ctx.set_physics(phys)
    gpu_ctx.load(f)
    src = _sources(f.boxsize)
    gpu_ctx.set_sources(src, SPECTRA, seed=0x1234_5678_9ABC)
    em = Emitter(_sources(f.boxsize), SPECTRA, seed=0x1234_5678_9ABC, boxsize=f.boxsize)
    tick_time = float(g["tick_time"])
    for first, K, R in [(1, 3, 1000), (4, 5, 257)]:          # two calls in a row continue the state
        dev = gpu_ctx.emit_rays(R, K, first, tick_time)
        ref = em.rays(R, K, first, tick_time)
        _compare(dev, ref)
        lastemit, cursor = gpu_ctx.sources_state()
        assert np.array_equal(lastemit, em.lastemit)
        assert np.array_equal(cursor, em.cursor)


def test_run_ticks_emit_equals_host_rays(gpu_ctx, phys):
    """Emission + ticks on the device = the same rays emitted, then passed in."""
    from psphray_b200 import api
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    tick_time = float(g["tick_time"])
    src = [Src((0.0, 0.0, 0.0), 5e-2 * 1e50 / phys.units.SEC)]
    spec = [(np.array([13.6 * phys.units.EV]), np.array([1.0]))]
    a = api.Context(0)
    try:
        for ctx in (gpu_ctx, a):
            ctx.set_physics(phys)
            ctx.load(f)
            ctx.build_tree(8)
            ctx.set_sources(src, spec, seed=99)
        st_dev = gpu_ctx.run_ticks_emit(64, 6, 1, tick_time)
        rays = a.emit_rays(64, 6, 1, tick_time)
        st_host = a.run_ticks(rays, 64, 6, 1, tick_time)
        assert st_dev["hits"] == st_host["hits"] > 0
        s1, s2 = gpu_ctx.state(), a.state()
        for k in ("lambdaH", "ie", "hits", "lasthit"):
            assert np.array_equal(s1[k], s2[k]), k
    finally:
        a.close()


def test_emit_errors(gpu_ctx, phys):
    from psphray_b200 import api
    fresh = api.Context(0)
    try:
        with pytest.raises(api.PsgError):
            fresh.emit_rays(16, 1, 1, 1.0)                  # no sources
        with pytest.raises(api.PsgError):
            fresh.set_sources([Src((0, 0, 0), 1.0, specid=5)], SPECTRA, seed=1)   # bad spectrum id
    finally:
        fresh.close()


def test_emit_vs_reference_emit_rays(gpu_ctx, phys, reference):
    """The device emitter against the reference's own emit_rays() with its
    source draws made at the device's uniforms (tests/test_emit_reference.py
    has the harness): per tick, the source of every ray and its photons
    (the reference's weights from the luminosity histories and lastemit,
    split evenly over a source's rays), and after the ticks each source's
    lastemit and history cursor, bit for bit."""
    from test_emit_reference import SEED, by_source, point_sources, reference_emission
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    gpu_ctx.set_physics(phys)
    gpu_ctx.load(f)
    R, tick_time, ticks = 400, 0.01, list(range(1, 9))
    ref, (r_last, r_cur) = reference_emission(reference, R, ticks, tick_time)
    srcs = point_sources()
    gpu_ctx.set_sources(srcs, [(np.array([13.6 * phys.units.EV]), np.array([1.0]))], seed=SEED)
    pos = np.array([s.pos for s in srcs], np.float32)
    for t, (isrc, nph) in zip(ticks, ref):
        rays = gpu_ctx.emit_rays(R, 1, t, tick_time)
        which = np.array([int(np.nonzero((pos == s).all(1))[0][0]) for s in rays["s"]])
        a_src, a_nph = by_source(which, rays["Nph"])
        b_src, b_nph = by_source(isrc, nph)
        assert np.array_equal(a_src, b_src), t
        assert np.array_equal(a_nph, b_nph), t
    lastemit, cursor = gpu_ctx.sources_state()
    assert np.array_equal(lastemit, r_last)
    assert np.array_equal(cursor.astype(np.int64), r_cur)
