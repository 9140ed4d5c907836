"""Source-ray emission pinned to the reference's own emit_rays()
(loop.c:163-195, 301-321, built from the reference sources with its
psystem_weight_srcs() and advance_cursor(), sources.c:55-78): its source
draws are made at the uniforms the library's emitter draws for each ray
(Philox stream 0, restated by oracle/emit.py), and the reference's
bookkeeping -- per-tick weights from each source's luminosity history and
the ticks since it last emitted, the source of every ray, the photon split
over the rays of a source, lastemit and the history cursor -- must come out
equal to the emission oracle's, bit for bit. The same against the device
emitter is in tests/test_gpu_emit.py. Directions and energies are drawn
from other streams and are not part of this comparison."""
import numpy as np
import pytest

from emit import Emitter, _draw, _u01
from test_emit_oracle import SPECTRA, Src

SEED = 0x1234_5678_9ABC


def point_sources(box=1.0):
    """Twelve point sources, four with luminosity histories, so that the
    cursor advances and the weights change between ticks."""
    rng = np.random.default_rng(17)
    out = []
    for i in range(12):
        pos = tuple(rng.random(3) * box)
        if i % 3 == 0:
            out.append(Src(pos, ticks=(0, 2 + i // 3, 5 + i // 3), ngamma_dots=(0.5, 3.0 + i, 0.1)))
        else:
            out.append(Src(pos, float(10 ** rng.uniform(-1, 1))))
    return out


def source_uniforms(R, tick):
    x = _draw(R, tick, 0, SEED)
    return _u01(x[:, 0], x[:, 1])


def reference_emission(reference, R, ticks, tick_time):
    from conftest import golden_field, load_golden
    reference.load(golden_field(load_golden("uniform16.npz")))      # (the epoch and box of emit_rays())
    reference.set_sources(point_sources())
    out = []
    for t in ticks:
        isrc, nph = reference.emit_source_rays(R, t, tick_time, source_uniforms(R, t),
                                               freq=13.6 * reference.units.EV)
        out.append((isrc, nph))
    return out, reference.sources_state()


def by_source(src_of_ray, nph):
    o = np.lexsort((nph, src_of_ray))
    return src_of_ray[o], nph[o]


def test_emission_matches_reference(reference):
    R, tick_time = 400, 0.01
    ticks = list(range(1, 9))
    ref, (r_last, r_cur) = reference_emission(reference, R, ticks, tick_time)
    srcs = point_sources()
    em = Emitter(srcs, SPECTRA, seed=SEED, boxsize=1.0)
    pos = np.array([s.pos for s in srcs], np.float32)
    for t, (isrc, nph) in zip(ticks, ref):
        rays = em.rays(R, 1, t, tick_time)
        # the oracle's source of each ray, from the ray's start point
        which = np.array([int(np.nonzero((pos == s).all(1))[0][0]) for s in rays["s"]])
        a_src, a_nph = by_source(which, rays["Nph"])
        b_src, b_nph = by_source(isrc, nph)
        assert np.array_equal(a_src, b_src), t
        assert np.array_equal(a_nph, b_nph), t
    assert np.array_equal(em.lastemit, r_last)
    assert np.array_equal(em.cursor.astype(np.int64), r_cur)
    assert len(set(r_cur)) > 1 and len(set(r_last)) >= 1
