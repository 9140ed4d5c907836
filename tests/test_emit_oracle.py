"""The emission oracle (oracle/emit.py): its generator against the published
Philox4x32-10 known-answer vectors, and its bookkeeping against the
reference's emit_rays() semantics (src/loop.c:163-373, src/sources.c:58-78):
photons conserved per tick, lastemit, the luminosity-history cursor, the
even split of a source's photons over its rays, source frequencies
proportional to weight, isotropic unit directions, plane-source squares."""
from dataclasses import dataclass

import numpy as np
import pytest

from emit import Emitter, philox4x32_10

# Random123 kat_vectors, philox4x32 with 10 rounds: (counter, key, output)
KAT = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
       ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
       ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
        (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_philox_kat(ctr, key, out):
    got = philox4x32_10(np.array([ctr], np.uint32), key)[0]
    assert tuple(int(v) for v in got) == out


@dataclass
class Src:
    pos: tuple
    ngamma_dot: float = 0.0
    lastemit: int = 0
    type: int = 1
    specid: int = 0
    ticks: tuple | None = None
    ngamma_dots: tuple | None = None
    dir: tuple = (0.0, 0.0, 1.0)
    a: tuple = (1.0, 0.0, 0.0)
    b: tuple = (0.0, 1.0, 0.0)
    radius: float = 0.0


SPECTRA = [(np.array([1.0]), np.array([1.0])), (np.array([1.0, 2.0, 4.0]), np.array([1.0, 2.0, 1.0]))]


def test_photons_conserved_and_lastemit():
    src = [Src((0.1, 0.2, 0.3), 1e3), Src((0.5, 0.5, 0.5), 1e1), Src((0.9, 0.1, 0.4), 1e5, specid=1)]
    em = Emitter(src, SPECTRA, seed=5, boxsize=1.0)
    tick_time, R = 0.01, 64
    owed = np.zeros(3)
    for tick in range(1, 30):
        w = np.array([s.ngamma_dot for s in src]) * (tick - em.lastemit) * tick_time
        before = em.lastemit.copy()
        rays = em.rays(R, 1, tick, tick_time)
        drawn = em.lastemit == tick
        # every drawn source emits exactly its accumulated photons; the others carry theirs
        assert rays["Nph"].sum() == pytest.approx(w[drawn].sum(), rel=1e-12)
        assert np.all(em.lastemit[~drawn] == before[~drawn])
        owed = w
    assert np.all(owed >= 0)
    assert np.all(rays["length"] == 2.0)


def test_even_split_and_weighted_choice():
    src = [Src((0, 0, 0), 1.0), Src((1, 1, 1), 3.0)]
    em = Emitter(src, SPECTRA, seed=11, boxsize=2.0)
    R = 20000
    rays = em.rays(R, 1, 1, 1.0)
    from_second = rays["s"][:, 0] == 1.0
    frac = from_second.mean()
    assert abs(frac - 0.75) < 5 * np.sqrt(0.75 * 0.25 / R)
    # a source's photons split evenly over its rays
    assert np.allclose(rays["Nph"][from_second], 3.0 / from_second.sum(), rtol=1e-12)
    assert np.allclose(rays["Nph"][~from_second], 1.0 / (~from_second).sum(), rtol=1e-12)


def test_isotropic_unit_directions_and_spectrum():
    em = Emitter([Src((0, 0, 0), 1.0, specid=1)], SPECTRA, seed=3, boxsize=1.0)
    rays = em.rays(40000, 1, 7, 1.0)
    d = rays["dir"].astype(np.float64)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    assert np.all(np.abs(d.mean(axis=0)) < 0.02)
    assert np.all(np.abs((d ** 2).mean(axis=0) - 1 / 3) < 0.02)
    f = rays["freq"]
    for e, p in zip([1.0, 2.0, 4.0], [0.25, 0.5, 0.25]):
        assert abs((f == e).mean() - p) < 0.02


def test_history_cursor_and_plane_source():
    s = Src((0.5, 0.5, 0.0), type=0, ticks=(0, 10, 20), ngamma_dots=(1.0, 2.0, 4.0), radius=0.25,
            dir=(0.0, 0.0, 1.0))
    em = Emitter([s], SPECTRA, seed=1, boxsize=1.0)
    nph = []
    for tick in (5, 10, 11, 25):
        rays = em.rays(100, 1, tick, 1.0)
        nph.append(rays["Nph"].sum())
        assert np.all(np.abs(rays["s"][:, :2] - 0.5) <= 0.25)
        assert np.all(rays["dir"][:, 2] == 1.0)
    # weights use the history entry active at the tick, times the ticks since the last emission
    assert nph == pytest.approx([1.0 * 5, 2.0 * 5, 2.0 * 1, 4.0 * 14])
    assert list(em.cursor) == [2]
