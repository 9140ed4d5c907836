"""Seeded synthetic SPH fields and host-generated rays for the hot path.

The reference reads gas snapshots (massiveblack / psphray formats) and emits
rays from sources (src/loop.c:163-373). For throughput and parity work the
inputs are generated here with fixed seeds, with the shapes of the workloads
the hot path is measured on:

* ``uniform_field`` -- equal-mass hydrogen particles at uniform-random
  positions in a vacuum-boundary cube (the Iliev-test-1 style set-up);
* ``lognormal_field`` -- particles placed by mass on a log-normal density
  field built from a Gaussian random field with P(k) ~ k^-2.

Smoothing lengths are the distance to the 32nd nearest neighbour (the
cubic-spline support radius ``h`` used by src/sph-depth.c:10-23).

``RaySchedule`` reproduces the per-tick photon bookkeeping of emit_rays():
sources are drawn by accumulated-photon weight (loop.c:172-195,
sources.c:67-78), every source's photons since its last emission are split
evenly over the rays drawn for it (loop.c:305-321), directions are isotropic
and the ray length is twice the box (loop.c:267). Random numbers come from a
counter-based generator (numpy Philox) keyed on (seed, tick), so any tick's
rays can be regenerated independently and identically on every host.
"""
from __future__ import annotations

from dataclasses import dataclass, field as dfield

import numpy as np

from .units import Units

RAY_DTYPE = np.dtype([("s", "<f4", 3), ("dir", "<f4", 3), ("Nph", "<f8"),
                      ("freq", "<f8"), ("length", "<f8")])


@dataclass
class Field:
    """Particle arrays in the reference's storage types (psystem.h:32-78)."""
    pos: np.ndarray      # float32 [N,3]
    mass: np.ndarray     # float32 [N]
    sml: np.ndarray      # float32 [N]
    rho: np.ndarray      # float32 [N]
    ie: np.ndarray       # float32 [N]
    xHI: np.ndarray      # float32 [N]
    ye: np.ndarray       # float32 [N]
    boxsize: float
    units: Units

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def _smoothing_lengths(pos: np.ndarray, nngb: int, chunk: int = 1 << 20) -> np.ndarray:
    """Distance to the nngb-th neighbour; queried in chunks of points so that
    16.8 M particles need ~0.5 GB of neighbour lists at a time, not ~9 GB."""
    from scipy.spatial import cKDTree
    p64 = pos.astype(np.float64)
    tree = cKDTree(p64)
    sml = np.empty(len(pos), dtype=np.float32)
    for i in range(0, len(pos), chunk):
        d, _ = tree.query(p64[i:i + chunk], k=nngb + 1, workers=-1)
        sml[i:i + chunk] = d[:, nngb]
    return sml


def _finish(pos, units: Units, boxsize: float, nH_mean_cgs: float, T: float,
            xHII0: float, rho_rel: np.ndarray | None, nngb: int) -> Field:
    n = pos.shape[0]
    vol_cm3 = (boxsize / units.CM) ** 3
    n_h_total = nH_mean_cgs * vol_cm3
    mass_p = n_h_total / n / units.H_PER_MASS
    mass = np.full(n, mass_p, dtype=np.float32)
    sml = _smoothing_lengths(pos, nngb)
    rho_mean = mass_p * n / boxsize ** 3
    if rho_rel is None:
        rho = np.full(n, rho_mean, dtype=np.float32)
    else:
        rho = (rho_mean * rho_rel).astype(np.float32)
    ye = np.full(n, xHII0, dtype=np.float32)
    xHI = np.full(n, 1.0 - xHII0, dtype=np.float32)
    ie = np.array([units.Tye2ie(T, float(y)) for y in ye[:1]], dtype=np.float32)
    ie = np.full(n, ie[0], dtype=np.float32)
    return Field(pos=pos.astype(np.float32), mass=mass, sml=sml, rho=rho, ie=ie,
                 xHI=xHI, ye=ye, boxsize=float(boxsize), units=units)


def uniform_field(n_side: int, seed: int, box_kpc: float = 6.6, nH: float = 1e-3,
                  T: float = 1e4, xHII0: float = 1.2e-3, nngb: int = 32,
                  units: Units | None = None) -> Field:
    """n_side**3 particles at seeded uniform-random positions in [0, L)^3."""
    units = units or Units(hmf=1.0)
    boxsize = box_kpc * units.KPC
    rng = np.random.Generator(np.random.Philox(key=seed))
    n = n_side ** 3
    pos = (rng.random((n, 3)) * boxsize).astype(np.float32)
    pos = np.minimum(pos, np.nextafter(np.float32(boxsize), np.float32(0)))
    return _finish(pos, units, boxsize, nH, T, xHII0, None, nngb)


def lognormal_field(n_side: int, seed: int, sigma: float = 1.0, box_kpc: float = 6.6,
                    nH: float = 1e-3, T: float = 1e4, xHII0: float = 1.2e-3,
                    nngb: int = 32, units: Units | None = None) -> Field:
    """Particles placed by mass on exp(sigma*g) with g a unit-variance Gaussian
    random field of spectrum P(k) ~ k^-2 on an n_side^3 grid."""
    units = units or Units(hmf=1.0)
    boxsize = box_kpc * units.KPC
    rng = np.random.Generator(np.random.Philox(key=seed))
    g = n_side
    kx = np.fft.fftfreq(g) * g
    kz = np.fft.rfftfreq(g) * g
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    amp = np.sqrt(1.0 / k2)          # sqrt(P(k)) with P ~ k^-2
    amp[0, 0, 0] = 0.0
    noise = np.fft.rfftn(rng.standard_normal((g, g, g)))
    gauss = np.fft.irfftn(noise * amp, s=(g, g, g), axes=(0, 1, 2))
    gauss = (gauss - gauss.mean()) / gauss.std()
    dens = np.exp(sigma * gauss - 0.5 * sigma * sigma)
    dens /= dens.mean()
    n = n_side ** 3
    prob = dens.ravel() / dens.sum()
    cells = rng.choice(prob.size, size=n, p=prob)
    ci = np.stack(np.unravel_index(cells, (g, g, g)), axis=1).astype(np.float64)
    pos = (ci + rng.random((n, 3))) * (boxsize / g)
    pos = np.minimum(pos.astype(np.float32), np.nextafter(np.float32(boxsize), np.float32(0)))
    rho_rel = dens.ravel()[cells]
    return _finish(pos, units, boxsize, nH, T, xHII0, rho_rel, nngb)


@dataclass
class Source:
    pos: tuple
    ngamma_dot: float       # photons per internal time unit (sources.c:172)
    lastemit: int = 0


@dataclass
class RaySchedule:
    """Host-side ray producer with emit_rays() bookkeeping (loop.c:163-373)."""
    sources: list
    nray: int
    tick_time: float
    boxsize: float
    seed: int
    energies: np.ndarray = dfield(default_factory=lambda: np.zeros(0))  # spectrum bins
    eweights: np.ndarray = dfield(default_factory=lambda: np.zeros(0))  # photon weights

    def rays_for_tick(self, tick: int) -> np.ndarray:
        rng = np.random.Generator(np.random.Philox(key=self.seed, counter=[tick, 0, 0, 0]))
        ns = len(self.sources)
        w = np.array([s.ngamma_dot * (tick - s.lastemit) * self.tick_time for s in self.sources])
        if ns == 1:
            isrc = np.zeros(self.nray, dtype=np.int64)
        else:
            isrc = np.sort(rng.choice(ns, size=self.nray, p=w / w.sum()))
        counts = np.bincount(isrc, minlength=ns)
        out = np.zeros(self.nray, dtype=RAY_DTYPE)
        u = rng.random(self.nray) * 2.0 - 1.0
        phi = rng.random(self.nray) * (2.0 * np.pi)
        st = np.sqrt(np.maximum(0.0, 1.0 - u * u))
        out["dir"][:, 0] = st * np.cos(phi)
        out["dir"][:, 1] = st * np.sin(phi)
        out["dir"][:, 2] = u
        srcpos = np.array([s.pos for s in self.sources], dtype=np.float64)
        out["s"] = srcpos[isrc]
        out["Nph"] = w[isrc] / counts[isrc]
        if len(self.energies) == 1:
            out["freq"] = self.energies[0]
        else:
            p = self.eweights / self.eweights.sum()
            out["freq"] = self.energies[rng.choice(len(self.energies), size=self.nray, p=p)]
        out["length"] = self.boxsize * 2
        for i in np.unique(isrc):
            self.sources[i].lastemit = tick
        return out

    def rays_for_ticks(self, tick0: int, nticks: int) -> np.ndarray:
        return np.concatenate([self.rays_for_tick(t) for t in range(tick0, tick0 + nticks)])


def blackbody_bins(units: Units, T: float = 1e5, nbins: int = 8,
                   emin_ry: float = 1.0, emax_ry: float = 10.0):
    """Photon energies and photon-number weights of an nbins-line blackbody
    spectrum (spectra.c:29-31 shape, integrated over log-spaced bins)."""
    edges = np.geomspace(emin_ry, emax_ry, nbins + 1) * units.RY_ENG
    mids = np.sqrt(edges[1:] * edges[:-1])
    kT = units.BOLTZMANN * T
    nwt = mids ** 2 / np.expm1(mids / kT) * (edges[1:] - edges[:-1])
    return mids, nwt


@dataclass
class Workload:
    name: str
    field: Field
    schedule: RaySchedule
    nticks: int
    tick_time: float
    isothermal: bool


def make_workload(name: str, seed: int = 20261203, n_side: int | None = None,
                  nray: int | None = None) -> Workload:
    """The measured workloads. ``n_side``/``nray`` override sizes for tests."""
    units = Units(hmf=1.0)
    duration = 500 * units.MYR
    nticks = 10000
    tick_time = duration / nticks
    if name in ("iliev32", "iliev64"):
        ns = n_side or (32 if name == "iliev32" else 64)
        R = nray or (32 if name == "iliev32" else 1024)
        f = uniform_field(ns, seed, units=units)
        src = [Source(pos=(0.0, 0.0, 0.0), ngamma_dot=5e-2 * 1e50 / units.SEC)]
        sch = RaySchedule(sources=src, nray=R, tick_time=tick_time, boxsize=f.boxsize,
                          seed=seed + 1, energies=np.array([13.6 * units.EV]),
                          eweights=np.array([1.0]))
        return Workload(name, f, sch, nticks, tick_time, True)
    if name == "lognormal128":
        ns = n_side or 128
        R = nray or 8192
        f = lognormal_field(ns, seed, sigma=1.0, units=units)
        rng = np.random.Generator(np.random.Philox(key=seed + 7))
        nsrc = 16
        pos = rng.random((nsrc, 3)) * f.boxsize
        lum = 10 ** rng.uniform(47, 49, nsrc)
        src = [Source(pos=tuple(p), ngamma_dot=l / units.SEC) for p, l in zip(pos, lum)]
        e, w = blackbody_bins(units)
        sch = RaySchedule(sources=src, nray=R, tick_time=tick_time, boxsize=f.boxsize,
                          seed=seed + 1, energies=e, eweights=w)
        return Workload(name, f, sch, nticks, tick_time, False)
    if name == "lognormal256":
        # the full pipeline's field: 256^3 particles, sigma 1.5, 256 sources
        # of 1e46-1e49 photons/s, 65536 rays per tick, not isothermal
        ns = n_side or 256
        R = nray or 65536
        f = lognormal_field(ns, seed, sigma=1.5, units=units)
        rng = np.random.Generator(np.random.Philox(key=seed + 7))
        nsrc = 256
        pos = rng.random((nsrc, 3)) * f.boxsize
        lum = 10 ** rng.uniform(46, 49, nsrc)
        src = [Source(pos=tuple(p), ngamma_dot=l / units.SEC) for p, l in zip(pos, lum)]
        e, w = blackbody_bins(units)
        sch = RaySchedule(sources=src, nray=R, tick_time=tick_time, boxsize=f.boxsize,
                          seed=seed + 1, energies=e, eweights=w)
        return Workload(name, f, sch, nticks, tick_time, False)
    raise ValueError(f"unknown workload {name}")
