"""Oracle for recombination rays (test infrastructure only; never on the
product path).

Restates, in numpy, what the device does at the start of a tick when not on
the spot:

- lte_table(): lte_fill() src/lte.c:46-72 for hydrogen -- 128 rows of
  log T = 3 + i*7/128, 1024 energies E_HI + j*15 E_HI/1024, weights
  sigma_HI(E) E^3 exp(-(E - E_HI)/kT), summed in order per row;
- emit(): the recombination half of emit_rays() src/loop.c:197-232,
  273-300, 305-320, 345-356 -- the previous tick's emitters (particles on
  the hit lists of its source rays and of its first recombination ray),
  nrec draws by yGrecHII/xHI (xHI = 0 as 1e-10) or, with nrec < 0, every
  emitter above the threshold (nrec = 0: none); rays in (emitter, draw) order, photons
  yGrecHII*NH split over the rays of each emitter, position of the
  emitter, isotropic direction, length 0.2 box, energy from lte_gen_freq()
  src/lte.c:36-44 at the emitter's temperature psys_T() src/psystem.h:180;
  then the photons leave yGrecHII, ray by ray in float, not below 0;
- the library's own draws (Philox4x32-10, oracle/emit.py): stream 4 the
  emitter (counter = draw index), 5 the direction and 6 the energy
  (counter = the ray's index after the sort). The weights are summed in
  the caller's particle order.

The reference's GSL MT19937 and Walker tables cannot be reproduced on the
device; parity is against this restatement, whose table is pinned against
the reference's own lte_fill() and lte_gen_freq() (tests/test_recomb_oracle.py).
"""
from __future__ import annotations

import numpy as np

from emit import _draw, _u01

NLOGT, NFREQ = 128, 1024


def lte_table(hi_energy: float, boltzmann: float, xs_hi, weights: bool = False):
    """(freq[NFREQ], cdf[NLOGT][NFREQ]) (and the weights themselves with
    weights=True); xs_hi(E) is sigma_HI."""
    fmin, fmax = hi_energy, 16.0 * hi_energy
    fstep = (fmax - fmin) / NFREQ
    freq = np.array([fmin + fstep * j for j in range(NFREQ)])
    sig = np.array([xs_hi(f) for f in freq])
    cdf = np.zeros((NLOGT, NFREQ))
    wt = np.zeros((NLOGT, NFREQ))
    tstep = (10.0 - 3.0) / NLOGT
    for i in range(NLOGT):
        kT = boltzmann * 10.0 ** (3.0 + tstep * i)
        w = sig * freq * freq * freq * np.exp(-(freq - fmin) / kT)
        wt[i] = w
        acc = 0.0
        for j in range(NFREQ):
            acc += w[j]
            cdf[i, j] = acc
    return (freq, cdf, wt) if weights else (freq, cdf)


def lte_index(cdf_row: np.ndarray, u: float) -> int:
    total = cdf_row[-1]
    j = int(np.searchsorted(cdf_row, u * total, side="right"))
    if j >= NFREQ:
        j = int(np.searchsorted(cdf_row, total, side="left"))
    return j


def temperature(ie, lam, c) -> np.ndarray:
    """ieye2T() src/config.h:106-110 with psys_ye() (no yeMET), the
    product's rounding order."""
    he_e = c["hemf"] / c["hmf"] * 0.25 * 2.0
    ye = (1.0 - lam) + he_e
    den = (c["hemf"] * 0.25 + c["hmf"]) + c["hmf"] * ye
    return ((c["MPROTON_OVER_BOLTZMANN"] * ie.astype(np.float64)) / den * 2.0) / 3.0


def emit(yg, lam, mark, pos, mass, ie, tick: int, nrec: int, seed: int, boxsize: float, consts: dict,
         lte=None, threshold: float = 0.1):
    """State arrays in caller order. Returns (rays, emitter index, yGrecHII
    after the emission). lte = (freq, cdf) or None (disableLTE)."""
    from psphray_b200.fields import RAY_DTYPE
    n = len(lam)
    marked = mark == tick - 1
    yg64 = yg.astype(np.float64)
    if nrec == 0:
        return np.zeros(0, RAY_DTYPE), np.zeros(0, np.int64), yg.copy()
    if nrec > 0:
        x = np.where(lam == 0.0, 1e-10, lam)
        w = np.where(marked, yg64 / x, 0.0)
        cdf = np.cumsum(w)
        total = cdf[-1]
        if not total > 0.0:
            return np.zeros(0, RAY_DTYPE), np.zeros(0, np.int64), yg.copy()
        d = _draw(nrec, tick, 4, seed)
        c = np.searchsorted(cdf, _u01(d[:, 0], d[:, 1]) * total, side="right")
        c[c >= n] = np.searchsorted(cdf, total, side="left")
        keys = (c.astype(np.int64) << 24) | np.arange(nrec, dtype=np.int64)
        em = c[np.argsort(keys, kind="stable")].astype(np.int64)
    else:
        em = np.nonzero(marked & (yg64 > threshold))[0].astype(np.int64)
    M = len(em)
    rays = np.zeros(M, RAY_DTYPE)
    if M == 0:
        return rays, em, yg.copy()
    _, inv, cnt = np.unique(em, return_inverse=True, return_counts=True)
    c_of = cnt[inv].astype(np.float64)
    NH = mass[em].astype(np.float64) * consts["H_PER_MASS"]
    rays["Nph"] = (yg64[em] * NH) * (1.0 / c_of)
    rays["s"] = pos[em].astype(np.float32)
    rays["length"] = boxsize * 2.0 * 0.1
    d5 = _draw(M, tick, 5, seed)
    cz = 2.0 * _u01(d5[:, 0], d5[:, 1]) - 1.0
    phi = (2.0 * 3.141592653589793) * _u01(d5[:, 2], d5[:, 3])
    st = np.sqrt(np.maximum(0.0, 1.0 - cz * cz))
    rays["dir"] = np.stack([st * np.cos(phi), st * np.sin(phi), cz], axis=1).astype(np.float32)
    if lte is None:
        rays["freq"] = consts["HI_ENERGY"]
    else:
        freq, table = lte
        T = temperature(ie[em], lam[em], consts)
        rows = np.clip(np.trunc((np.log10(T) - 3.0) / (7.0 / NLOGT)).astype(np.int64), 0, NLOGT - 1)
        d6 = _draw(M, tick, 6, seed)
        u = _u01(d6[:, 0], d6[:, 1])
        fstep = (16.0 * consts["HI_ENERGY"] - consts["HI_ENERGY"]) / NFREQ
        rays["freq"] = [consts["HI_ENERGY"] + fstep * lte_index(table[r], uu) for r, uu in zip(rows, u)]
    out = yg.copy()
    for i in range(M):
        p = em[i]
        y = np.float32(out[p])
        y = np.float32(np.float64(y) - rays["Nph"][i] / NH[i])
        out[p] = max(y, np.float32(0.0))
    return rays, em, out


def iso_step(lam0, gdep, time, nH, T, yeMET, he_e, ar_get):
    """One isothermal step not on the spot, as the device computes it: the
    case-A Riccati closed form for lambdaH and the exact integral of the
    recombination photons, d(yGrecHII)/ds = time*alpha_AB*ye*x_HII
    (solve.c:83-86). ar_get(column, logT) gives the rate table's columns.
    Returns (lambdaH unclamped, yGrecHII gained)."""
    import math
    logT = math.log10(T)
    gamma = ar_get("HIci", logT) * nH
    aA = ar_get("HIIrcA", logT) * nH
    aB = ar_get("HIIrcB", logT) * nH
    m = yeMET + he_e
    a = time * (aA + gamma)
    b = time * (aA + (aA + gamma) * (1 + m))
    q = time * (gamma * (1 + m) + aA * m)
    c = time * aA * (1 + m) - gdep
    if not a > 0:
        return lam0 + c, 0.0
    k = math.sqrt(q * q + 4 * a * gdep)
    ph = -math.expm1(-k) / k if k > 1e-6 else 1 - k * (0.5 - k / 6)
    p1 = 2 * c / (b + k)
    y0 = lam0 - p1
    z = a * y0 * ph
    L = 1 + z * (0.5 + z * (1 / 3 + 0.25 * z)) if abs(z) < 1e-4 else -math.log1p(-z) / z
    I1 = p1 + y0 * ph * L
    lam1 = p1 + y0 * math.exp(-k) / (1 - a * y0 * ph)
    aab = max(aA - aB, 0.0)
    return lam1, time * aab * ((1 + m) - (2 + m) * I1) + (aab / (aA + gamma)) * (lam1 - lam0 + b * I1 - c)


def noniso_step(lam0, ie0, gdep, heat, time, nH, yeMET, yg0, consts, ar_get, rtol=1e-11):
    """One step not isothermal and not on the spot, integrated tightly
    (Radau): function() solve.c:76-141 for hydrogen with case-A
    recombination, eta = HII rcc A, and the recombination photons
    (solve.c:83-86). Returns (lambdaH clamped to [0,1], ie, yGrecHII)."""
    import math

    from scipy.integrate import solve_ivp
    hmf, hemf = consts["hmf"], consts["hemf"]
    he_e = hemf / hmf * 0.5
    hpm, mob = consts["H_PER_MASS"], consts["MPROTON_OVER_BOLTZMANN"]

    def f(s, x):
        lam, e = x[0], x[1]
        xHII = 1.0 - lam
        ye = xHII + he_e + yeMET
        T = mob * e / (hemf * 0.25 + hmf + hmf * ye) * 2.0 / 3.0
        lt = math.log10(T)
        gam, aA, aB = (ar_get(k, lt) * nH for k in ("HIci", "HIIrcA", "HIIrcB"))
        eta, psi, zeta, beta = (ar_get(k, lt) * nH for k in ("HIIrccA", "HIcec", "HIcic", "Brem"))
        chi = ar_get("Compton", lt)
        L = hpm * ((zeta + psi) * ye * lam + eta * ye * xHII + beta * ye * xHII + chi * ye)
        return [-gdep + time * ye * (aA * xHII - gam * lam), heat - time * L, time * max(aA - aB, 0.0) * ye * xHII]
    sol = solve_ivp(f, (0.0, 1.0), [lam0, ie0, yg0], method="Radau", rtol=rtol,
                    atol=[1e-14, 1e-14 * abs(ie0), 1e-15])
    return min(1.0, max(0.0, sol.y[0, -1])), sol.y[1, -1], sol.y[2, -1]
