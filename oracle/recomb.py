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


def temperature(ie, lam, c, l1=None, l2=None) -> np.ndarray:
    """ieye2T() src/config.h:106-110 with psys_ye() (no yeMET; helium
    fractions l1 = x_HeI, l2 = x_HeII, 0 with HOnly), the product's
    rounding order."""
    l1 = np.zeros_like(lam) if l1 is None else l1
    l2 = np.zeros_like(lam) if l2 is None else l2
    ye = (1.0 - lam) + c["hemf"] / c["hmf"] * 0.25 * (l2 + 2 * (1.0 - l2 - l1))
    den = (c["hemf"] * 0.25 + c["hmf"]) + c["hmf"] * ye
    return ((c["MPROTON_OVER_BOLTZMANN"] * ie.astype(np.float64)) / den * 2.0) / 3.0


THRESHOLDS = ("HI_ENERGY", "HEI_ENERGY", "HEII_ENERGY")
PICK_STREAMS = (4, 7, 8)        # the emitter draws of HII, HeII, HeIII recombinations


def emit(yg, lam, mark, pos, mass, ie, tick: int, nrec: int, seed: int, boxsize: float, consts: dict,
         lte=None, threshold: float = 0.1, l1=None, l2=None, types: bool = False):
    """State arrays in caller order. yg: yGrecHII, or the list [yGrecHII,
    yGrecHeII, yGrecHeIII] (helium); lte: (freq, cdf) or a list of them per
    species, None for disableLTE. Returns (rays, emitter index[, type],
    yGrec after the emission, in the form given)."""
    from psphray_b200.fields import RAY_DTYPE
    single = not isinstance(yg, (list, tuple))
    ygs = [yg] if single else list(yg)
    ltes = [lte] if (single or lte is None or not isinstance(lte, list)) else lte
    n = len(lam)
    marked = mark == tick - 1
    keys = []
    if nrec != 0:
        for s, y in enumerate(ygs):
            y64 = y.astype(np.float64)
            if nrec > 0:
                x = np.where(lam == 0.0, 1e-10, lam)
                w = np.where(marked, y64 / x, 0.0)
                cdf = np.cumsum(w)
                total = cdf[-1]
                if not total > 0.0:
                    continue
                d = _draw(nrec, tick, PICK_STREAMS[s], seed)
                c = np.searchsorted(cdf, _u01(d[:, 0], d[:, 1]) * total, side="right")
                c[c >= n] = np.searchsorted(cdf, total, side="left")
                keys.append((np.int64(s) << 56) | (c.astype(np.int64) << 24) | np.arange(nrec, dtype=np.int64))
            else:
                c = np.nonzero(marked & (y64 > threshold))[0].astype(np.int64)
                keys.append((np.int64(s) << 56) | (c << 24))
    keys = np.sort(np.concatenate(keys)) if keys else np.zeros(0, np.int64)
    em = (keys >> 24) & 0xFFFFFFFF
    typ = (keys >> 56).astype(np.int32)
    M = len(keys)
    rays = np.zeros(M, RAY_DTYPE)
    outs = [y.copy() for y in ygs]
    if M:
        run = keys >> 24
        _, inv, cnt = np.unique(run, return_inverse=True, return_counts=True)
        c_of = cnt[inv].astype(np.float64)
        per = np.where(typ == 0, consts["H_PER_MASS"], consts.get("HE_PER_MASS", 0.0))
        N = mass[em].astype(np.float64) * per
        ygv = np.array([float(ygs[s][p]) for s, p in zip(typ, em)])
        rays["Nph"] = (ygv * N) * (1.0 / c_of)
        rays["s"] = pos[em].astype(np.float32)
        rays["length"] = boxsize * 2.0 * 0.1
        d5 = _draw(M, tick, 5, seed)
        cz = 2.0 * _u01(d5[:, 0], d5[:, 1]) - 1.0
        phi = (2.0 * 3.141592653589793) * _u01(d5[:, 2], d5[:, 3])
        st = np.sqrt(np.maximum(0.0, 1.0 - cz * cz))
        rays["dir"] = np.stack([st * np.cos(phi), st * np.sin(phi), cz], axis=1).astype(np.float32)
        if lte is None:
            rays["freq"] = [consts[THRESHOLDS[s]] for s in typ]
        else:
            T = temperature(ie[em], lam[em], consts, None if l1 is None else l1[em], None if l2 is None else l2[em])
            rows = np.clip(np.trunc((np.log10(T) - 3.0) / (7.0 / NLOGT)).astype(np.int64), 0, NLOGT - 1)
            d6 = _draw(M, tick, 6, seed)
            u = _u01(d6[:, 0], d6[:, 1])
            fr = []
            for s, r, uu in zip(typ, rows, u):
                th = consts[THRESHOLDS[s]]
                fr.append(th + (16.0 * th - th) / NFREQ * lte_index(ltes[s][1][r], uu))
            rays["freq"] = fr
        for i in range(M):
            s, p = typ[i], em[i]
            y = np.float32(np.float64(np.float32(outs[s][p])) - rays["Nph"][i] / N[i])
            outs[s][p] = max(y, np.float32(0.0))
    after = outs[0] if single else outs
    return (rays, em, typ, after) if types else (rays, em, after)


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
