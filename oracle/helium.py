"""Oracle for helium and secondary ionisation (test infrastructure only;
never on the product path).

- secion_get(): tabfun2_get() src/tabfun.c:173-222 on a table built by
  psg_secion_table_build() (secion_init() src/secion.c:74-98), restated in
  Python: clamped rows or columns interpolate along the other axis, inside
  the table bilinear;
- he_step(): one step of function() src/solve.c:76-141 with helium, on
  the spot or not (then with the three recombination-photon counts),
  integrated tightly (Radau) over (lambdaH, lambdaHeI, lambdaHeII, ie),
  with LSODA's exit clamps (src/solve.c:208-213);
- load_split(): the helium fractions and yeMET that psystem_read_epoch()
  src/psystem.c:340-358 takes out of the ye block.
"""
from __future__ import annotations

import math

import numpy as np

NE, NX = 4096, 1024


def secion_get(table: np.ndarray, col: int, E: float, y: float, ev: float) -> float:
    """table[3][NE][NX] (PhiHI, PhiHeI, Eh); E in internal energy units."""
    min1, min2 = 10 * ev, -8.0
    step1 = (200 * ev - min1) / NE
    step2 = (0.0 - min2) / NX
    inv1, inv2 = 1.0 / step1, 1.0 / step2
    d = table[col]
    xind = int((E - min1) * inv1)
    yind = int((y - min2) * inv2)
    row = None
    if xind < 0:
        row = 0
    if xind >= NE - 1:
        row = NE - 1
    if row is not None:
        if yind < 0:
            return d[row, 0]
        if yind >= NX - 1:
            return d[row, NX - 1]
        left, right = min2 + yind * step2, min2 + (yind + 1) * step2
        return ((right - y) * d[row, yind] + (y - left) * d[row, yind + 1]) * inv2
    lin = None
    if yind < 0:
        lin = 0
    if yind >= NX - 1:
        lin = NX - 1
    if lin is not None:
        left, right = min1 + xind * step1, min1 + (xind + 1) * step1
        return ((right - E) * d[xind, lin] + (E - left) * d[xind + 1, lin]) * inv1
    x1, x2 = min1 + xind * step1, min1 + (xind + 1) * step1
    y1, y2 = min2 + yind * step2, min2 + (yind + 1) * step2
    fac = inv1 * inv2
    return fac * (d[xind, yind] * (x2 - E) * (y2 - y) + d[xind + 1, yind] * (E - x1) * (y2 - y)
                  + d[xind, yind + 1] * (x2 - E) * (y - y1) + d[xind + 1, yind + 1] * (E - x1) * (y - y1))


def load_split(xHI: np.ndarray, ye: np.ndarray, hmf: float):
    """(lambdaHeI, lambdaHeII, yeMET) from the xHI and ye blocks."""
    n = len(xHI)
    l1, l2, ym = np.zeros(n), np.zeros(n), np.zeros(n, np.float32)
    for i in range(n):
        xhii = 1.0 - float(xHI[i])
        yem = max(float(ye[i]) - xhii, 0.0)
        x2 = yem * hmf / (1 - hmf) * 4
        x3 = max(x2 - 1.0, 0.0)
        x2 = min(1.0, x2)
        x3 = min(1.0 - x2, x3)
        x1 = 1.0 - x2 - x3
        l1[i] = 1.0 if (x1 >= 1.0 or x2 + x3 <= 0.0) else (0.0 if (x1 <= 0.0 or x2 + x3 >= 1.0) else x1)
        l2[i] = 1.0 if (x2 >= 1.0 or x1 + x3 <= 0.0) else (0.0 if (x2 <= 0.0 or x3 + x1 >= 1.0) else x2)
        ym[i] = max(yem - (x2 + 2 * x3) * (1 - hmf) / hmf * 0.25, 0.0)
    return l1, l2, ym


def he_step(x0, yeMET, gHI, gHeI, gHeII, heat, time, nH, T, consts, ar_get, isothermal: bool, rtol=1e-10,
            on_the_spot: bool = True, rec0=(0.0, 0.0, 0.0), h_only: bool = False):
    """x0 = (lambdaH, lambdaHeI, lambdaHeII, ie); returns the four after one
    step, clamped as solve.c:208-210 does; not on the spot (case A) also
    the three recombination-photon counts from rec0 (clamped at 0,
    solve.c:211-213). With h_only the helium fractions stay put
    (solve.c:88-90, 96-98)."""
    from scipy.integrate import solve_ivp
    hmf, hemf = consts["hmf"], consts["hemf"]
    hpm, mob = consts["H_PER_MASS"], consts["MPROTON_OVER_BOLTZMANN"]

    def f(s, x):
        xHI, xHII, xHeII = x[0], 1.0 - x[0], x[2]
        xHeIII = 1.0 - x[2] - x[1]
        ye = (xHII + hemf / hmf * 0.25 * (xHeII + 2 * xHeIII)) + yeMET
        Tk = T if isothermal else mob * x[3] / (hemf * 0.25 + hmf + hmf * ye) * 2.0 / 3.0
        lt = math.log10(Tk)
        r = {k: ar_get(k, lt) * nH for k in ("HIci", "HIIrcA", "HIIrcB", "HeIci", "HeIIci", "HeIIrcA", "HeIIrcB",
                                              "HeIIIrcA", "HeIIIrcB", "HIIrccA", "HIIrccB", "HIcec", "HIcic", "Brem")}
        if on_the_spot:
            d0 = -gHI + time * (-r["HIci"] * ye * xHI + r["HIIrcB"] * ye * xHII)
            d1 = -gHeI + time * (-r["HeIci"] * ye * xHI + r["HeIIrcB"] * ye * xHeII)
            d2 = -gHeII + time * (-r["HeIIci"] * ye * xHI - r["HeIIrcB"] * ye * xHeII + r["HeIIIrcB"] * ye * xHeIII)
            dr = [0.0, 0.0, 0.0]
        else:
            xHeI = x[1]
            d0 = -gHI + time * (-r["HIci"] * ye * xHI + r["HIIrcA"] * ye * xHII)
            d1 = -gHeI + time * (-r["HeIci"] * ye * xHeI + r["HeIIrcA"] * ye * xHeII)
            d2 = -gHeII + time * (-r["HeIIci"] * ye * xHeII - r["HeIIrcA"] * ye * xHeII + r["HeIIIrcA"] * ye * xHeIII)
            dr = [time * max(r["HIIrcA"] - r["HIIrcB"], 0.0) * ye * xHII,
                  time * max(r["HeIIrcA"] - r["HeIIrcB"], 0.0) * ye * xHeII,
                  time * max(r["HeIIIrcA"] - r["HeIIIrcB"], 0.0) * ye * xHeIII]
        if isothermal:
            d3 = 0.0
        else:
            eta = r["HIIrccB"] if on_the_spot else r["HIIrccA"]
            L = hpm * ((r["HIcic"] + r["HIcec"]) * ye * xHI + eta * ye * xHII + r["Brem"] * ye * xHII
                       + ar_get("Compton", lt) * ye)
            d3 = heat - time * L
        if h_only:
            d1 = d2 = 0.0
            dr[1] = dr[2] = 0.0
        return [d0, d1, d2, d3] + dr
    sol = solve_ivp(f, (0.0, 1.0), list(x0) + list(rec0), method="Radau", rtol=rtol,
                    atol=[1e-13, 1e-13, 1e-13, 1e-13 * abs(x0[3]), 1e-15, 1e-15, 1e-15])
    x = sol.y[:, -1]
    l0 = min(1.0, max(0.0, x[0]))
    l1 = min(1.0, max(0.0, x[1]))
    l2 = min(1.0 - l1, max(0.0, x[2]))
    if on_the_spot:
        return l0, l1, l2, x[3]
    return l0, l1, l2, x[3], max(x[4], 0.0), max(x[5], 0.0), max(x[6], 0.0)
