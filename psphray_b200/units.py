"""Internal unit system of psphray, restated.

Follows ``units_init()`` (src/units.c:66-104) and the defaults of
``cfg_init()`` (src/config.c:15-23): lengths in kpc/h, masses in 1e10 Msun/h
(``massGramh``), times in ``timeSh``. Every constant is computed in the same
order of double operations as the reference so the values are bit-identical.
Also restates ``ieye2T`` / ``Tye2ie`` (src/config.h:106-114).
"""
from __future__ import annotations

from dataclasses import dataclass, field


@dataclass
class Units:
    h: float = 0.72
    hmf: float = 0.76
    length_cmh: float = 3.0835455558318480e21
    mass_gramh: float = 1.9847005219450705e43
    time_sh: float = 3.08568025e16
    hemf: float = field(init=False)

    def __post_init__(self) -> None:
        self.hemf = 1.0 - self.hmf
        C_H = self.h
        self.CM = C_H / self.length_cmh
        self.GRAM = C_H / self.mass_gramh
        self.SEC = C_H / self.time_sh
        self.M = self.CM * 100
        self.KM = self.M * 1000
        self.KPC = self.M * 3.08568025e19
        self.YR = self.SEC * 31556926.0
        self.KG = self.GRAM * 1000
        self.MYR = self.YR * 1e6
        self.MSUN = self.KG * 1.98892e30
        self.MPROTON = self.KG * 1.67262158e-27
        self.KELVIN = 1.0
        self.BOLTZMANN = 1.3806503e-23 * self.M * self.M * self.KG / self.SEC / self.SEC
        self.J = self.KG * self.M * self.M / (self.SEC * self.SEC)
        self.EV = 1.602176487e-19 * self.J
        self.ERG = 1e-7 * self.J
        self.RY_ENG = 13.60569253 * self.EV
        self.H_PER_MASS = self.hmf / self.MPROTON
        self.HE_PER_MASS = self.hemf / (4 * self.MPROTON)
        self.HI_ENERGY = 13.60569253 * self.EV
        self.HEI_ENERGY = 24.587 * self.EV
        self.HEII_ENERGY = 54.416 * self.EV
        self.MPROTON_OVER_BOLTZMANN = self.MPROTON / self.BOLTZMANN
        self.BOLTZMANN_OVER_MPROTON = 1.0 / (self.MPROTON / self.BOLTZMANN)

    def ieye2T(self, ie: float, ye: float) -> float:
        return self.MPROTON_OVER_BOLTZMANN * ie / (self.hemf * 0.25 + self.hmf + self.hmf * ye) * 2.0 / 3.0

    def Tye2ie(self, T: float, ye: float) -> float:
        return T * self.BOLTZMANN_OVER_MPROTON * (self.hemf * 0.25 + self.hmf + self.hmf * ye) / 2.0 * 3.0
