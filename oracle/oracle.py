"""ctypes driver for oracle/_ref/libpsg_oracle.so, the C restatement of the
hot path (oracle/psg_oracle.c). Test and baseline infrastructure only.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpsg_oracle.so")
HIT_DTYPE = np.dtype([("ipar", "<i8"), ("d", "<f8"), ("b", "<f8")])

P = C.POINTER(C.c_double)


class POTables(C.Structure):
    _fields_ = [("ar_nrows", C.c_int), ("ar_min", C.c_double), ("ar_step_inv", C.c_double),
                ("ar_logT", P), ("ar_col", P * 9),
                ("xs_nrows", C.c_int), ("xs_min", C.c_double), ("xs_step_inv", C.c_double),
                ("xs_cut_HI", C.c_double), ("xs_eng", P), ("xs_HI", P),
                ("kernel", P), ("kernel_n", C.c_int),
                ("H_PER_MASS", C.c_double), ("HI_ENERGY", C.c_double),
                ("MPROTON_OVER_BOLTZMANN", C.c_double), ("BOLTZMANN_OVER_MPROTON", C.c_double),
                ("hmf", C.c_double), ("hemf", C.c_double),
                ("isothermal", C.c_int), ("on_the_spot", C.c_int), ("adiabatic", C.c_int)]


class POState(C.Structure):
    _fields_ = [("n", C.c_size_t)] + [(k, C.c_void_p) for k in (
        "pos", "mass", "sml", "rho", "yeMET", "flag", "lambdaH", "ie", "yGdepHI", "heat", "hits", "lasthit")]


class POStats(C.Structure):
    _fields_ = [("total_hits", C.c_double), ("saturated", C.c_double), ("active", C.c_double),
                ("lost_photons", C.c_double)]


def _lib():
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle oracle`")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.po_tree_build.restype = vp
    L.po_tree_build.argtypes = [C.c_size_t, vp, vp, C.c_double, C.c_int]
    L.po_tree_free.argtypes = [vp]
    L.po_tree_ncells.restype = C.c_size_t
    L.po_tree_ncells.argtypes = [vp]
    L.po_tree_skipped.restype = C.c_size_t
    L.po_tree_skipped.argtypes = [vp]
    L.po_tree_cells.argtypes = [vp] * 8
    L.po_trace.restype = C.c_size_t
    L.po_trace.argtypes = [vp, vp, vp, vp, vp, C.POINTER(vp), C.POINTER(C.c_size_t)]
    L.po_free.argtypes = [vp]
    L.po_tick.argtypes = [vp, C.POINTER(POState), C.POINTER(POTables), vp, C.c_size_t, C.c_int64,
                          C.c_double, C.POINTER(POStats)]
    L.po_deposit.argtypes = [C.POINTER(POState), C.POINTER(POTables), vp, C.c_size_t, vp, vp,
                             C.POINTER(POStats)]
    L.po_solve.argtypes = [C.POINTER(POTables), C.POINTER(C.c_double), C.POINTER(C.c_double)] + [C.c_double] * 6
    L.po_solve.restype = C.c_int
    L.po_solve_numeric.argtypes = L.po_solve.argtypes
    L.po_solve_numeric.restype = C.c_int
    L.po_pluecker.argtypes = [vp, C.c_float, vp, vp]
    L.po_pluecker.restype = C.c_int
    return L


class Oracle:
    """CPU restatement over one field; holds its own particle state."""

    def __init__(self, field, phys, isothermal=True, on_the_spot=True, adiabatic=False, flag=None):
        self.L = _lib()
        self.f = field
        t = phys.tables_for_oracle()
        self._t = t
        cu = phys.cu
        cols = (P * 9)(*[t["ar_cols"][i].ctypes.data_as(P) for i in range(9)])
        self.tb = POTables(t["ar_nrows"], t["ar_min"], t["ar_step_inv"], t["ar_logT"].ctypes.data_as(P), cols,
                           t["xs_nrows"], t["xs_min"], t["xs_step_inv"], t["xs_cut_HI"],
                           t["xs_eng"].ctypes.data_as(P), t["xs_HI"].ctypes.data_as(P),
                           t["kernel"].ctypes.data_as(P), len(t["kernel"]),
                           cu.H_PER_MASS, cu.HI_ENERGY, cu.MPROTON_OVER_BOLTZMANN, cu.BOLTZMANN_OVER_MPROTON,
                           cu.hmf, cu.hemf, int(isothermal), int(on_the_spot), int(adiabatic))
        n = field.n
        self.pos = np.ascontiguousarray(field.pos, np.float32)
        self.sml = np.ascontiguousarray(field.sml, np.float32)
        self.mass = np.ascontiguousarray(field.mass, np.float32)
        self.rho = np.ascontiguousarray(field.rho, np.float32)
        xHI = field.xHI.astype(np.float64)
        xHII = 1.0 - xHI
        self.lambdaH = np.where((xHI >= 1.0) | (xHII <= 0.0), 1.0,
                                np.where((xHI <= 0.0) | (xHII >= 1.0), 0.0, xHI))
        self.yeMET = np.maximum(field.ye.astype(np.float64) - xHII, 0.0).astype(np.float32)
        self.ie = field.ie.astype(np.float32).copy()
        self.yGdepHI = np.zeros(n)
        self.heat = np.zeros(n)
        self.hits = np.zeros(n, np.int32)
        self.lasthit = np.zeros(n, np.int64)
        self.flag = None if flag is None else np.ascontiguousarray(flag, np.int8)
        self.tree = None

    def build_tree(self, ppc=8):
        if self.tree:
            self.L.po_tree_free(self.tree)
        self.tree = self.L.po_tree_build(self.f.n, self.pos.ctypes.data, self.sml.ctypes.data,
                                         self.f.boxsize, int(ppc))

    def tree_cells(self):
        nc = self.L.po_tree_ncells(self.tree)
        head = np.zeros(nc, np.int64); fc = np.zeros(nc, np.int64); par = np.zeros(nc, np.int64)
        npar = np.zeros(nc, np.uint32); bot = np.zeros((nc, 3), np.float32); top = np.zeros((nc, 3), np.float32)
        nxt = np.zeros(self.f.n, np.int64)
        self.L.po_tree_cells(self.tree, *[a.ctypes.data for a in (head, fc, par, npar, bot, top, nxt)])
        return dict(head=head, first_child=fc, parent=par, npar=npar, bot=bot, top=top, next=nxt,
                    skipped=self.L.po_tree_skipped(self.tree))

    def _state(self):
        self._st = POState(self.f.n, self.pos.ctypes.data, self.mass.ctypes.data, self.sml.ctypes.data,
                           self.rho.ctypes.data, self.yeMET.ctypes.data,
                           None if self.flag is None else self.flag.ctypes.data,
                           self.lambdaH.ctypes.data, self.ie.ctypes.data, self.yGdepHI.ctypes.data,
                           self.heat.ctypes.data, self.hits.ctypes.data, self.lasthit.ctypes.data)
        return self._st

    def trace(self, ray) -> np.ndarray:
        r = np.ascontiguousarray(np.atleast_1d(ray))
        x = C.c_void_p(); cap = C.c_size_t(0)
        n = self.L.po_trace(self.tree, self.pos.ctypes.data, self.sml.ctypes.data,
                            None if self.flag is None else self.flag.ctypes.data, r.ctypes.data,
                            C.byref(x), C.byref(cap))
        out = np.zeros(n, HIT_DTYPE)
        if n:
            C.memmove(out.ctypes.data, x, n * HIT_DTYPE.itemsize)
        self.L.po_free(x)
        return out

    def trace_all(self, rays):
        hits = [self.trace(r) for r in rays]
        off = np.zeros(len(rays) + 1, np.int64)
        off[1:] = np.cumsum([len(h) for h in hits])
        return off, (np.concatenate(hits) if hits else np.zeros(0, HIT_DTYPE))

    def tick(self, rays, tick, tick_time) -> dict:
        rays = np.ascontiguousarray(rays)
        st = POStats()
        rc = self.L.po_tick(self.tree, C.byref(self._state()), C.byref(self.tb), rays.ctypes.data,
                            len(rays), int(tick), float(tick_time), C.byref(st))
        return dict(hits=st.total_hits, saturated=st.saturated, active=st.active,
                    lost_photons=st.lost_photons, rc=rc)

    def deposit(self, rays, offsets, hits) -> dict:
        rays = np.ascontiguousarray(rays)
        offsets = np.ascontiguousarray(offsets, np.int64)
        hits = np.ascontiguousarray(hits, HIT_DTYPE)
        st = POStats()
        self.L.po_deposit(C.byref(self._state()), C.byref(self.tb), rays.ctypes.data, len(rays),
                          offsets.ctypes.data, hits.ctypes.data, C.byref(st))
        return dict(hits=st.total_hits, saturated=st.saturated, lost_photons=st.lost_photons)

    def solve(self, lambdaH, ie, yeMET, g, heat, time, nH, T, numeric=False):
        lam = C.c_double(lambdaH); e = C.c_double(ie)
        fn = self.L.po_solve_numeric if numeric else self.L.po_solve
        rc = fn(C.byref(self.tb), C.byref(lam), C.byref(e), yeMET, g, heat, time, nH, T)
        return lam.value, e.value, rc
