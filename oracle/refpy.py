"""ctypes driver for oracle/_ref/libpsphray_ref.so (the reference's own CPU
code, built by oracle/Makefile). Test and baseline infrastructure only: the
product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpsphray_ref.so")
EULER_LIB_PATH = os.path.join(HERE, "_ref", "libpsphray_ref_euler.so")   # solve.c without USE_LSODA


class Xtype(C.Structure):
    """psystem.h:108-112"""
    _fields_ = [("ipar", C.c_int64), ("d", C.c_double), ("b", C.c_double)]


class Step(C.Structure):
    """psystem.h:84-105"""
    _fields_ = [(n, C.c_double) for n in (
        "lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yeMET", "yGdepHI", "yGdepHeI",
        "yGdepHeII", "heat", "time", "nH", "T", "yGrecHII", "yGrecHeII", "yGrecHeIII",
        "step_remain")] + [("refined", C.c_int), ("ipar", C.c_int64)]


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


class Reference:
    """One process-wide instance: the reference keeps its state in globals."""

    _libs = {}

    def __init__(self, rates_path: str, units, isothermal=True, on_the_spot=True,
                 h_only=True, adiabatic=False, threads: int | None = None, lib_path: str = LIB_PATH):
        if lib_path in Reference._libs:
            raise RuntimeError("the reference harness holds global state; one instance per library and process")
        if not os.path.exists(lib_path):
            raise FileNotFoundError(f"{lib_path} missing: run `make -C oracle ref REF=<psphray tree>`")
        lib = C.CDLL(lib_path)
        Reference._libs[lib_path] = lib
        self.lib = lib
        lib.ref_setup.argtypes = [C.c_char_p] + [C.c_double] * 5 + [C.c_int] * 4
        lib.ref_sph_depth.restype = C.c_double
        lib.ref_sph_depth.argtypes = [C.c_double]
        lib.ref_ar_get.restype = C.c_double
        lib.ref_ar_get.argtypes = [C.c_int, C.c_double]
        lib.ref_xs_get.restype = C.c_double
        lib.ref_xs_get.argtypes = [C.c_int, C.c_double]
        lib.ref_load_particles.argtypes = [C.c_size_t] + [C.c_void_p] * 8 + [C.c_double]
        lib.ref_rt_trace.restype = C.c_size_t
        lib.ref_rt_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_float,
                                     C.POINTER(C.POINTER(Xtype)), C.POINTER(C.c_size_t)]
        lib.ref_free.argtypes = [C.c_void_p]
        lib.ref_set_rays.argtypes = [C.c_size_t, C.c_void_p, C.c_long, C.c_double]
        lib.ref_ray_nhits.restype = C.c_size_t
        lib.ref_ray_nhits.argtypes = [C.c_size_t]
        lib.ref_ray_hits.restype = C.c_size_t
        lib.ref_ray_hits.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_active_count.restype = C.c_size_t
        lib.ref_tree_ncells.restype = C.c_size_t
        lib.ref_step_evolve.argtypes = [C.c_void_p, C.c_size_t]
        lib.ref_sizeof_step.restype = C.c_size_t
        lib.ref_set_secondary.argtypes = [C.c_int]
        lib.ref_secion_get.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.ref_secion_get.restype = C.c_double
        lib.ref_get_he.argtypes = [C.c_void_p] * 5
        lib.ref_set_he.argtypes = [C.c_void_p] * 2
        lib.ref_get_ygrec.argtypes = [C.c_void_p]
        lib.ref_get_ygrec3.argtypes = [C.c_void_p] * 3
        lib.ref_set_ygrec3.argtypes = [C.c_void_p] * 3
        lib.ref_set_ygrec.argtypes = [C.c_void_p]
        lib.ref_lte_row.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        lib.ref_lte_row.restype = C.c_int
        lib.ref_lte_gen_freq.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.ref_lte_gen_freq.restype = C.c_double
        lib.ref_set_sources.argtypes = [C.c_int] + [C.c_void_p] * 6
        lib.ref_get_sources.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_emit_source_rays.argtypes = [C.c_int, C.c_int64, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                             C.c_void_p]
        lib.ref_emit_source_rays.restype = C.c_int
        assert lib.ref_sizeof_step() == C.sizeof(Step)
        self.units = units
        lib.ref_setup(rates_path.encode(), units.h, units.hmf, units.length_cmh,
                      units.mass_gramh, units.time_sh, int(isothermal), int(on_the_spot),
                      int(h_only), int(adiabatic))
        if threads is not None:
            lib.ref_set_threads(int(threads))
        ids = (C.c_int * 12)()
        lib.ref_ids(ids)
        self.ids = dict(zip(["HIci", "HIIrcA", "HIIrcB", "HIIrccA", "HIIrccB", "HIcic",
                             "HIcec", "Brem", "Compton", "XS_HI", "XS_HeI", "XS_HeII"],
                            list(ids)))
        self.n = 0

    def set_threads(self, n: int) -> None:
        self.lib.ref_set_threads(int(n))

    def units_vector(self) -> np.ndarray:
        out = np.zeros(16)
        self.lib.ref_units(_p(out, C.c_double))
        return out

    def load(self, f) -> None:
        self.n = f.n
        self._keep = [np.ascontiguousarray(a) for a in (f.pos, f.mass, f.sml, f.rho, f.ie, f.xHI, f.ye)]
        args = [a.ctypes.data for a in self._keep]
        self.lib.ref_load_particles(f.n, *args, None, f.boxsize)

    def build_tree(self, ppc: int = 8) -> None:
        self.lib.ref_build_tree(int(ppc))

    def tree(self):
        nc = self.lib.ref_tree_ncells()
        head = np.zeros(nc, np.int64); fc = np.zeros(nc, np.int64); par = np.zeros(nc, np.int64)
        npar = np.zeros(nc, np.uint32); bot = np.zeros((nc, 3), np.float32); top = np.zeros((nc, 3), np.float32)
        self.lib.ref_tree_cells(*[a.ctypes.data_as(C.c_void_p) for a in (head, fc, par, npar, bot, top)])
        nxt = np.zeros(self.n, np.int64)
        self.lib.ref_tree_next(nxt.ctypes.data_as(C.c_void_p))
        return dict(head=head, first_child=fc, parent=par, npar=npar, bot=bot, top=top, next=nxt)

    def rt_trace(self, s, d, dist):
        """rt_trace() raytrace.c:153 for one ray: (ipar, d, b) in walk order."""
        s = np.ascontiguousarray(s, np.float32); d = np.ascontiguousarray(d, np.float32)
        x = C.POINTER(Xtype)(); size = C.c_size_t(0)
        n = self.lib.ref_rt_trace(s.ctypes.data, d.ctypes.data, C.c_float(dist), C.byref(x), C.byref(size))
        arr = np.ctypeslib.as_array(C.cast(x, C.POINTER(C.c_char)), shape=(n * C.sizeof(Xtype),)).copy() if n else np.zeros(0, np.uint8)
        self.lib.ref_free(C.cast(x, C.c_void_p))
        rec = arr.view(np.dtype([("ipar", "<i8"), ("d", "<f8"), ("b", "<f8")]))
        return rec

    def set_rays(self, rays: np.ndarray, tick: int, tick_time: float) -> None:
        self._rays = np.ascontiguousarray(rays)
        self.lib.ref_set_rays(len(rays), self._rays.ctypes.data, int(tick), float(tick_time))

    def trace(self):
        self.lib.ref_trace()

    def deposit(self):
        self.lib.ref_deposit()

    def merge(self):
        self.lib.ref_merge()

    def update(self):
        self.lib.ref_update()

    def tick(self, rays, tick, tick_time):
        self.set_rays(rays, tick, tick_time)
        self.trace(); self.deposit(); self.merge(); self.update()

    def ray_hits(self, i: int):
        n = self.lib.ref_ray_nhits(i)
        ipar = np.zeros(n, np.int64); d = np.zeros(n); b = np.zeros(n)
        self.lib.ref_ray_hits(i, ipar.ctypes.data, d.ctypes.data, b.ctypes.data)
        return ipar, d, b

    def active(self) -> np.ndarray:
        n = self.lib.ref_active_count()
        out = np.zeros(n, np.int64)
        self.lib.ref_active(out.ctypes.data_as(C.c_void_p))
        return out

    def state(self):
        n = self.n
        lam = np.zeros(n); ie = np.zeros(n, np.float32); yg = np.zeros(n, np.float32)
        heat = np.zeros(n, np.float32); hits = np.zeros(n, np.int32); lh = np.zeros(n, np.int64)
        self.lib.ref_get_state(*[a.ctypes.data_as(C.c_void_p) for a in (lam, ie, yg, heat, hits, lh)])
        return dict(lambdaH=lam, ie=ie, yGdepHI=yg, heat=heat, hits=hits, lasthit=lh)

    def set_state(self, lambdaH=None, ie=None, lasthit=None):
        keep = [np.ascontiguousarray(lambdaH, np.float64) if lambdaH is not None else None,
                np.ascontiguousarray(ie, np.float32) if ie is not None else None,
                np.ascontiguousarray(lasthit, np.int64) if lasthit is not None else None]
        self.lib.ref_set_state(*[a.ctypes.data_as(C.c_void_p) if a is not None else None for a in keep])

    def set_secondary(self, on: bool) -> None:
        """psphray.secondaryIonization (builds secion.c's table once)."""
        self.lib.ref_set_secondary(int(bool(on)))

    def secion_get(self, col: int, E: float, log10x: float) -> float:
        """secion_get() src/secion.c for column 0 PhiHI, 1 PhiHeI, 2 Eh."""
        return self.lib.ref_secion_get(int(col), float(E), float(log10x))

    def he_state(self) -> dict:
        n = self.n
        a, b = np.zeros(n), np.zeros(n)
        c, d, e = (np.zeros(n, np.float32) for _ in range(3))
        self.lib.ref_get_he(*[x.ctypes.data_as(C.c_void_p) for x in (a, b, c, d, e)])
        return dict(lambdaHeI=a, lambdaHeII=b, yGdepHeI=c, yGdepHeII=d, yeMET=e)

    def set_he(self, lambdaHeI=None, lambdaHeII=None) -> None:
        keep = [None if v is None else np.ascontiguousarray(v, np.float64) for v in (lambdaHeI, lambdaHeII)]
        self.lib.ref_set_he(*[None if v is None else v.ctypes.data_as(C.c_void_p) for v in keep])

    def ygrec(self) -> np.ndarray:
        """yGrecHII of every particle (runs not on the spot)."""
        out = np.zeros(self.n, np.float32)
        self.lib.ref_get_ygrec(out.ctypes.data_as(C.c_void_p))
        return out

    def set_ygrec(self, yg) -> None:
        a = np.ascontiguousarray(yg, np.float32)
        self.lib.ref_set_ygrec(a.ctypes.data_as(C.c_void_p))

    def ygrec3(self):
        """[yGrecHII, yGrecHeII, yGrecHeIII] of every particle."""
        out = [np.zeros(self.n, np.float32) for _ in range(3)]
        self.lib.ref_get_ygrec3(*[a.ctypes.data_as(C.c_void_p) for a in out])
        return out

    def set_ygrec3(self, ygs) -> None:
        keep = [np.ascontiguousarray(a, np.float32) for a in ygs]
        self.lib.ref_set_ygrec3(*[a.ctypes.data_as(C.c_void_p) for a in keep])

    def lte_init(self) -> None:
        """lte_init() src/lte.c:30-34: the LTE recombination spectra."""
        self.lib.ref_lte_init()

    def lte_row(self, row: int, species: int = 0):
        """(energies, weights) of a row of the species' table (0 HI, 1 HeI,
        2 HeII; lte_fill() src/lte.c:46-72)."""
        f = np.zeros(1024); w = np.zeros(1024)
        n = self.lib.ref_lte_row(int(species), int(row), f.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p))
        return f[:n], w[:n]

    def lte_gen_freq(self, logT: float, u: float, species: int = 0) -> float:
        """lte_gen_freq() src/lte.c:36-44 of the species' table drawing at uniform u."""
        return self.lib.ref_lte_gen_freq(int(species), float(logT), float(u))

    def stats(self) -> dict:
        out = np.zeros(8)
        self.lib.ref_stats(out.ctypes.data_as(C.c_void_p))
        keys = ["hits", "saturated", "raytrace_time", "deposit_time", "merge_time",
                "update_time", "evolve_count", "lost_photons"]
        return dict(zip(keys, out.tolist()))

    def reset_stats(self):
        self.lib.ref_reset_stats()

    def step_evolve(self, steps):
        """step_evolve() solve.c:317 on an array of Step structs (in place)."""
        self.lib.ref_step_evolve(C.cast(steps, C.c_void_p), len(steps))
        return steps

    def sph_depth(self, r_h: float) -> float:
        return self.lib.ref_sph_depth(r_h)

    def ar_get(self, col: str, logT: float) -> float:
        return self.lib.ref_ar_get(self.ids[col], logT)

    def xs_get(self, col: str, freq: float) -> float:
        return self.lib.ref_xs_get(self.ids[col], freq)

    # ---- source rays: emit_rays() loop.c:163-373 with psystem_weight_srcs()
    def set_sources(self, sources) -> None:
        """Point sources: objects with pos, lastemit and either ngamma_dot or
        a history (ticks, ngamma_dots), as psystem.h's Source."""
        pos, hticks, hngd, off, nh, last = [], [], [], [], [], []
        for src in sources:
            t = list(src.ticks) if getattr(src, "ticks", None) is not None else [0]
            v = list(src.ngamma_dots) if getattr(src, "ngamma_dots", None) is not None else [src.ngamma_dot]
            off.append(len(hticks)); nh.append(len(t))
            hticks += t; hngd += v
            pos += [float(x) for x in src.pos]
            last.append(int(src.lastemit))
        self._src_keep = [np.ascontiguousarray(pos, np.float64), np.ascontiguousarray(hticks, np.int64),
                          np.ascontiguousarray(hngd, np.float64), np.ascontiguousarray(off, np.int32),
                          np.ascontiguousarray(nh, np.int32), np.ascontiguousarray(last, np.int64)]
        self.nsrc = len(sources)
        self.lib.ref_set_sources(self.nsrc, *[a.ctypes.data for a in self._src_keep])

    def sources_state(self):
        lastemit = np.zeros(self.nsrc, np.int64); cursor = np.zeros(self.nsrc, np.int64)
        self.lib.ref_get_sources(lastemit.ctypes.data, cursor.ctypes.data)
        return lastemit, cursor

    def emit_source_rays(self, nray: int, tick: int, tick_time: float, u, freq: float = 1.0):
        """One tick's source rays with the draws made at the uniforms u (ray
        order): each ray's source and photons, in the reference's ray order
        (by source)."""
        u = np.ascontiguousarray(u, np.float64)
        assert len(u) == nray
        isrc = np.zeros(nray, np.int64); nph = np.zeros(nray)
        n = self.lib.ref_emit_source_rays(int(nray), int(tick), float(tick_time), float(freq), u.ctypes.data,
                                          isrc.ctypes.data, nph.ctypes.data)
        return isrc[:n], nph[:n]
