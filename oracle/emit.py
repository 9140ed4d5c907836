"""Oracle for source-ray emission (test infrastructure only; never on the
product path).

Restates, in numpy, what the device emission computes:

- the source-ray half of emit_rays() src/loop.c:163-373: per tick, weights
  Ngamma_dot*(tick-lastemit)*tick_time (psystem_weight_srcs()
  src/sources.c:67-78, with the history cursor of advance_cursor()
  src/sources.c:58-66), a source per ray drawn by weight, the source's
  photons split evenly over the rays that drew it (src/loop.c:305-320),
  lastemit set for every source that emitted (src/loop.c:324-328), point
  sources isotropic, plane sources a uniform point of the square
  (src/loop.c:242-262), an energy per ray from the source's spectrum
  (spec_gen_freq() src/spectra.c:50-60), length twice the box;
- the library's own random stream, Philox4x32-10 of Salmon et al. (SC'11):
  counter (ray index in the tick, tick low word, tick high word, stream),
  key = the 64-bit seed; a double uniform from the top 53 bits of two words.
  The reference's GSL MT19937 stream cannot be reproduced on the device, so
  parity here is against this restatement, and the semantics above against
  the reference's code (photon conservation, lastemit, cursor).
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr: np.ndarray, key: tuple[int, int]) -> np.ndarray:
    """ctr: uint32 array [..., 4]; returns the 4 output words, same shape."""
    c = [ctr[..., i].astype(np.uint64) for i in range(4)]
    k0, k1 = key[0] & 0xFFFFFFFF, key[1] & 0xFFFFFFFF
    for r in range(10):
        if r:
            k0 = (k0 + W0) & 0xFFFFFFFF
            k1 = (k1 + W1) & 0xFFFFFFFF
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        n0 = (p1 >> np.uint64(32)) ^ c[1] ^ np.uint64(k0)
        n2 = (p0 >> np.uint64(32)) ^ c[3] ^ np.uint64(k1)
        c = [n0 & MASK, p1 & MASK, n2 & MASK, p0 & MASK]
    return np.stack(c, axis=-1).astype(np.uint32)


def _u01(hi: np.ndarray, lo: np.ndarray) -> np.ndarray:
    x = (hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)
    return (x >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def _draw(nray: int, tick: int, stream: int, seed: int) -> np.ndarray:
    ctr = np.zeros((nray, 4), np.uint32)
    ctr[:, 0] = np.arange(nray, dtype=np.uint32)
    ctr[:, 1] = np.uint32(tick & 0xFFFFFFFF)
    ctr[:, 2] = np.uint32((tick >> 32) & 0xFFFFFFFF)
    ctr[:, 3] = np.uint32(stream)
    return philox4x32_10(ctr, (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))


class Emitter:
    """Sources (objects with pos, lastemit, ngamma_dot or ticks/ngamma_dots,
    optional type/specid/dir/a/b/radius) and spectra [(energies, weights)]."""

    def __init__(self, sources, spectra, seed: int, boxsize: float):
        self.src = sources
        self.seed = int(seed)
        self.length = 2.0 * boxsize
        self.lastemit = np.array([int(s.lastemit) for s in sources], np.int64)
        self.cursor = np.zeros(len(sources), np.int32)
        self.hist = []
        for s in sources:
            t = getattr(s, "ticks", None)
            self.hist.append((np.array([0] if t is None else t, np.int64),
                              np.array([s.ngamma_dot] if t is None else s.ngamma_dots, np.float64)))
        self.spec = []
        for eng, wt in spectra:
            eng = np.asarray(eng, np.float64)
            w = np.asarray(wt, np.float64) if len(eng) > 1 else np.ones(1)
            cdf = np.zeros(len(w))
            acc = 0.0
            for k in range(len(w)):          # in order, as the library sums
                acc += w[k]
                cdf[k] = acc
            self.spec.append((eng, cdf))

    def rays(self, nray: int, nticks: int, first_tick: int, tick_time: float) -> np.ndarray:
        from psphray_b200.fields import RAY_DTYPE
        out = np.zeros(nray * nticks, RAY_DTYPE)
        ns = len(self.src)
        for t in range(nticks):
            tick = first_tick + t
            w = np.zeros(ns)
            for i in range(ns):
                ticks, ngd = self.hist[i]
                c = self.cursor[i]
                while c < len(ticks) - 1 and ticks[c + 1] <= tick:
                    c += 1
                self.cursor[i] = c
                w[i] = (ngd[c] * float(tick - self.lastemit[i])) * tick_time
            cdf = np.zeros(ns)
            acc = 0.0
            for i in range(ns):
                acc += w[i]
                cdf[i] = acc
            pos_idx = np.nonzero(w > 0)[0]
            last_pos = int(pos_idx[-1]) if len(pos_idx) else 0
            x = _draw(nray, tick, 0, self.seed)
            target = _u01(x[:, 0], x[:, 1]) * cdf[-1]
            isrc = np.searchsorted(cdf, target, side="right")
            isrc[isrc >= ns] = last_pos
            cnt = np.bincount(isrc, minlength=ns)
            nph = np.where(cnt > 0, w * (1.0 / np.maximum(cnt, 1)), 0.0)
            self.lastemit[cnt > 0] = tick
            r = out[t * nray:(t + 1) * nray]
            r["Nph"] = nph[isrc]
            r["length"] = self.length
            x1 = _draw(nray, tick, 1, self.seed)
            c = 2.0 * _u01(x1[:, 0], x1[:, 1]) - 1.0
            phi = (2.0 * 3.141592653589793) * _u01(x1[:, 2], x1[:, 3])
            st = np.sqrt(np.maximum(0.0, 1.0 - c * c))
            x3 = _draw(nray, tick, 3, self.seed)
            u = 2.0 * _u01(x3[:, 0], x3[:, 1]) - 1.0
            v = 2.0 * _u01(x3[:, 2], x3[:, 3]) - 1.0
            x2 = _draw(nray, tick, 2, self.seed)
            uf = _u01(x2[:, 0], x2[:, 1])
            for j, i in enumerate(isrc):
                s = self.src[i]
                if int(getattr(s, "type", 1)) == 1:
                    r["s"][j] = np.asarray(s.pos, np.float64).astype(np.float32)
                    r["dir"][j] = np.array([st[j] * np.cos(phi[j]), st[j] * np.sin(phi[j]), c[j]]).astype(np.float32)
                else:
                    p, a, b = (np.asarray(getattr(s, k), np.float64) for k in ("pos", "a", "b"))
                    r["s"][j] = ((p + (u[j] * a) * s.radius) + (v[j] * b) * s.radius).astype(np.float32)
                    r["dir"][j] = np.asarray(s.dir, np.float64).astype(np.float32)
                eng, scdf = self.spec[int(getattr(s, "specid", 0))]
                if len(eng) == 1:
                    r["freq"][j] = eng[0]
                else:
                    k = int(np.searchsorted(scdf, uf[j] * scdf[-1], side="right"))
                    r["freq"][j] = eng[min(k, len(eng) - 1)]
        return out
