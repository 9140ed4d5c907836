"""The deposit's group logic (psg_tick.cu: deposit_ray, settle_capped),
modelled hit by hit in Python, against the sequential recurrence of
loop.c:440-590 that it parallelises: per ray, TM_{j+1} = TM_j - a_j with
a_j = TM_j*(-expm1(-tau_j)) capped at the hit's neutral atoms N_j, and the
ray ends after the first hit that leaves TM/Nph < 1e-10.

The model keeps the kernel's order of evaluation where it matters to the
decisions: in the one-at-a-time form, TM before hit j is
TM*exp(-(sum of the earlier tau)) from the last settled hit; in the
affine-map form, each hit is the map TM -> TM - N (guessed capped) or
TM -> TM*(1 - m) (not), composed over the earlier hits of the pass, and a
pass settles the hits before the first whose decision or cut disagrees
with the guess. Both forms must reach the sequential recurrence's cap
decisions and ray ends exactly, and its deposits to rounding."""
import math
import random

import pytest

CUT = 1e-10


def below(TM, Nph):
    return TM < 0 or TM / Nph < CUT


def sequential(Nph, taus, Ns):
    out, ncap = [], 0
    TM = Nph
    for tau, N in zip(taus, Ns):
        if tau == 0.0:
            out.append(-1.0)
            continue
        a = TM * -math.expm1(-tau)
        if a > N:
            a = N
            ncap += 1
        TM -= a
        out.append(a)
        if below(TM, Nph):
            out += [-1.0] * (len(taus) - len(out))
            return out, ncap, True
    return out, ncap, False


def group(Nph, taus, Ns, aff):
    """One step of NT = len(taus) hits, the kernel's loop."""
    NT = len(taus)
    delta = [-1.0] * NT
    ncap, start, done, TM = 0, 0, False, Nph
    m1 = [(-math.expm1(-x) if x != 0.0 else 0.0) for x in taus]
    while not done and start < NT:
        # optical-depth scan from start
        ex, f, seen = 0.0, NT, {}
        for t in range(start, NT):
            if taus[t] == 0.0:
                continue
            TMj = TM * math.exp(-ex)
            a = TMj * m1[t]
            seen[t] = (TMj, a)
            if (a > Ns[t] or below(TMj - a, Nph)) and f == NT:
                f = t
            ex += taus[t]
        for t in range(start, f):
            if t in seen:
                delta[t] = seen[t][1]
        if f == NT:
            break
        TMj, a = seen[f]
        if a > Ns[f]:
            a = Ns[f]
            ncap += 1
        delta[f] = a
        TM = TMj - a
        done = below(TM, Nph)
        start = f + 1
        if aff and not done:
            # settle_capped(): passes of composed affine maps
            guess = [t >= start and taus[t] != 0.0 and TM * m1[t] > Ns[t] for t in range(NT)]
            while start < NT:
                A, B, m, res = 1.0, 0.0, NT, {}
                for t in range(start, NT):
                    if taus[t] == 0.0:
                        continue
                    TMj = A * TM + B
                    a = TMj * m1[t]
                    cap = a > Ns[t]
                    after = TMj - Ns[t] if cap else TMj - a
                    res[t] = (a, cap, after)
                    if (cap != guess[t] or below(after, Nph)) and m == NT:
                        m = t
                    if guess[t]:
                        B = B - Ns[t]
                    else:
                        A, B = A * (1.0 - m1[t]), B * (1.0 - m1[t])
                for t in range(start, min(m + 1, NT)):
                    if t in res:
                        a, cap, _ = res[t]
                        delta[t] = Ns[t] if cap else a
                        ncap += cap
                if m == NT:
                    break
                TM = res[m][2]
                start = m + 1
                guess = [res.get(t, (0.0, False, 0.0))[1] for t in range(NT)]
                if below(TM, Nph):
                    done = True
                    break
            break
    return delta, ncap, done


def _rays(kind, n, seed):
    rng = random.Random(seed)
    for _ in range(n):
        NT = rng.choice([32, 128, 512])
        if kind == "mixed":
            Nph = 10 ** rng.uniform(0, 12)
            taus = [0.0 if rng.random() < 0.1 else 10 ** rng.uniform(-6, 1) for _ in range(NT)]
            Ns = [10 ** rng.uniform(-3, 3) for _ in range(NT)]
        elif kind == "bright":
            # long capped runs through ionised gas: tiny tau and atoms, many photons
            Nph = 10 ** rng.uniform(6, 12)
            taus = [0.0 if rng.random() < 0.05 else 10 ** rng.uniform(-8, -2) for _ in range(NT)]
            Ns = [t * 10 ** rng.uniform(-1, 2) for t in taus]
        else:
            # dim rays that end on the cut inside the step
            Nph = 1.0
            taus = [10 ** rng.uniform(-2, 0.5) for _ in range(NT)]
            Ns = [10 ** rng.uniform(-4, 0) for _ in range(NT)]
        yield Nph, taus, Ns


@pytest.mark.parametrize("aff", [False, True])
@pytest.mark.parametrize("kind", ["mixed", "bright", "cut"])
def test_group_settle_matches_sequential(kind, aff):
    ncap_all = 0
    for Nph, taus, Ns in _rays(kind, 400, {"mixed": 1, "bright": 2, "cut": 3}[kind]):
        d_seq, c_seq, e_seq = sequential(Nph, taus, Ns)
        d_grp, c_grp, e_grp = group(Nph, taus, Ns, aff)
        assert c_grp == c_seq and e_grp == e_seq
        for a, b in zip(d_seq, d_grp):
            assert (a < 0) == (b < 0)
            if a > 0:
                assert abs(a - b) <= 1e-10 * a
        ncap_all += c_seq
    if kind == "bright":
        assert ncap_all > 10_000
