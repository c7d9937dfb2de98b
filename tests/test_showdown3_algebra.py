"""CPU check of the three-way showdown algebra that k_term_sd2 runs on the
GPU: a numpy restatement of the rank-order sweep (same state, same update
and evaluation order) against brute-force tuple enumeration with the
reference payoffs (street_solve.cu:936-1002), on random river boards and on
boards with large tie groups.  Hand strengths come from the oracle's
evaluator (pinned to hand_eval.h)."""
import numpy as np
import pytest

from cards import card_to_int
from oracle.oracle import Oracle

D = 47
POT, BET = 100.0, 30.0


def _setup(seed, nh, board=None):
    rng = np.random.default_rng(seed)
    if board is None:
        board = [int(c) for c in rng.permutation(52)[:5]]
    orc = Oracle()
    rest = [c for c in range(52) if c not in board]
    combos = [(a, b) for i, a in enumerate(rest) for b in rest[i + 1:]]
    strength = {cb: int(orc.eval7(board + list(cb))) for cb in combos}
    order = sorted(combos, key=lambda cb: strength[cb])
    dense = {c: i for i, c in enumerate(rest)}

    def rand_range():
        sel = rng.choice(len(combos), nh, replace=False)
        return {combos[i]: float(rng.uniform(0, 1)) * (rng.random() > 0.2) for i in sel}

    return strength, order, dense, rand_range(), rand_range(), rand_range()


def _brute(strength, trav, opp1, opp2):
    out = {}
    for h in trav:
        v = 0.0
        for o1, r1 in opp1.items():
            for o2, r2 in opp2.items():
                if len({*h, *o1, *o2}) < 6 or r1 * r2 <= 0.0:
                    continue
                s, s1, s2 = strength[h], strength[o1], strength[o2]
                if s < max(s1, s2):
                    v -= r1 * r2 * BET
                else:
                    v += r1 * r2 * (POT / (1 + (s1 == s) + (s2 == s)) - BET)
        out[h] = v
    return out


class Sweep:
    """The kernel's state: M1, M2, P = M1 M2, card sums u1, u2, w = M2 u1 + M1 u2,
    d(c) = sum_b M1[c][b] M2[c][b], F1, F2, Q = sum u1 u2, D = sum d / 2."""

    def __init__(self):
        self.M = [np.zeros((D, D)), np.zeros((D, D))]
        self.P = np.zeros((D, D))
        self.u = [np.zeros(D), np.zeros(D)]
        self.w = np.zeros(D)
        self.d = np.zeros(D)
        self.F = [0.0, 0.0]
        self.Q = 0.0
        self.Dd = 0.0

    def mass(self, a, b):
        M1, M2, u1, u2 = self.M[0], self.M[1], self.u[0], self.u[1]
        m1, m2 = M1[a, b], M2[a, b]
        ga = u1[a] * u2[a] + self.w[a] - 2 * self.d[a]
        gb = u1[b] * u2[b] + self.w[b] - 2 * self.d[b]
        A1 = self.F[0] - u1[a] - u1[b] + m1
        A2 = self.F[1] - u2[a] - u2[b] + m2
        return (A1 * A2 + (self.Dd - self.Q) + ga + gb - m2 * (u1[a] + u1[b]) - m1 * (u2[a] + u2[b])
                + 3 * m1 * m2 - (self.P[a, b] + self.P[b, a]))

    def add(self, who, hands):
        Mo, Mx, uo, ux = self.M[who], self.M[1 - who], self.u[who], self.u[1 - who]
        for (x, y), r in hands:          # P: rows (opponent 1) or columns (opponent 2)
            if who == 0:
                self.P[x, :] += r * Mx[y, :]
                self.P[y, :] += r * Mx[x, :]
            else:
                self.P[:, x] += r * Mx[:, y]
                self.P[:, y] += r * Mx[:, x]
        for (x, y), r in hands:          # w, then the scalars and card sums
            self.w += r * (Mx[:, x] + Mx[:, y])
            self.w[x] += r * ux[y]
            self.w[y] += r * ux[x]
        for (x, y), r in hands:
            m = Mx[x, y]
            self.Q += r * (ux[x] + ux[y])
            self.Dd += r * m
            self.d[x] += r * m
            self.d[y] += r * m
            uo[x] += r
            uo[y] += r
            self.F[who] += r
        for (x, y), r in hands:
            Mo[x, y] = Mo[y, x] = r


def _sweep(strength, order, dense, trav, opp1, opp2):
    st, V, q = Sweep(), {}, 0
    while q < len(order):
        hi = q
        while hi < len(order) and strength[order[hi]] == strength[order[q]]:
            hi += 1
        group = order[q:hi]
        hs = [h for h in group if h in trav]
        h1 = [((dense[c[0]], dense[c[1]]), opp1[c]) for c in group if opp1.get(c, 0.0) > 0]
        h2 = [((dense[c[0]], dense[c[1]]), opp2[c]) for c in group if opp2.get(c, 0.0) > 0]
        for h in hs:                     # opponents weaker: A, and D(L, E) directly
            a, b = dense[h[0]], dense[h[1]]
            M1, u1 = st.M[0], st.u[0]
            dle = sum(r * (st.F[0] - u1[a] - u1[b] - u1[x] - u1[y] + M1[a, b] + M1[a, x] + M1[a, y]
                           + M1[b, x] + M1[b, y] + M1[x, y])
                      for (x, y), r in h2 if len({a, b, x, y}) == 4)
            V[h] = POT * (0.5 * st.mass(a, b) + dle / 6)
        st.add(0, h1)
        for h in hs:
            V[h] += POT / 6 * st.mass(dense[h[0]], dense[h[1]])
        st.add(1, h2)
        for h in hs:
            V[h] += POT / 3 * st.mass(dense[h[0]], dense[h[1]])
        q = hi
    return {h: V[h] - BET * st.mass(dense[h[0]], dense[h[1]]) for h in trav}


@pytest.mark.parametrize("seed,nh,board", [
    (0, 12, None), (1, 14, None), (2, 10, None),
    (3, 12, ["Ks", "Kd", "Kh", "Kc", "2s"]),
    (4, 10, ["As", "Ks", "Qs", "Js", "Ts"]),
])
def test_sweep_matches_enumeration(seed, nh, board):
    b = None if board is None else [card_to_int(c) for c in board]
    strength, order, dense, trav, opp1, opp2 = _setup(seed, nh, b)
    want = _brute(strength, trav, opp1, opp2)
    got = _sweep(strength, order, dense, trav, opp1, opp2)
    scale = max(1.0, max(abs(v) for v in want.values()))
    for h in trav:
        assert abs(got[h] - want[h]) <= 1e-9 * scale, (h, got[h], want[h])


def _direct(order, dense, opp1, opp2, qend):
    """The state of the hands at rank positions [0, qend) computed directly,
    as the kernel does at the start of each run: d = diag(P) and
    w = M2 u1 + M1 u2 = column sums + row sums of P (M1, M2 symmetric)."""
    st = Sweep()
    for c in order[:qend]:
        x, y = dense[c[0]], dense[c[1]]
        for k, opp in enumerate((opp1, opp2)):
            r = opp.get(c, 0.0)
            if r > 0:
                st.M[k][x, y] = st.M[k][y, x] = r
    st.P = st.M[0] @ st.M[1]
    st.u = [st.M[0].sum(0), st.M[1].sum(0)]
    st.d = np.diag(st.P).copy()
    st.w = st.P.sum(0) + st.P.sum(1)
    st.F = [0.5 * st.u[0].sum(), 0.5 * st.u[1].sum()]
    st.Q = float(st.u[0] @ st.u[1])
    st.Dd = 0.5 * st.d.sum()
    return st


def _sweep_runs(strength, order, dense, trav, opp1, opp2, nruns):
    """The sweep cut into runs of tie groups, each starting from a directly
    computed state, in the kernel's class form: A before the group, both tie
    sums D(L, E) + D(E, L) directly, C after the group, T2 = C - A - T1 (0
    when opponent 2 holds nothing in the group); the loss class from a direct
    state of all hands."""
    groups, q = [], 0
    while q < len(order):
        hi = q
        while hi < len(order) and strength[order[hi]] == strength[order[q]]:
            hi += 1
        groups.append((q, hi))
        q = hi
    cuts = [len(groups) * k // nruns for k in range(nruns + 1)]
    cls = {}
    for k in range(nruns):
        g0, g1 = cuts[k], cuts[k + 1]
        if g0 == g1:
            continue
        st = _direct(order, dense, opp1, opp2, groups[g0][0])
        for lo, hi in groups[g0:g1]:
            group = order[lo:hi]
            hs = [h for h in group if h in trav]
            h1 = [((dense[c[0]], dense[c[1]]), opp1[c]) for c in group if opp1.get(c, 0.0) > 0]
            h2 = [((dense[c[0]], dense[c[1]]), opp2[c]) for c in group if opp2.get(c, 0.0) > 0]
            for h in hs:                 # A, and both tie sums directly (four-card removals)
                a, b = dense[h[0]], dense[h[1]]
                M1, u1, M2, u2 = st.M[0], st.u[0], st.M[1], st.u[1]
                dle = sum(r * (st.F[0] - u1[a] - u1[b] - u1[x] - u1[y] + M1[a, b] + M1[a, x] + M1[a, y]
                               + M1[b, x] + M1[b, y] + M1[x, y])
                          for (x, y), r in h2 if len({a, b, x, y}) == 4)
                del_ = sum(r * (st.F[1] - u2[a] - u2[b] - u2[x] - u2[y] + M2[a, b] + M2[a, x] + M2[a, y]
                                + M2[b, x] + M2[b, y] + M2[x, y])
                           for (x, y), r in h1 if len({a, b, x, y}) == 4)
                cls[h] = [st.mass(a, b), dle + del_, len(h2) > 0]
            st.add(0, h1)
            st.add(1, h2)
            for h in hs:
                cls[h].append(st.mass(dense[h[0]], dense[h[1]]))
    full = _direct(order, dense, opp1, opp2, len(order))
    out = {}
    for h in trav:
        A, T1, opp2_present, C = cls[h]
        Z = full.mass(dense[h[0]], dense[h[1]])
        T2 = (C - A) - T1 if opp2_present else 0.0
        out[h] = (POT - BET) * A + (POT / 2 - BET) * T1 + (POT / 3 - BET) * T2 - BET * (Z - C)
    return out


@pytest.mark.parametrize("seed,nh,board,nruns", [
    (5, 12, None, 3), (6, 14, None, 7), (7, 10, None, 16),
    (8, 12, ["Ks", "Kd", "Kh", "Kc", "2s"], 4),
    (9, 10, ["As", "Ks", "Qs", "Js", "Ts"], 2),
])
def test_runs_from_direct_states_match_enumeration(seed, nh, board, nruns):
    b = None if board is None else [card_to_int(c) for c in board]
    strength, order, dense, trav, opp1, opp2 = _setup(seed, nh, b)
    want = _brute(strength, trav, opp1, opp2)
    got = _sweep_runs(strength, order, dense, trav, opp1, opp2, nruns)
    scale = max(1.0, max(abs(v) for v in want.values()))
    for h in trav:
        assert abs(got[h] - want[h]) <= 1e-9 * scale, (h, got[h], want[h])


def test_direct_state_equals_incremental():
    strength, order, dense, trav, opp1, opp2 = _setup(10, 40, None)
    inc = Sweep()
    inc.add(0, [((dense[c[0]], dense[c[1]]), opp1[c]) for c in order if opp1.get(c, 0.0) > 0])
    inc.add(1, [((dense[c[0]], dense[c[1]]), opp2[c]) for c in order if opp2.get(c, 0.0) > 0])
    dr = _direct(order, dense, opp1, opp2, len(order))
    for a, b in [(inc.P, dr.P), (inc.w, dr.w), (inc.d, dr.d), (inc.u[0], dr.u[0]), (inc.u[1], dr.u[1])]:
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12)
    assert abs(inc.Q - dr.Q) < 1e-9 and abs(inc.Dd - dr.Dd) < 1e-9
    assert abs(inc.F[0] - dr.F[0]) < 1e-9 and abs(inc.F[1] - dr.F[1]) < 1e-9
