"""CPU check of the card-removal algebra for more than two counted
opponents, the form a future kernel for 4-player folds and leaves would
evaluate (the reference enumerates opponent tuples, street_solve.cu:771-823
and :1079-1127, which is out of reach at full range size).

Two opponents with symmetric combo matrices A, B (zero diagonal) and every
hand avoiding a card set S:
  D2(S) = F_A(S) F_B(S) - Q(S) + E(S),
  F_A(S) = F_A - sum_{c in S} u_A(c) + sum_{pairs in S} A,
  Q(S)   = Q - sum_{e in S} w(e) + sum_{e, f in S} P[e][f]
           - sum_{c in S} u~_A(c) u~_B(c),   u~_A(c) = u_A(c) - sum_{e in S} A[c][e],
  E(S)   = E - sum_{c in S} d(c) + sum_{pairs in S} A B,
with u = M 1, F = sum u / 2, P = A B, w = A u_B + B u_A, Q = u_A . u_B,
d = diag P, E = <A, B> / 2: O(|S|^2) lookups once P, w, u, d are known.
Three opponents: condition on the third opponent's hand,
  D3(h) = sum_{o3 disjoint from h} C(o3) D2(h + o3),
O(H) per traverser hand instead of O(H^2).  Checked against brute-force
enumeration of disjoint tuples on small decks."""
import itertools

import numpy as np
import pytest


def rand_matrix(rng, n, density):
    M = np.zeros((n, n))
    for x in range(n):
        for y in range(x + 1, n):
            if rng.random() < density:
                M[x, y] = M[y, x] = rng.uniform(0, 1)
    return M


class TwoOpp:
    """Aggregates of two opponents' matrices for avoid-set queries."""

    def __init__(self, A, B):
        self.A, self.B = A, B
        self.uA, self.uB = A.sum(1), B.sum(1)
        self.FA, self.FB = self.uA.sum() / 2, self.uB.sum() / 2
        self.P = A @ B
        self.w = A @ self.uB + B @ self.uA
        self.Q = float(self.uA @ self.uB)
        self.d = np.diag(self.P).copy()
        self.E = float((A * B).sum()) / 2

    def mass(self, S):
        A, B, S = self.A, self.B, sorted(set(S))
        pairs = list(itertools.combinations(S, 2))
        FA = self.FA - sum(self.uA[c] for c in S) + sum(A[c, e] for c, e in pairs)
        FB = self.FB - sum(self.uB[c] for c in S) + sum(B[c, e] for c, e in pairs)
        Q = self.Q - sum(self.w[e] for e in S) + sum(self.P[e, f] for e in S for f in S)
        Q -= sum((self.uA[c] - sum(A[c, e] for e in S)) * (self.uB[c] - sum(B[c, e] for e in S)) for c in S)
        E = self.E - sum(self.d[c] for c in S) + sum(A[c, e] * B[c, e] for c, e in pairs)
        return FA * FB - Q + E


def hands(M):
    n = M.shape[0]
    return [((x, y), M[x, y]) for x in range(n) for y in range(x + 1, n) if M[x, y] > 0]


def brute(mats, S):
    """Sum over pairwise disjoint tuples (one hand per opponent) avoiding S."""
    lists = [[(h, r) for h, r in hands(M) if not set(h) & set(S)] for M in mats]
    tot = 0.0
    for combo in itertools.product(*lists):
        cards = [c for h, _ in combo for c in h]
        if len(set(cards)) == len(cards):
            tot += float(np.prod([r for _, r in combo]))
    return tot


def three_opp(two, C, h):
    tot = 0.0
    for (x, y), r in hands(C):
        if x in h or y in h:
            continue
        tot += r * two.mass(list(h) + [x, y])
    return tot


@pytest.mark.parametrize("seed,n,density", [(0, 10, 0.6), (1, 12, 0.4), (2, 9, 0.9)])
def test_two_opponents_any_avoid_set(seed, n, density):
    rng = np.random.default_rng(seed)
    A, B = rand_matrix(rng, n, density), rand_matrix(rng, n, density)
    two = TwoOpp(A, B)
    for size in (0, 1, 2, 3, 4, 6):
        for _ in range(4):
            S = [int(c) for c in rng.choice(n, size, replace=False)]
            want = brute([A, B], S)
            assert abs(two.mass(S) - want) <= 1e-9 * max(1.0, want), (S, two.mass(S), want)


@pytest.mark.parametrize("seed,n,density", [(3, 10, 0.5), (4, 11, 0.35)])
def test_three_opponents_by_conditioning(seed, n, density):
    rng = np.random.default_rng(seed)
    A, B, C = (rand_matrix(rng, n, density) for _ in range(3))
    two = TwoOpp(A, B)
    for a, b in [(0, 1), (2, 7), (n - 2, n - 1)]:
        want = brute([A, B, C], [a, b])
        got = three_opp(two, C, (a, b))
        assert abs(got - want) <= 1e-9 * max(1.0, want), ((a, b), got, want)


def test_two_opponent_form_matches_the_kernel_closed_form():
    # |S| = 2 reproduces the closed form the two-opponent kernel evaluates per
    # traverser hand (a, b): A1 A2 + (D - Q) + g(a) + g(b) - m2 (u1(a) + u1(b))
    # - m1 (u2(a) + u2(b)) + 3 m1 m2 - P[a][b] - P[b][a], g = u1 u2 + w - 2 d
    rng = np.random.default_rng(5)
    n = 12
    A, B = rand_matrix(rng, n, 0.5), rand_matrix(rng, n, 0.5)
    two = TwoOpp(A, B)
    g = two.uA * two.uB + two.w - 2 * two.d
    for a, b in [(0, 1), (3, 9), (10, 11)]:
        m1, m2 = A[a, b], B[a, b]
        A1 = two.FA - two.uA[a] - two.uA[b] + m1
        A2 = two.FB - two.uB[a] - two.uB[b] + m2
        k = (A1 * A2 + (two.E - two.Q) + g[a] + g[b] - m2 * (two.uA[a] + two.uA[b])
             - m1 * (two.uB[a] + two.uB[b]) + 3 * m1 * m2 - two.P[a, b] - two.P[b, a])
        assert abs(k - two.mass([a, b])) <= 1e-9 * max(1.0, abs(k))


# ---------------------------------------------------------------------------
# Three opponents for every traverser hand at once, as matrix contractions.
# Cluster expansion of the pairwise disjointness over the opponents' hands:
#   prod_{i<j} (1 - c_ij), c_ij = [o_i and o_j share a card]
# gives, with every hand avoiding h = {a, b} (superscript h),
#   D3 = F_A F_B F_C - W_AB F_C - W_AC F_B - W_BC F_A
#        + S_A(B, C) + S_B(A, C) + S_C(A, B) - T3,
#   W_XY     = sum_c u_X u_Y - <X, Y> / 2          (pairs sharing a card)
#   S_X(Y,Z) = sum_{o} X(o) t_Y(o) t_Z(o),  t_Y({x, y}) = u_Y(x) + u_Y(y) - Y_xy
#   T3       = sum_c u_A u_B u_C - sum_{x<y} A B C + tr(A B C)
# (three pairwise-intersecting 2-card hands share one card or form a
# triangle).  Each piece is a sum over card indices with the factor
# r(x) = 1 - [x = a] - [x = b] on every summed index; multiplying those out
# turns every term into a contraction with free indices (a, b): O(n^3) per
# term and terminal, for all traverser hands together.
# ---------------------------------------------------------------------------


class Terms:
    """Sums of products of matrices over card indices: a term is
    (coefficient, [(matrix name, (i, j))], summed indices); every summed
    index carries the avoid-h factor r()."""

    def __init__(self, terms=None):
        self.terms = terms or []

    _fresh = [0]

    @classmethod
    def sym(cls):
        cls._fresh[0] += 1
        return f"s{cls._fresh[0]}"

    @classmethod
    def base(cls, coef, factors, summed):
        return cls([(coef, list(factors), list(summed))])

    def __add__(self, o):
        return Terms(self.terms + o.terms)

    def __mul__(self, o):
        if not isinstance(o, Terms):
            return Terms([(c * o, f, s) for c, f, s in self.terms])
        return Terms([(c1 * c2, f1 + f2, s1 + s2) for c1, f1, s1 in self.terms for c2, f2, s2 in o.terms])

    __rmul__ = __mul__

    def __neg__(self):
        return self * -1.0

    def __sub__(self, o):
        return self + (-o)

    def evaluate(self, mats, n):
        """Matrix over (a, b): the sum with r() expanded, by einsum."""
        out = np.zeros((n, n))
        for coef, factors, summed in self.terms:
            for choice in itertools.product((None, "a", "b"), repeat=len(summed)):
                sub = {s: (s if c is None else c) for s, c in zip(summed, choice)}
                sign = (-1.0) ** sum(c is not None for c in choice)
                idx = [tuple(sub.get(i, i) for i in ij) for _, ij in factors]
                names = sorted({i for ij in idx for i in ij})
                letter = {nm: chr(ord("c") + k) for k, nm in enumerate(n_ for n_ in names if n_ not in "ab")}
                letter.update({"a": "a", "b": "b"})
                free = "".join(x for x in "ab" if x in names)
                spec = ",".join("".join(letter[i] for i in ij) for ij in idx) + "->" + free
                val = np.einsum(spec, *[mats[m] for m, _ in factors], optimize=True)
                if free == "ab":
                    out += sign * coef * val
                elif free == "a":
                    out += sign * coef * val[:, None]
                elif free == "b":
                    out += sign * coef * val[None, :]
                else:
                    out += sign * coef * val
        return out


def F(X):
    x, y = Terms.sym(), Terms.sym()
    return Terms.base(0.5, [(X, (x, y))], [x, y])


def W(X, Y):
    c, y, z, x2, y2 = (Terms.sym() for _ in range(5))
    q = Terms.base(1.0, [(X, (c, y)), (Y, (c, z))], [c, y, z])
    e = Terms.base(0.5, [(X, (x2, y2)), (Y, (x2, y2))], [x2, y2])
    return q - e


def star(X, Y, Z):
    # 1/2 sum_{x,y} X_xy (sum_z Y_xz + sum_z Y_yz - Y_xy) (same for Z)
    x, y = Terms.sym(), Terms.sym()

    def t(M):
        z1, z2 = Terms.sym(), Terms.sym()
        return (Terms.base(1.0, [(M, (x, z1))], [z1]) + Terms.base(1.0, [(M, (y, z2))], [z2])
                - Terms.base(1.0, [(M, (x, y))], []))

    return Terms.base(0.5, [(X, (x, y))], [x, y]) * t(Y) * t(Z)


def triangle(A, B, C):
    c, y, z, w = (Terms.sym() for _ in range(4))
    common = Terms.base(1.0, [(A, (c, y)), (B, (c, z)), (C, (c, w))], [c, y, z, w])
    x2, y2 = Terms.sym(), Terms.sym()
    same = Terms.base(0.5, [(A, (x2, y2)), (B, (x2, y2)), (C, (x2, y2))], [x2, y2])
    p, q, r = Terms.sym(), Terms.sym(), Terms.sym()
    cyc = Terms.base(1.0, [(A, (p, q)), (B, (q, r)), (C, (r, p))], [p, q, r])
    return common - same + cyc


def d3_contracted():
    return (F("A") * F("B") * F("C") - W("A", "B") * F("C") - W("A", "C") * F("B") - W("B", "C") * F("A")
            + star("A", "B", "C") + star("B", "A", "C") + star("C", "A", "B") - triangle("A", "B", "C"))


@pytest.mark.parametrize("seed,n,density", [(6, 9, 0.6), (7, 10, 0.4)])
def test_three_opponents_as_contractions(seed, n, density):
    rng = np.random.default_rng(seed)
    A, B, C = (rand_matrix(rng, n, density) for _ in range(3))
    D3 = d3_contracted().evaluate({"A": A, "B": B, "C": C}, n)
    two = TwoOpp(A, B)
    for a in range(n):
        for b in range(a + 1, n):
            want = three_opp(two, C, (a, b))
            assert abs(D3[a, b] - want) <= 1e-9 * max(1.0, abs(want)), ((a, b), D3[a, b], want)
    # and one hand against enumeration directly
    assert abs(D3[1, 4] - brute([A, B, C], [1, 4])) <= 1e-9 * max(1.0, abs(D3[1, 4]))
