"""Test infrastructure: a restatement of the reference's turn and flop
leaf-value producers (python/leaf_values.py), the input a depth-limited turn
or flop subgame takes for its continuation leaves.  Only tests/ use it, as the checker of a
future device producer; tests/golden/make_leaf_golden.py pins it against the
reference module itself (leaf_values_*.npz).

Per turn leaf (one per betting-tree leaf, before the continuation
expansion) and each of the 4^N continuation bias profiles:
  value(p, h) = first-order bias adjustment of hand h's river equity at the
                leaf's pot,
where the equity is averaged over the runouts -- river cards of a turn (all
of them, or 12 drawn with numpy's RandomState(42) when some range holds
more than 50 hands), turn and river cards of a flop (likewise sampled) -- of the
unweighted share of opponent hand tuples the hand beats (ties split), with
the tuples enumerated when there are at most 2000 of them and otherwise 2000
drawn with Python's random.Random(42), as the reference does.  Hand
strengths come from the oracle's evaluator (pinned to src/hand_eval.h); the
golden script checks that it orders hands as the reference module's own
evaluator does."""
import itertools
import random

import numpy as np

from oracle.oracle import Oracle

# per bias profile (0 unmodified, 1 fold, 2 call, 3 raise):
# leaf_values.py:86, :89
FOLD_PROB = (0.0, 0.35, 0.0, 0.0)
POT_FACTOR = (1.0, 0.7, 1.0, 1.4)
RIVER_SAMPLES = 12        # leaf_values.py:762
RANGE_SAMPLE_ABOVE = 50   # :763
TUPLE_LIMIT = 2000        # :617


def biased_value(equity, pot, s_self, s_opp):
    """leaf_values.py:91-121: with the opponent's fold probability the hand
    collects half the pot; otherwise (equity - 1/2) of the pot scaled by both
    profiles' pot factors."""
    fold = FOLD_PROB[s_opp]
    showdown = pot * (POT_FACTOR[s_self] * POT_FACTOR[s_opp])
    return fold * (0.5 * pot) + (1.0 - fold) * ((equity - 0.5) * showdown)


def leaf_infos(td, num_players):
    """leaf_values.py:189-262: (leaf index before the expansion, pot, bets)
    of every continuation chain -- N nested levels of 4-way decisions, the
    first owned by player 0, ending in leaves."""
    nodes, children = td.nodes, td.children

    def chain(x, depth):
        n = nodes[x]
        if n.type != 0 or n.num_children != 4:
            return False
        kids = [children[n.first_child + c] for c in range(4)]
        if depth == num_players - 1:
            return all(nodes[k].type == 4 for k in kids)
        return all(chain(k, depth + 1) for k in kids)

    per = 4 ** num_players
    out = []
    for x in range(td.num_nodes):
        n = nodes[x]
        if n.type != 0 or n.player != 0 or n.num_children != 4 or not chain(x, 0):
            continue
        y = x
        for _ in range(num_players):
            y = children[nodes[y].first_child]
        out.append((nodes[y].leaf_idx // per, n.pot, tuple(n.bets[p] for p in range(num_players))))
    return sorted(out, key=lambda t: t[0])


def _equity_one_runout(hero, hands, strength, raw, cnt):
    """leaf_values.py:573-691 for one river card: hero's share of the
    opponent tuples it beats, over tuples with no shared card."""
    mine = strength[hero]
    if not mine:
        return
    opps = [q for q in range(len(hands)) if q != hero]
    lists = [list(strength[q].keys()) for q in opps]
    total = 1
    for lst in lists:
        total *= len(lst)
    if total == 0:
        return
    if total <= TUPLE_LIMIT:
        tuples = list(itertools.product(*lists))
    else:
        rng = random.Random(42)
        tuples = [tuple(rng.choice(lst) for lst in lists) for _ in range(TUPLE_LIMIT)]
    for h, s in mine.items():
        c0, c1 = hands[hero][h][0], hands[hero][h][1]
        won, n = 0.0, 0
        for tup in tuples:
            cards = [c for q, o in zip(opps, tup) for c in hands[q][o][:2]]
            if c0 in cards or c1 in cards or len(set(cards)) < len(cards):
                continue
            best = max(strength[q][o] for q, o in zip(opps, tup))
            n += 1
            if s > best:
                won += 1.0
            elif s == best:
                won += 1.0 / (1 + sum(1 for q, o in zip(opps, tup) if strength[q][o] == s))
        if n > 0:
            raw[hero, h] += won / n
            cnt[hero, h] += 1.0


def turn_runouts(board4, player_hands):
    """River cards of a turn (leaf_values.py:754-770)."""
    on_board = set(board4)
    rivers = [c for c in range(52) if c not in on_board]
    if len(rivers) > RIVER_SAMPLES and any(len(h) > RANGE_SAMPLE_ABOVE for h in player_hands):
        rivers = sorted(np.random.RandomState(42).choice(rivers, RIVER_SAMPLES, replace=False))
    return [[int(r)] for r in rivers]


def flop_runouts(board3, player_hands):
    """Turn and river cards of a flop (leaf_values.py:479-499): 12 turn cards
    drawn with RandomState(42) and, per turn card tc, 12 river cards drawn
    with RandomState(43 + tc), when some range holds more than 50 hands."""
    on_board = set(board3)
    large = any(len(h) > RANGE_SAMPLE_ABOVE for h in player_hands)
    turns = [c for c in range(52) if c not in on_board]
    if len(turns) > RIVER_SAMPLES and large:
        turns = sorted(np.random.RandomState(42).choice(turns, RIVER_SAMPLES, replace=False))
    out = []
    for tc in turns:
        rivers = [c for c in range(52) if c not in on_board and c != tc]
        if len(rivers) > RIVER_SAMPLES and large:
            rivers = sorted(np.random.RandomState(43 + int(tc)).choice(rivers, RIVER_SAMPLES, replace=False))
        out.extend([int(tc), int(rc)] for rc in rivers)
    return out


def turn_leaf_values(board4, infos, max_hands, player_hands, oracle=None):
    """leaf_values.py:694-816: float32 [len(infos) * 4^N, N, max_hands];
    player_hands[p] = [(card, card, weight), ...]."""
    return _leaf_values(board4, turn_runouts(board4, player_hands), infos, max_hands, player_hands, oracle)


def flop_leaf_values(board3, infos, max_hands, player_hands, oracle=None):
    """leaf_values.py:408-571: the same over turn and river cards."""
    return _leaf_values(board3, flop_runouts(board3, player_hands), infos, max_hands, player_hands, oracle)


def _leaf_values(board, runouts, infos, max_hands, player_hands, oracle):
    orc = oracle or Oracle()
    N = len(player_hands)
    nh = [len(h) for h in player_hands]
    raw = np.zeros((N, max_hands), dtype=np.float64)
    cnt = np.zeros((N, max_hands), dtype=np.float64)
    for extra in runouts:
        b5 = list(board) + extra
        dead = set(b5)
        strength = []
        for p in range(N):
            strength.append({h: orc.eval7(b5 + [c0, c1]) for h, (c0, c1, _w) in enumerate(player_hands[p])
                             if c0 not in dead and c1 not in dead})
        for p in range(N):
            _equity_one_runout(p, player_hands, strength, raw, cnt)
    ok = cnt > 0
    raw[ok] /= cnt[ok]
    return _bias_rows(raw, infos, max_hands, nh)


def _bias_rows(raw, infos, max_hands, nh):
    """leaf_values.py:795-814: the rows of every leaf descriptor and profile."""
    N = len(nh)
    per = 4 ** N
    total = len(infos) * per
    out = np.zeros((total, N, max_hands), dtype=np.float32)
    for leaf, pot, _bets in infos:
        for combo in range(per):
            flat = leaf * per + combo
            if flat >= total:
                continue
            prof = [(combo // 4 ** i) % 4 for i in range(N)]
            for p in range(N):
                if N > 2:
                    s_opp = max(0, min(3, int(round(sum(prof[q] for q in range(N) if q != p) / (N - 1)))))
                else:
                    s_opp = prof[1 - p]
                m = min(nh[p], max_hands)
                # biased_value over the row: the same IEEE operations, element by element
                out[flat, p, :m] = biased_value(raw[p, :m], pot, prof[p], s_opp)
    return out


def _reference_tuples(lists):
    """leaf_values.py:603-629: the opponent tuples scored on one runout."""
    total = 1
    for lst in lists:
        total *= len(lst)
    if total == 0:
        return []
    if total <= TUPLE_LIMIT:
        return list(itertools.product(*lists))
    rng = random.Random(42)
    return [tuple(rng.choice(lst) for lst in lists) for _ in range(TUPLE_LIMIT)]


def leaf_values_vectorised(board, runouts, infos, max_hands, player_hands, oracle=None):
    """The same values as _leaf_values with numpy over (hero hand, tuple):
    per runout and hero player, the tuples' card masks, best strengths and
    tie counts, each hand's per-tuple credit (1, 1/k or 0), and the credits
    summed with a running sum in tuple order (np.cumsum adds left to right,
    like the reference's loop) -- fast enough for full-size ranges."""
    orc = oracle or Oracle()
    N = len(player_hands)
    nh = [len(h) for h in player_hands]
    raw = np.zeros((N, max_hands), dtype=np.float64)
    cnt = np.zeros((N, max_hands), dtype=np.float64)
    cards = [np.array([(int(h[0]), int(h[1])) for h in ph], dtype=np.int64).reshape(-1, 2) for ph in player_hands]
    one = np.uint64(1)
    bits = [(one << c[:, 0].astype(np.uint64)) | (one << c[:, 1].astype(np.uint64)) for c in cards]
    for extra in runouts:
        b5 = list(board) + list(extra)
        dead = set(b5)
        live = [np.array([h for h in range(nh[p]) if cards[p][h, 0] not in dead and cards[p][h, 1] not in dead],
                         dtype=np.int64) for p in range(N)]
        st = [np.zeros(nh[p], dtype=np.int64) for p in range(N)]
        for p in range(N):
            for h in live[p]:
                st[p][h] = orc.eval7(b5 + [int(cards[p][h, 0]), int(cards[p][h, 1])])
        for p in range(N):
            if not len(live[p]):
                continue
            opps = [q for q in range(N) if q != p]
            tup = _reference_tuples([live[q].tolist() for q in opps])
            if not tup:
                continue
            tup = np.array(tup, dtype=np.int64)
            mask = np.zeros(len(tup), dtype=np.uint64)
            clash = np.zeros(len(tup), dtype=bool)
            best = np.zeros(len(tup), dtype=np.int64)
            for k, q in enumerate(opps):
                b = bits[q][tup[:, k]]
                clash |= (mask & b) != 0
                mask |= b
                best = np.maximum(best, st[q][tup[:, k]])
            nbest = sum((st[q][tup[:, k]] == best).astype(np.int64) for k, q in enumerate(opps))
            hero = live[p]
            blocked = ((bits[p][hero][:, None] & mask[None, :]) != 0) | clash[None, :]
            hs = st[p][hero][:, None]
            credit = np.where(hs > best[None, :], 1.0, np.where(hs == best[None, :], 1.0 / (1.0 + nbest[None, :]), 0.0))
            credit[blocked] = 0.0
            valid = (~blocked).sum(axis=1)
            wins = np.cumsum(credit, axis=1)[:, -1]
            ok = valid > 0
            raw[p, hero[ok]] += wins[ok] / valid[ok]
            cnt[p, hero[ok]] += 1.0
    ok = cnt > 0
    raw[ok] /= cnt[ok]
    return _bias_rows(raw, infos, max_hands, nh)
