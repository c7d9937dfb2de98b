"""Range narrowing between streets, with the solve's side on the GPU.

Same interface as the reference module python/range_narrowing.py
(RangeNarrower :35-208, generate_all_hands :211-232, make_blueprint_probs
:235-264): a per-player list of (card0, card1, weight) entries, Bayesian
updates w' = w * P(action | hand) with a floor of 0.005 for entries that had
weight, then scaling so the largest weight is 1.

Where the probabilities come from the street solver's own average strategy
(python/hud_solver.py:345-362, the production path), narrow_from_solver()
runs the update on the device through ss_session_narrow: the solve's
strategy sums stay resident in the session and only the range crosses to the
host -- the reference instead copies every average strategy to the host,
builds a Python dictionary per hand and loops over it.  Both give the same
weights bit for bit (FP64 in both).  RangeNarrower.update() keeps the
reference's host update for probabilities from other sources (blueprints),
which are not part of this path.
"""
WEIGHT_FLOOR = 0.005      # python/range_narrowing.py:47


class RangeNarrower:
    """Bayesian range tracker for several players across streets."""

    WEIGHT_FLOOR = WEIGHT_FLOOR

    def __init__(self):
        self._ranges = {}
        self._action_log = {}

    def set_initial_range(self, player, hands):
        self._ranges[player] = [(c0, c1, w) for c0, c1, w in hands]
        self._action_log[player] = []

    def set_uniform_range(self, player):
        self._ranges[player] = [(a, b, 1.0) for a in range(52) for b in range(a + 1, 52)]
        self._action_log[player] = []

    def update(self, player, action, blueprint_probs):
        """w' = w * P(action | (c0, c1)), P = 1 / max(#distinct P, 2) for an
        entry missing from blueprint_probs; floor, then scale to a maximum of
        1 (python/range_narrowing.py:83-130)."""
        if player not in self._ranges:
            return
        fallback = 1.0 / max(len(set(blueprint_probs.values())), 2)
        out = []
        for c0, c1, w in self._ranges[player]:
            p = blueprint_probs.get((c0, c1))
            nw = w * (fallback if p is None else p)
            if nw < WEIGHT_FLOOR and w > 0:
                nw = WEIGHT_FLOOR
            out.append((c0, c1, nw))
        self._set_scaled(player, out)
        self._action_log.setdefault(player, []).append(action)

    def _set_scaled(self, player, entries):
        top = max(w for _, _, w in entries) if entries else 1.0
        self._ranges[player] = [(c0, c1, w / top) for c0, c1, w in entries] if top > 0 else entries

    def remove_folded_hands(self, player, blueprint_probs):
        """Drop entries with P(fold | hand) >= 0.95 (python/range_narrowing.py:132-156)."""
        if player not in self._ranges:
            return
        self._ranges[player] = [(c0, c1, w) for c0, c1, w in self._ranges[player]
                                if blueprint_probs.get((c0, c1), 0) < 0.95]

    def get_weighted_hands(self, player):
        return sorted(self._ranges.get(player, []), key=lambda e: -e[2])

    def get_hand_count(self, player):
        return sum(1 for _, _, w in self._ranges.get(player, []) if w > WEIGHT_FLOOR)

    def get_action_log(self, player):
        return self._action_log.get(player, [])

    def copy(self):
        new = RangeNarrower()
        new._ranges = {p: list(h) for p, h in self._ranges.items()}
        new._action_log = {p: list(a) for p, a in self._action_log.items()}
        return new


def narrow_from_solver(narrower, player_key, solver, solve_player, action, node=None):
    """The production update (python/hud_solver.py:345-362 then
    RangeNarrower.update): P(action | hand) from `solver`'s average strategy
    of `solve_player` at its first decision node (or `node`), on the device.
    `solver` is a StreetSolverGPU solved with resident=True.  Returns True
    when the update was applied, False when no probability was positive (the
    range is then unchanged and the reference falls back to other sources)."""
    if player_key not in narrower._ranges:
        return False
    entries = narrower._ranges[player_key]
    applied, weights = solver.narrow_weights(solve_player, action, [(c0, c1) for c0, c1, _ in entries],
                                             [w for _, _, w in entries], node=node)
    if not applied:
        return False
    narrower._ranges[player_key] = [(c0, c1, w) for (c0, c1, _), w in zip(entries, weights)]
    narrower._action_log.setdefault(player_key, []).append(action)
    return True


def generate_all_hands(board_cards=None):
    """Every 2-card combo without a board card, weight 1.0."""
    blocked = set(board_cards or [])
    return [(a, b, 1.0) for a in range(52) if a not in blocked for b in range(a + 1, 52) if b not in blocked]


def make_blueprint_probs(hand_strategies, action):
    """{(c0, c1): P(action)} from {"AhKs": {"actions": [{"action", "frequency"}]}}: the
    first listed action whose name contains `action` (case-insensitive)."""
    try:
        from cards import card_to_int
    except ImportError:  # imported as part of a package
        from .cards import card_to_int
    out = {}
    for hand, strat in hand_strategies.items():
        a, b = card_to_int(hand[:2]), card_to_int(hand[2:])
        p = 0.0
        for act in strat.get("actions", []):
            if action.lower() in act.get("action", "").lower():
                p = act.get("frequency", 0.0)
                break
        out[(min(a, b), max(a, b))] = p
    return out

