"""Card helpers with the reference conventions (python/solver.py:20-107).

card = rank * 4 + suit, ranks "23456789TJQKA" = 0..12, suits "cdhs" = 0..3.
parse_range_string accepts the same PioSOLVER-style syntax as the reference:
specific combos ("AhKh", optionally ":0.5" weighted), suited / offsuit groups
("AKs", "AKo"), pairs ("QQ"), comma separated; duplicates are dropped, first
occurrence wins, and combos are returned as (low card, high card, weight).
"""
RANKS = "23456789TJQKA"
SUITS = "cdhs"
_RANK = {r: i for i, r in enumerate(RANKS)}
_SUIT = {s: i for i, s in enumerate(SUITS)}


def card_to_int(card_str):
    """'Ah' -> 50."""
    if len(card_str) < 2 or card_str[0] not in _RANK or card_str[1] not in _SUIT:
        raise ValueError(f"Invalid card: {card_str}")
    return _RANK[card_str[0]] * 4 + _SUIT[card_str[1]]


def int_to_card(card):
    """50 -> 'Ah'."""
    return RANKS[card >> 2] + SUITS[card & 3]


def _group(token, weight):
    """Expand one range token into (c0, c1, weight) tuples."""
    if len(token) == 4:
        a, b = card_to_int(token[:2]), card_to_int(token[2:])
        return [(min(a, b), max(a, b), weight)]
    if len(token) == 3:
        r0, r1, kind = _RANK.get(token[0], -1), _RANK.get(token[1], -1), token[2]
        if r0 < 0 or r1 < 0:
            return []
        if kind == "s":
            return [(min(r0 * 4 + s, r1 * 4 + s), max(r0 * 4 + s, r1 * 4 + s), weight)
                    for s in range(4) if r0 != r1]
        if kind == "o":
            out = []
            for s0 in range(4):
                for s1 in range(4):
                    if s0 != s1:
                        a, b = r0 * 4 + s0, r1 * 4 + s1
                        out.append((min(a, b), max(a, b), weight))
            return out
        return []
    if len(token) == 2:
        r0, r1 = _RANK.get(token[0], -1), _RANK.get(token[1], -1)
        if r0 < 0 or r0 != r1:
            return []
        return [(r0 * 4 + s0, r0 * 4 + s1, weight) for s0 in range(4) for s1 in range(s0 + 1, 4)]
    return []


def parse_range_string(range_str):
    """'AA,AKs:0.5' -> [(c0, c1, w), ...] without duplicate combos."""
    out, seen = [], set()
    for part in (range_str or "").split(","):
        part = part.strip()
        if not part:
            continue
        weight = 1.0
        if ":" in part:
            part, w = part.rsplit(":", 1)
            try:
                weight = float(w)
            except ValueError:
                pass
        for c0, c1, w in _group(part, weight):
            key = (min(c0, c1), max(c0, c1))
            if key not in seen:
                seen.add(key)
                out.append((key[0], key[1], w))
    return out
