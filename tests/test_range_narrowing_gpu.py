"""Range narrowing on the device (ss_session_narrow) against the reference's
host path over the same solve.

The reference narrows between streets by copying the solve's average
strategies to the host, reading the solver player's first decision node
(get_avg_strategy: frequencies above 0.001 per label, keyed by the combo),
turning it into P(action | hand) (python/hud_solver.py:355-360) and calling
RangeNarrower.update (python/range_narrowing.py:83-130; the host mirror here
is pinned to it bit for bit by tests/test_range_narrowing.py).  The device
form reads the session's strategy sums in place; both must give the same
weights bit for bit.
"""
import numpy as np
import pytest

import range_narrowing as rn
import street_solver_gpu as ssg
import workloads as wl


def host_path(nr, key, solver, player, action):
    probs = {k: v.get(action, 0.0) for k, v in solver.get_avg_strategy(player).items()}
    if not any(v > 0 for v in probs.values()):
        return False
    nr.update(key, action, probs)
    return True


def solver_for(cfg, iters):
    ranges = [[(int(a), int(b), float(w)) for (a, b), w in zip(h, ws)]
              for h, ws in zip(cfg["hands"], cfg["weights"])]
    rng = np.random.default_rng(cfg["seed"])

    def leaf_fn(tree, player_hands, max_h, pot):   # turn subgames: seeded continuation values
        return rng.normal(0.0, 0.3 * pot, (tree.num_leaves, len(player_hands), max_h)).astype(np.float32)

    s = ssg.StreetSolverGPU(board=cfg["board"], pot_bb=cfg["pot"] / 100, stack_bb=cfg["stack"] / 100,
                            player_ranges=ranges, bet_sizes=cfg["bet_sizes"], max_hands=1326,
                            leaf_value_fn=leaf_fn)
    s.solve(iterations=iters, resident=True)
    return s


def narrowers(board):
    a = rn.RangeNarrower()
    a.set_uniform_range("villain")                # every combo, board-blocked ones included
    rng = np.random.default_rng(5)
    hands = [(c1, c0, float(rng.random())) if rng.random() < 0.05 else (c0, c1, float(rng.random()) * (rng.random() > 0.1))
             for c0, c1, _ in rn.generate_all_hands(board) if rng.random() < 0.5]
    b = rn.RangeNarrower()
    b.set_initial_range("villain", hands)         # entries with c0 > c1 and zero weights
    return [a, b]


@pytest.mark.gpu
@pytest.mark.parametrize("name,seed,nh,over,player", [
    ("hu_river", 61, 300, {}, 1),
    ("hu_river", 62, None, {}, 0),
    ("turn3", 63, 120, {"bet_sizes": [0.75], "max_raises": 1}, 2),
])
def test_device_narrowing_equals_reference_host_path(name, seed, nh, over, player):
    cfg = wl.config(name, seed=seed, num_hands=nh, **over)
    s = solver_for(cfg, 40)
    node = next(int(s._output.avg_strategy_node_ids[d]) for d in range(s._output.num_avg_nodes)
                if s._tree.nodes[s._output.avg_strategy_node_ids[d]].player == player)
    labels = ssg._build_labels_at_node(s._tree, node)
    checked = 0
    for action in labels + ["Raise 999%"]:
        for nr in narrowers(cfg["board"]):
            dev, host = nr.copy(), nr.copy()
            a = rn.narrow_from_solver(dev, "villain", s, player, action)
            b = host_path(host, "villain", s, player, action)
            assert a == b, action
            assert [float(w).hex() for _, _, w in dev._ranges["villain"]] == \
                   [float(w).hex() for _, _, w in host._ranges["villain"]], action
            assert dev.get_action_log("villain") == host.get_action_log("villain")
            checked += a
    assert checked >= 2
    s.free()
