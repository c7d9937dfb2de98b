"""Batched and served forms: every subgame's result must be the same whether
it is solved alone or together with others (the batch merges launches, not
arithmetic -- three-way showdown sweeps keep each subgame's own run merge),
and retirement at an exploitability target must hold."""
import numpy as np
import pytest

import workloads as wl


def mixed_subgames():
    """Subgames of different street, player count, tree shape and range size."""
    specs = [
        ("hu_river", 41, 60, {}),
        ("hu_river", 42, 150, {"bet_sizes": [0.33, 0.75, 1.5], "max_raises": 3}),
        ("turn3", 43, 12, {"bet_sizes": [0.75], "max_raises": 2}),
        ("turn3", 44, 16, {"bet_sizes": [0.5, 1.0], "max_raises": 1}),
        ("hu_river", 45, 90, {"bet_sizes": [1.0], "max_raises": 1}),
    ]
    subs = []
    for name, seed, nh, over in specs:
        cfg = wl.config(name, seed=seed, num_hands=nh, **over)
        sg = wl.AbiSubgame(cfg, max_hands=200)
        sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
        subs.append(sg)
    # a 3-player river (three-way showdowns)
    cfg = wl.config("river6", seed=47, num_players=3, bet_sizes=[1.0], max_raises=1)
    cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(47), cfg["board"], 3, 50)
    sg = wl.AbiSubgame(cfg, max_hands=200)
    subs.append(sg)
    # a heads-up turn with continuation leaves
    cfg = wl.config("hu_river", seed=46, num_hands=40)
    cfg["board"] = cfg["board"][:4]
    cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(46), cfg["board"], 2, 40)
    sg = wl.AbiSubgame(cfg, max_hands=200)
    sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
    subs.append(sg)
    return subs


def identical(a, b):
    for k in ("root_strategy", "root_ev", "avg_strategies", "avg_node_ids"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.gpu
def test_batch_equals_alone():
    subs = mixed_subgames()
    rc, together = wl.batch_solve(subs, 37, graph_iterations=10)
    assert rc == 0, wl.ssg.last_error(subs[0].lib)
    for sg, r in zip(subs, together):
        rc, alone = sg.solve(37)
        assert rc == 0
        identical(r, alone)
        assert r["stats"]["iterations_run"] == 37
    for sg in subs:
        sg.free()


@pytest.mark.gpu
@pytest.mark.parametrize("count", [3, 15])
def test_batch_many_sweeps_equal_alone(count):
    # full-range 3-player rivers, 40 three-way showdowns per traverser each:
    # 3 or 15 of them in one launch (120 / 600 terminals) -- each sweep still
    # uses its own subgame's run split, so results are identical to solos
    subs = []
    for seed in range(71, 71 + count):
        cfg = wl.config("river6", seed=seed, num_players=3)
        cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(seed), cfg["board"], 3, None)
        subs.append(wl.AbiSubgame(cfg, max_hands=1326))
    rc, together = wl.batch_solve(subs, 37, graph_iterations=10)
    assert rc == 0, wl.ssg.last_error(subs[0].lib)
    for sg, r in zip(subs, together):
        rc, alone = sg.solve(37)
        assert rc == 0
        identical(r, alone)
    for sg in subs:
        sg.free()


@pytest.mark.gpu
def test_batch_retires_at_target():
    subs = mixed_subgames()[:3]
    rc, res = wl.batch_solve(subs, 1500, target=1.0, check_every=25)
    assert rc == 0, wl.ssg.last_error(subs[0].lib)
    for r in res:
        st = r["stats"]
        assert 0 <= st["exploitability_pct"] <= 1.0 or st["iterations_run"] == 1500
        assert st["iterations_run"] % 25 == 0
    for sg in subs:
        sg.free()


@pytest.mark.gpu
def test_server_alone_equals_mix():
    subs = mixed_subgames()
    lib = subs[0].lib
    alone = []
    for sg in subs:
        srv = wl.Server(lib, block_iterations=25, target_exploitability=2.0, max_iterations=300)
        rid = srv.submit(sg)
        alone.append(srv.wait(rid, sg.nh))
        srv.close()
    srv = wl.Server(lib, block_iterations=25, target_exploitability=2.0, max_iterations=300)
    ids = [srv.submit(sg) for sg in subs]
    mixed = [srv.wait(i, sg.nh) for i, sg in zip(ids, subs)]
    srv.close()
    for a, m in zip(alone, mixed):
        identical(a, m)
        assert a["stats"]["iterations_run"] == m["stats"]["iterations_run"]
        assert m["latency_ms"] > 0
    for sg in subs:
        sg.free()


@pytest.mark.gpu
def test_server_arrival_while_running_equals_alone():
    """Continuous batching: the second request is submitted only once the
    first has run at least one block on the GPU (and is still running), so
    it joins a batch in flight; both results equal their solo results."""
    subs = mixed_subgames()
    first, second = subs[1], subs[6]
    lib = first.lib
    kw = dict(block_iterations=25, target_exploitability=0.05, max_iterations=400)
    alone = []
    for sg in (first, second):
        srv = wl.Server(lib, **kw)
        alone.append(srv.wait(srv.submit(sg), sg.nh))
        srv.close()
    assert alone[0]["stats"]["iterations_run"] >= 75   # the first runs several blocks alone
    srv = wl.Server(lib, **kw)
    a = srv.submit(first)
    import time
    t0 = time.time()
    while True:
        state, its = srv.progress(a)
        if its >= 25:
            break
        assert time.time() - t0 < 60, "first request never ran a block"
        time.sleep(0.001)
    assert state == 1 and its < alone[0]["stats"]["iterations_run"]
    b = srv.submit(second)
    mixed = [srv.wait(a, first.nh), srv.wait(b, second.nh)]
    srv.close()
    for x, m in zip(alone, mixed):
        identical(x, m)
        assert x["stats"]["iterations_run"] == m["stats"]["iterations_run"]
        assert x["stats"]["exploitability_pct"] == pytest.approx(m["stats"]["exploitability_pct"], rel=1e-9)
    for sg in subs:
        sg.free()


@pytest.mark.gpu
def test_server_memory_budget_queues_requests():
    # a tiny budget admits one request at a time; all still finish
    subs = mixed_subgames()[:3]
    srv = wl.Server(subs[0].lib, memory_budget_gb=0.001, block_iterations=25, target_exploitability=5.0,
                    max_iterations=100)
    ids = [srv.submit(sg) for sg in subs]
    res = [srv.wait(i, sg.nh) for i, sg in zip(ids, subs)]
    srv.close()
    assert all(r["stats"]["iterations_run"] > 0 for r in res)
    for sg in subs:
        sg.free()


@pytest.mark.gpu
def test_server_failure_retires_only_that_request():
    """A request whose leaf values hold NaN fails with its own error (its
    exploitability is not finite) while the requests batched with it finish
    with their solo results."""
    subs = mixed_subgames()
    good = [subs[2], subs[6]]
    lib = good[0].lib
    cfg = wl.config("turn3", seed=48, num_hands=12, bet_sizes=[0.75], max_raises=2)
    bad = wl.AbiSubgame(cfg, max_hands=200)
    lv = wl.leaf_values_for(cfg, bad.num_leaves)
    lv[:, :, 3] = np.nan
    bad.set_leaf_values(lv)
    kw = dict(block_iterations=25, target_exploitability=2.0, max_iterations=300)
    alone = []
    for sg in good:
        srv = wl.Server(lib, **kw)
        alone.append(srv.wait(srv.submit(sg), sg.nh))
        srv.close()
    srv = wl.Server(lib, **kw)
    ids = [srv.submit(good[0]), srv.submit(bad), srv.submit(good[1])]
    first = srv.wait(ids[0], good[0].nh)
    with pytest.raises(RuntimeError, match="non-finite"):
        srv.wait(ids[1], bad.nh)
    last = srv.wait(ids[2], good[1].nh)
    srv.close()
    for a, m in zip(alone, (first, last)):
        identical(a, m)
        assert a["stats"]["iterations_run"] == m["stats"]["iterations_run"]
    for sg in subs + [bad]:
        sg.free()
